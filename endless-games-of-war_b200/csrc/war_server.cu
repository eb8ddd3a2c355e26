// war_server.cu — continuous batching of enumeration jobs (war_server_* in include/war.h).  No counterpart
// in the reference, which runs one job per process.
//
// Jobs of any n, mode, rule and rank range are submitted from any thread.  A worker thread admits them,
// in submission order, into resident accumulator slots on the device; the number of slots is what the
// device-memory budget allows, so a job waits in the queue until a slot (its accumulators) is free.
// Every "tick" the worker cuts the admitted jobs' remaining ranges into tasks (each a run of work units of
// one job, about task_ranks ranks), sharing the tick's rank budget round-robin so that a short job is not
// stuck behind a long one, and runs the whole tick as one launch per kernel variant: each block plays one
// task with the refill loop of war_refill.cuh and adds its results to that task's job slot.  Jobs of
// different n and mode therefore run side by side on the device.  Two ticks are in flight at a time (the
// next one is queued before the previous one is waited for), so the GPU does not wait for the host; a job
// whose last task was in a finished tick is read back, its slot freed and its result published.
//
// Jobs of the same n and rule share one cycle memo (war_refill.cuh): its entries are facts about n and the
// rule, so every job of that class, now and later, decides its games from what the earlier ones found.
// The tables come from one arena that war_server_create reserves inside the memory budget (after the
// accumulator slots); a class takes its table from the arena when its first job is admitted, cleared on
// the compute stream, and keeps it until the server ends.  The worker thread never calls cudaMalloc, which
// would synchronise the device in the middle of the tick stream.  A class whose table no longer fits runs
// without the memo.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>
#include "war_host.h"
#include "war_refill.cuh"

namespace war {

struct ServeTask {
    BatchArgs args;   // the job's parameters and this task's units
    u32 slot;         // accumulator slot of the job
    u32 pad;
    u64 counter;      // the task's work-unit counter (zero when uploaded)
};

template <int RULE, int G, bool CANON, bool SHAPE, bool EXTRA, int V>
__global__ void __launch_bounds__(G == 1 ? 1024 : 512) serve_kernel(ServeTask* __restrict__ tasks,
                                                                   DevAcc* __restrict__ slots) {
    extern __shared__ u32 sh[];
    __shared__ BatchArgs A;
    ServeTask* t = tasks + blockIdx.x;
    const u32* src = (const u32*)&t->args;
    for (int i = threadIdx.x; i < (int)(sizeof(BatchArgs) / 4); i += blockDim.x) ((u32*)&A)[i] = src[i];
    __syncthreads();
    refill_dispatch<RULE, G, CANON, SHAPE, EXTRA, V>(A, slots + t->slot, &t->counter, sh);
}

typedef void (*ServeFn)(ServeTask*, DevAcc*);

template <int RULE, int G, int V>
static ServeFn serve_pick(bool canon, bool shape, bool extra) {
    if (!canon) return extra ? serve_kernel<RULE, G, false, false, true, V> : serve_kernel<RULE, G, false, false, false, V>;
    if (shape) return extra ? serve_kernel<RULE, G, true, true, true, V> : serve_kernel<RULE, G, true, true, false, V>;
    return extra ? serve_kernel<RULE, G, true, false, true, V> : serve_kernel<RULE, G, true, false, false, V>;
}

// Launch shapes of the serving kernel: one game per thread, 256-thread blocks, the multiply-add turn form;
// latched records with the path memo where it applies (memo = 1: n <= 14 and a table), with the landmark
// memo for deals of n = 15 (memo = 2), latched records without a memo otherwise, and the immediate-record
// loop for the loop-shape test.
struct Variant {
    int canon, rule, shape, extra, memo;
    bool operator<(const Variant& o) const {
        return std::tie(canon, rule, shape, extra, memo) < std::tie(o.canon, o.rule, o.shape, o.extra, o.memo);
    }
    bool operator==(const Variant& o) const { return !(*this < o) && !(o < *this); }
    int games() const { return 1; }
    int threads() const { return 256; }
    ServeFn fn() const {
        const bool c = canon != 0;
        if (rule) return shape ? serve_pick<1, 1, 1>(c, true, extra)
                         : memo == 1 ? serve_pick<1, 1, 31>(c, false, extra)
                         : memo == 2 ? serve_pick<1, 1, 7>(c, false, extra) : serve_pick<1, 1, 3>(c, false, extra);
        return shape ? serve_pick<0, 1, 1>(c, true, extra)
                     : memo == 1 ? serve_pick<0, 1, 31>(c, false, extra)
                     : memo == 2 ? serve_pick<0, 1, 7>(c, false, extra) : serve_pick<0, 1, 3>(c, false, extra);
    }
};

struct SJob {
    war_job job;
    int state = 0;       // 0 queued, 1 running, 2 done, 3 failed
    int status = 0;
    double t_submit = 0, t_admit = 0, t_finish = 0;
    int slot = -1;
    Plan plan;
    u64 next_main = 0;
    bool extras_issued = false;
    u64 per_unit = 1;    // ranks per main unit
    BatchArgs base;
    Variant var;
    war_result* result = nullptr;
};

struct Tick {
    ServeTask* h_tasks = nullptr;   // pinned
    Unit* h_units = nullptr;        // pinned
    ServeTask* d_tasks = nullptr;
    Unit* d_units = nullptr;
    int ntasks = 0, nunits = 0;
    std::vector<std::pair<Variant, std::pair<int, int>>> groups;   // variant -> [first task, count)
    std::vector<u64> finishing;     // jobs whose last task is in this tick
    std::vector<u64> admitted;      // jobs whose slot is cleared before this tick
    cudaEvent_t ev = nullptr;
    bool in_flight = false;
};

}  // namespace war

struct war_server {
    war_server_cfg cfg;
    int device = 0, sm_count = 0, nslots = 0, max_tasks = 0, max_units = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::deque<uint64_t> pending;
    std::map<uint64_t, war::SJob> jobs;
    std::vector<int> free_slots;
    std::map<std::pair<int, int>, std::pair<u64*, int>> memos;   // (n, rule) -> (table, log2 words)
    u64* memo_arena = nullptr;      // reserved at create; tables are carved from it in admission order
    u64 arena_words = 0, arena_used = 0;
    DevAcc* d_slots = nullptr;
    DevAcc* h_slot = nullptr;   // pinned readback buffer
    cudaStream_t s_comp = nullptr, s_copy = nullptr;
    war::Tick ticks[2];
    uint64_t next_id = 1, nticks = 0, jobs_done = 0, peak_resident = 0, resident = 0;
    int fatal = 0;
    std::chrono::steady_clock::time_point t0;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace war {
namespace {

constexpr u64 TASK_RANKS = 1ull << 16;   // ranks per task (about 15 ms of one block's work at n = 13)
constexpr int UNITS_PER_EXTRA_CAP = 512;   // sizing of the per-tick extra-unit pool

void set_args(war_server* s, SJob& J) {
    const war_job& job = J.job;
    const bool canon = job.mode == WAR_CANON;
    BatchArgs& a = J.base;
    memset(&a, 0, sizeof a);
    fill_fact(a.fact);
    a.n = job.n;
    a.m = J.plan.m;
    a.hbins = job.hbins;
    a.dbins = job.dbins;
    a.blk = (job.flags & WAR_F_SHAPE) && canon ? (job.blk ? job.blk : (job.n & -job.n)) : 0;
    a.W = canon ? 128 : 32;
    a.defer = canon ? 16 : 8;
    a.tk.k16 = 16u; a.tk.km16 = (u32)-16; a.tk.k2p28 = 1u << 28; a.tk.k4 = 4u; a.tk.one = 1u;
    a.tk.c0 = 2 * job.n - 4; a.tk.end2 = (u32)(4 * job.n * job.n);
    a.half = (job.flags & WAR_F_HALF) ? 1 : 0;
    a.sample = (job.flags & WAR_F_SAMPLE) ? 1 : 0;
    a.distinct = (job.flags & WAR_F_DISTINCT) && canon ? 1 : 0;
    a.seed = job.seed;
    a.thr = ((u64)job.sample_ppm << 32) / 1000000u;
    J.var.canon = canon ? 1 : 0;
    J.var.rule = job.rule;
    J.var.shape = a.blk ? 1 : 0;
    J.var.extra = (a.distinct || a.sample) ? 1 : 0;
    J.var.memo = 0;
    const bool landmarks = !canon && job.n == 15;   // the landmark memo serves n = 15 deals
    if (!a.blk && job.n >= 4 && (job.n <= 14 || landmarks) && s->cfg.memo_bits >= 0) {
        // the class's table: 2^bits words, grown with n (about a thousandth of the class's rank space)
        const std::pair<int, int> cls(job.n, job.rule);
        auto it = s->memos.find(cls);
        if (it == s->memos.end()) {
            const int cap = s->cfg.memo_bits ? s->cfg.memo_bits : 28;
            int bits = std::max(12, std::min(cap, 4 + (int)std::ceil(std::log2((double)fact(job.n)) * 0.75)));
            // the largest table of at most 2^bits words that the arena still holds (at least 2^12 words)
            const u64 left = s->arena_words - s->arena_used;
            while (bits >= 12 && (1ull << bits) > left) bits--;
            u64* t = nullptr;
            if (bits >= 12) {
                t = s->memo_arena + s->arena_used;
                if (cudaMemsetAsync(t, 0, sizeof(u64) << bits, s->s_comp) != cudaSuccess) {
                    t = nullptr;
                    cudaGetLastError();   // not cleared: the class runs without the memo
                } else {
                    s->arena_used += 1ull << bits;
                }
            }
            it = s->memos.emplace(cls, std::make_pair(t, bits)).first;
        }
        if (it->second.first) {
            a.memo = it->second.first;
            a.memo_bits = (u32)it->second.second;
            J.var.memo = landmarks ? 2 : 1;
        }
    }
}

bool remaining(const SJob& J) { return J.next_main < J.plan.main_count || (!J.extras_issued && !J.plan.extra.empty()); }

// Finishes a job whose accumulators are complete: reads its slot back and publishes the result.
void finish_job(war_server* s, u64 id) {
    SJob& J = s->jobs[id];
    cudaError_t e = cudaMemcpyAsync(s->h_slot, s->d_slots + J.slot, sizeof(DevAcc), cudaMemcpyDeviceToHost, s->s_copy);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->s_copy);
    std::lock_guard<std::mutex> lk(s->mu);
    if (e != cudaSuccess) {
        J.state = 3; J.status = WAR_ECUDA;
    } else if (s->h_slot->status) {
        J.state = 3; J.status = WAR_ECAP;
    } else {
        merge_acc(*s->h_slot, J.result, J.job.hbins, J.job.dbins);
        J.state = 2;
    }
    J.t_finish = s->now_ms();
    s->free_slots.push_back(J.slot);
    s->resident--;
    s->jobs_done++;
    s->cv_done.notify_all();
}

// Admits queued jobs into free slots (caller holds the lock).  Empty jobs finish at once.
void admit(war_server* s, Tick& T) {
    while (!s->pending.empty() && !s->free_slots.empty()) {
        u64 id = s->pending.front();
        s->pending.pop_front();
        SJob& J = s->jobs[id];
        J.t_admit = s->now_ms();
        const war_job& job = J.job;
        const bool canon = job.mode == WAR_CANON;
        if (job.lo == job.hi || (!canon && job.n == 1)) {   // nothing to play on the device
            if (!canon && job.n == 1) {
                J.result->done = 1; J.result->endhist[0] = 1;
                if ((job.flags & WAR_F_SAMPLE) && war_sample_pick(job.seed, job.sample_ppm, 0x10ull, 0x1ull))
                    J.result->s_count = 1;
            }
            J.state = 2; J.t_finish = J.t_admit; s->jobs_done++;
            s->cv_done.notify_all();
            continue;
        }
        const int M = canon ? job.n - 1 : job.n;
        make_plan(&job, std::max(1, std::min(canon ? 4 : 6, M)), J.plan);
        J.per_unit = fact(J.plan.m) * J.plan.games_per_order;
        set_args(s, J);
        J.slot = s->free_slots.back();
        s->free_slots.pop_back();
        J.state = 1;
        s->resident++;
        s->peak_resident = std::max<u64>(s->peak_resident, s->resident);
        T.admitted.push_back(id);
    }
}

// Cuts the running jobs' remaining work into this tick's tasks (caller holds the lock).
void build_tick(war_server* s, Tick& T) {
    T.ntasks = 0; T.nunits = 0; T.groups.clear(); T.finishing.clear();
    std::vector<u64> run;
    for (auto& kv : s->jobs)
        if (kv.second.state == 1 && remaining(kv.second)) run.push_back(kv.first);
    if (run.empty()) return;
    const u64 budget = s->cfg.tick_ranks;
    const u64 unit_cap = (u64)s->max_units * 8;
    u64 used = 0, units_used = 0;
    std::vector<std::pair<Variant, ServeTask>> tasks;
    std::vector<std::vector<Unit>> task_units;
    bool progress = true;
    while (progress && used < budget && (int)tasks.size() < s->max_tasks) {
        progress = false;
        for (u64 id : run) {
            if (used >= budget || (int)tasks.size() >= s->max_tasks) break;
            SJob& J = s->jobs[id];
            if (!remaining(J)) continue;
            ServeTask t;
            memset(&t, 0, sizeof t);
            t.args = J.base;
            t.slot = (u32)J.slot;
            std::vector<Unit> ex;
            if (J.next_main < J.plan.main_count) {
                u64 k = std::max<u64>(1, TASK_RANKS / J.per_unit);
                k = std::min(k, J.plan.main_count - J.next_main);
                t.args.main_base = J.plan.main_base + J.next_main;
                t.args.main_count = k;
                t.args.n_units = k;
                J.next_main += k;
                used += k * J.per_unit;
            } else {
                if (units_used + J.plan.extra.size() > unit_cap) continue;   // next tick
                units_used += J.plan.extra.size();
                ex = J.plan.extra;
                t.args.main_base = 0;
                t.args.main_count = 0;
                t.args.n_units = ex.size();
                J.extras_issued = true;
                used += 1;
            }
            if (!remaining(J)) T.finishing.push_back(id);
            tasks.push_back({J.var, t});
            task_units.push_back(std::move(ex));
            progress = true;
        }
    }
    // group by kernel variant, lay out tasks and extra units
    std::vector<int> order(tasks.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tasks[x].first < tasks[y].first; });
    for (int idx : order) {
        ServeTask t = tasks[idx].second;
        const std::vector<Unit>& ex = task_units[idx];
        if (!ex.empty()) {
            memcpy(T.h_units + T.nunits, ex.data(), sizeof(Unit) * ex.size());
            t.args.units = T.d_units + T.nunits;
            T.nunits += (int)ex.size();
        }
        if (T.groups.empty() || !(T.groups.back().first == tasks[idx].first))
            T.groups.push_back({tasks[idx].first, {T.ntasks, 0}});
        T.groups.back().second.second++;
        T.h_tasks[T.ntasks++] = t;
    }
}

cudaError_t launch_tick(war_server* s, Tick& T) {
    cudaError_t e;
    for (u64 id : T.admitted) {
        if ((e = cudaMemsetAsync(s->d_slots + s->jobs[id].slot, 0, sizeof(DevAcc), s->s_comp)) != cudaSuccess) return e;
    }
    T.admitted.clear();
    if (T.ntasks == 0) return cudaSuccess;
    if ((e = cudaMemcpyAsync(T.d_tasks, T.h_tasks, sizeof(ServeTask) * T.ntasks, cudaMemcpyHostToDevice, s->s_comp)))
        return e;
    if (T.nunits &&
        (e = cudaMemcpyAsync(T.d_units, T.h_units, sizeof(Unit) * T.nunits, cudaMemcpyHostToDevice, s->s_comp)))
        return e;
    for (auto& g : T.groups) {
        int hb = 0;
        for (int i = g.second.first; i < g.second.first + g.second.second; i++) hb = std::max(hb, T.h_tasks[i].args.hbins);
        // every task of the group zeroes and flushes hbins of its own; the launch provides the largest
        size_t shmem = sizeof(u32) * (size_t)(hb + WAR_EBINS);
        g.first.fn()<<<g.second.second, g.first.threads(), shmem, s->s_comp>>>(T.d_tasks + g.second.first, s->d_slots);
        note_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaEventRecord(T.ev, s->s_comp);
}

void worker_main(war_server* s) {
    cudaSetDevice(s->device);
    int cur = 0;
    for (;;) {
        Tick& T = s->ticks[cur];
        bool built = false;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            bool busy = s->ticks[cur ^ 1].in_flight;
            if (!busy) {
                s->cv_work.wait_for(lk, std::chrono::milliseconds(2), [&] {
                    if (s->stop || !s->pending.empty()) return true;
                    for (auto& kv : s->jobs) if (kv.second.state == 1 && remaining(kv.second)) return true;
                    return false;
                });
            }
            if (s->stop && s->pending.empty() && !busy) {
                bool any = false;
                for (auto& kv : s->jobs) if (kv.second.state == 1) any = true;
                if (!any) break;
            }
            if (!s->fatal) {
                admit(s, T);
                build_tick(s, T);
                built = T.ntasks > 0 || !T.admitted.empty();
            }
        }
        if (built) {
            cudaError_t e = launch_tick(s, T);
            if (e != cudaSuccess) {
                std::lock_guard<std::mutex> lk(s->mu);
                s->fatal = WAR_ECUDA;
                for (auto& kv : s->jobs)
                    if (kv.second.state <= 1) { kv.second.state = 3; kv.second.status = WAR_ECUDA; }
                s->cv_done.notify_all();
            } else if (T.ntasks > 0) {
                T.in_flight = true;
                s->nticks++;
            }
        }
        Tick& P = s->ticks[cur ^ 1];
        if (P.in_flight) {
            cudaError_t e = cudaEventSynchronize(P.ev);
            P.in_flight = false;
            if (e != cudaSuccess) {
                std::lock_guard<std::mutex> lk(s->mu);
                s->fatal = WAR_ECUDA;
                for (auto& kv : s->jobs)
                    if (kv.second.state <= 1) { kv.second.state = 3; kv.second.status = WAR_ECUDA; }
                s->cv_done.notify_all();
            } else {
                for (u64 id : P.finishing) finish_job(s, id);
            }
            P.finishing.clear();
        }
        cur ^= 1;
    }
}

}  // namespace
}  // namespace war

using namespace war;

extern "C" {

int war_server_create(const war_server_cfg* cfg, war_server** out) {
    if (!out) return fail(WAR_EINVAL, "out is NULL");
    *out = nullptr;
    war_server_cfg c;
    memset(&c, 0, sizeof c);
    if (cfg) c = *cfg;
    if (c.max_jobs < 0 || c.queue_cap < 0) return fail(WAR_EINVAL, "negative max_jobs / queue_cap");
    if (!c.max_jobs) c.max_jobs = 256;
    if (!c.queue_cap) c.queue_cap = 1 << 16;
    if (!c.tick_ranks) c.tick_ranks = 1ull << 27;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(WAR_ENODEV, "no CUDA device (%s)", cudaGetErrorString(e));
    war_server* s = new war_server();
    s->cfg = c;
    cudaGetDevice(&s->device);
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    u64 budget = c.mem_budget ? c.mem_budget : fr / 2;
    s->nslots = (int)std::min<u64>((u64)c.max_jobs, budget / sizeof(DevAcc));
    if (s->nslots < 1) {
        delete s;
        return fail(WAR_ENOMEM, "memory budget %llu holds no job accumulator (%zu bytes each)", (unsigned long long)budget,
                    sizeof(DevAcc));
    }
    // the memo arena: what the budget leaves after the slots, at most 16 GiB, reserved now so that the
    // worker thread never allocates; a smaller one when the device cannot give that much
    if (c.memo_bits >= 0) {
        const u64 rest = budget - (u64)s->nslots * sizeof(DevAcc);
        u64 words = std::min<u64>(rest / sizeof(u64), 1ull << 31);
        while (words >= (1ull << 12)) {
            if (cudaMalloc(&s->memo_arena, words * sizeof(u64)) == cudaSuccess) break;
            s->memo_arena = nullptr;
            cudaGetLastError();
            words /= 2;
        }
        s->arena_words = s->memo_arena ? words : 0;
    }
    s->max_tasks = 16384;
    s->max_units = s->max_tasks + 4 * UNITS_PER_EXTRA_CAP;
    bool ok = cudaMalloc(&s->d_slots, sizeof(DevAcc) * (size_t)s->nslots) == cudaSuccess &&
              cudaMallocHost(&s->h_slot, sizeof(DevAcc)) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->s_comp, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->s_copy, cudaStreamNonBlocking) == cudaSuccess;
    for (int i = 0; ok && i < 2; i++) {
        Tick& T = s->ticks[i];
        ok = cudaMallocHost(&T.h_tasks, sizeof(ServeTask) * s->max_tasks) == cudaSuccess &&
             cudaMallocHost(&T.h_units, sizeof(Unit) * (size_t)s->max_units * 8) == cudaSuccess &&
             cudaMalloc(&T.d_tasks, sizeof(ServeTask) * s->max_tasks) == cudaSuccess &&
             cudaMalloc(&T.d_units, sizeof(Unit) * (size_t)s->max_units * 8) == cudaSuccess &&
             cudaEventCreateWithFlags(&T.ev, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        war_server_destroy(s);
        return fail(WAR_ENOMEM, "server buffers could not be allocated");
    }
    for (int i = s->nslots - 1; i >= 0; i--) s->free_slots.push_back(i);
    s->t0 = std::chrono::steady_clock::now();
    s->worker = std::thread(worker_main, s);
    *out = s;
    return WAR_OK;
}

int war_server_submit(war_server* s, const war_job* job, uint64_t* id) {
    if (!s || !id) return fail(WAR_EINVAL, "NULL server or id");
    int st = check_job(job);
    if (st) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fatal) return fail(s->fatal, "server stopped after a CUDA error");
    if ((int)s->pending.size() >= s->cfg.queue_cap) return fail(WAR_EBUSY, "queue full (%d jobs)", s->cfg.queue_cap);
    u64 k = s->next_id++;
    SJob& J = s->jobs[k];
    J.job = *job;
    J.result = new war_result();
    memset(J.result, 0, sizeof(war_result));
    J.result->hbins = job->hbins;
    J.result->dbins = job->dbins;
    J.result->blk = (job->flags & WAR_F_SHAPE) && job->mode == WAR_CANON ? (job->blk ? job->blk : (job->n & -job->n)) : 0;
    J.t_submit = s->now_ms();
    s->pending.push_back(k);
    *id = k;
    s->cv_work.notify_one();
    return WAR_OK;
}

int war_server_poll(war_server* s, uint64_t id, war_result* res, war_job_status* st) {
    if (!s) return fail(WAR_EINVAL, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(WAR_ENOTFOUND, "no job %llu", (unsigned long long)id);
    SJob& J = it->second;
    if (st) {
        st->state = J.state; st->status = J.status;
        st->submit_ms = J.t_submit; st->admit_ms = J.t_admit; st->finish_ms = J.t_finish;
    }
    if (J.state < 2) return WAR_PENDING;
    int status = J.state == 2 ? WAR_OK : (J.status ? J.status : WAR_ECUDA);
    if (res && J.state == 2) *res = *J.result;
    delete J.result;
    s->jobs.erase(it);
    return status == WAR_OK ? WAR_OK : fail(status, "job %llu failed", (unsigned long long)id);
}

int war_server_drain(war_server* s, double timeout_ms) {
    if (!s) return fail(WAR_EINVAL, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto until = std::chrono::steady_clock::now() + std::chrono::microseconds((long long)(timeout_ms * 1000));
    bool ok = s->cv_done.wait_until(lk, until, [&] {
        if (!s->pending.empty()) return false;
        for (auto& kv : s->jobs) if (kv.second.state < 2) return false;
        return true;
    });
    return ok ? WAR_OK : fail(WAR_ETIMEOUT, "jobs still running after %.0f ms", timeout_ms);
}

int war_server_stats(war_server* s, uint64_t* ticks, uint64_t* jobs_done, uint64_t* peak_resident) {
    if (!s) return fail(WAR_EINVAL, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (ticks) *ticks = s->nticks;
    if (jobs_done) *jobs_done = s->jobs_done;
    if (peak_resident) *peak_resident = s->peak_resident;
    return WAR_OK;
}

int war_server_memo_info(war_server* s, uint64_t* arena_bytes, uint64_t* used_bytes, int32_t* classes) {
    if (!s) return fail(WAR_EINVAL, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    int k = 0;
    for (auto& kv : s->memos)
        if (kv.second.first) k++;
    if (arena_bytes) *arena_bytes = s->arena_words * sizeof(u64);
    if (used_bytes) *used_bytes = s->arena_used * sizeof(u64);
    if (classes) *classes = k;
    return WAR_OK;
}

int war_server_destroy(war_server* s) {
    if (!s) return WAR_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->pending.clear();
        for (auto& kv : s->jobs)
            if (kv.second.state == 0) { kv.second.state = 3; kv.second.status = WAR_EINVAL; }
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    for (auto& kv : s->jobs) delete kv.second.result;
    for (int i = 0; i < 2; i++) {
        Tick& T = s->ticks[i];
        if (T.h_tasks) cudaFreeHost(T.h_tasks);
        if (T.h_units) cudaFreeHost(T.h_units);
        if (T.d_tasks) cudaFree(T.d_tasks);
        if (T.d_units) cudaFree(T.d_units);
        if (T.ev) cudaEventDestroy(T.ev);
    }
    if (s->memo_arena) cudaFree(s->memo_arena);
    if (s->d_slots) cudaFree(s->d_slots);
    if (s->h_slot) cudaFreeHost(s->h_slot);
    if (s->s_comp) cudaStreamDestroy(s->s_comp);
    if (s->s_copy) cudaStreamDestroy(s->s_copy);
    delete s;
    return WAR_OK;
}

}  // extern "C"
