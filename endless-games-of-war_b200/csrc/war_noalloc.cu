// war_noalloc.cu — war_enumerate_noalloc: the refill kernel of war_enumerate with its scratch memory in
// a fixed array that the library declares statically, for callers that cannot allocate device memory.
//
// Who needs it: a host program whose own memory pool has reserved the GPU's memory (a cudaMalloc would
// fail or fragment that pool), and code on a latency-bound path that cannot take the implicit device
// synchronisation of cudaMalloc / cudaFree.  Such callers cannot use war_enumerate, whose first call
// allocates the accumulators, the unit list, a stream and events.
//
// What this entry point does instead: its scratch (the accumulators and work counter of one job plus up
// to WAR_NOALLOC_UNITS extra work units) is the file-scope array below, which every GPU that loads the
// library holds until the process exits.  On each device, the first call looks up the array's device
// address with cudaGetSymbolAddress (in host code the array's name is only a host-side stand-in, not a
// device address) and keeps it; that first call should therefore come before any stream capture.  It
// calls no cudaMalloc, cudaFree or other allocating routine, creates no stream or event, and plans the
// job into a fixed host array.  All calls share the one array and leave the last job's contents in it:
// each call clears the accumulators before its launch, and calls whose work overlaps on the GPU (from
// several host threads on different streams) race on it.  Host-side calls are serialised by a lock.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include "war_host.h"

namespace war {

// Fixed scratch of the no-allocation entry point: one job's accumulators followed by its extra units.
// A range split with block_m <= 8 needs at most a few dozen extra units; 1024 leaves ample room.
constexpr int WAR_NOALLOC_UNITS = 1024;
constexpr size_t WAR_NOALLOC_BYTES = sizeof(DevAcc) + sizeof(Unit) * WAR_NOALLOC_UNITS;

static __device__ __align__(256) unsigned char g_noalloc_scratch[WAR_NOALLOC_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;

struct NoallocHost {
    std::mutex mu;
    unsigned char* dev_scratch[MAX_DEVICES] = {};   // device address of g_noalloc_scratch, per device
    DevAcc acc;                                    // readback staging in static host storage
    Unit units[WAR_NOALLOC_UNITS];                 // the plan's extra units, staged for the copy
};

NoallocHost& host() {
    static NoallocHost h;
    return h;
}

// Aligned blocks of j! orders (j <= m) covering orders [x, y), largest first, into a fixed array.
bool put_blocks(u64 x, u64 y, int m, u32 k0, u32 k1, Unit* out, int cap, int& k) {
    while (x < y) {
        int j = m;
        while (j > 0 && (x % fact(j) != 0 || x + fact(j) > y)) j--;
        if (k >= cap) return false;
        out[k].r = x; out[k].j = (u32)j; out[k].k0 = k0; out[k].k1 = k1; out[k].pad = 0;
        k++;
        x += fact(j);
    }
    return true;
}

// The same plan as war_enumerate's: main units of m! orders plus extra units for the ragged ends and,
// for canonical positions, for the partial splits of the first and last order.  Returns the number of
// extra units, or -1 if they do not fit in cap.
int plan_fixed(const war_job* job, int m, u64& main_base, u64& main_count, u64& games_per_order, Unit* out, int cap) {
    const int n = job->n;
    int k = 0;
    main_base = 0;
    main_count = 0;
    u64 A, B;
    if (job->mode == WAR_DEALS) {
        A = job->lo; B = job->hi;
        games_per_order = 1;
    } else {
        const u64 s = (u64)(n - 1);
        games_per_order = s;
        const u64 lo = job->lo, hi = job->hi;
        if (lo >= hi) return 0;
        const u64 pa = lo / s, pb = hi / s;
        if (pa == pb) {
            if (cap < 1) return -1;
            out[0].r = pa; out[0].j = 0; out[0].k0 = (u32)(lo % s); out[0].k1 = (u32)(hi % s); out[0].pad = 0;
            return 1;
        }
        A = pa; B = pb;
        if (lo % s) {
            if (k >= cap) return -1;
            out[k].r = pa; out[k].j = 0; out[k].k0 = (u32)(lo % s); out[k].k1 = (u32)s; out[k].pad = 0;
            k++;
            A = pa + 1;
        }
        if (hi % s) {
            if (k >= cap) return -1;
            out[k].r = pb; out[k].j = 0; out[k].k0 = 0; out[k].k1 = (u32)(hi % s); out[k].pad = 0;
            k++;
        }
    }
    if (A >= B) return k;
    const u32 k1 = job->mode == WAR_CANON ? (u32)(n - 1) : 0u;
    const u64 fm = fact(m);
    const u64 A2 = (A + fm - 1) / fm * fm, B2 = B / fm * fm;
    if (A2 < B2) {
        if (!put_blocks(A, A2, m, 0, k1, out, cap, k)) return -1;
        main_base = A2 / fm;
        main_count = (B2 - A2) / fm;
        if (!put_blocks(B2, B, m, 0, k1, out, cap, k)) return -1;
    } else if (!put_blocks(A, B, m, 0, k1, out, cap, k)) {
        return -1;
    }
    return k;
}

}  // namespace
}  // namespace war

using namespace war;

extern "C" int war_enumerate_noalloc(const war_job* job, const war_tune* tune, war_result* out) {
    int st = check_job(job);
    if (st) return st;
    if (!out) return fail(WAR_EINVAL, "out is NULL");
    memset(out, 0, sizeof(*out));
    out->hbins = job->hbins;
    out->dbins = job->dbins;
    out->blk = (job->flags & WAR_F_SHAPE) ? (job->blk ? job->blk : (job->n & -job->n)) : 0;
    if (job->lo == job->hi) return WAR_OK;
    if (job->mode == WAR_DEALS && job->n == 1) {   // the one 1-card deal is over before it starts
        out->done = 1;
        out->endhist[0] = 1;
        if ((job->flags & WAR_F_SAMPLE) && war_sample_pick(job->seed, job->sample_ppm, 0x10ull, 0x1ull)) out->s_count = 1;
        return WAR_OK;
    }
    const bool canon = job->mode == WAR_CANON;
    const int M = canon ? job->n - 1 : job->n;
    int threads = (tune && tune->threads) ? tune->threads : 256;
    int games = (tune && tune->games) ? tune->games : 1;
    int block_m = (tune && tune->block_m) ? tune->block_m : (canon ? 5 : 6);
    int window = (tune && tune->window) ? tune->window : (canon ? 128 : 32);
    int defer = (tune && tune->defer) ? tune->defer : 1;
    int variant = tune ? tune->variant : 0;
    if (threads < 64 || threads > 1024 || (threads & 31)) return fail(WAR_EINVAL, "tune.threads=%d", threads);
    if (games != 1 && games != 2) return fail(WAR_EINVAL, "tune.games=%d (1 or 2)", games);
    if (block_m < 1 || block_m > 8) return fail(WAR_EINVAL, "tune.block_m=%d (1..8)", block_m);
    if (window < 1 || window > (1 << 16) || (window & (window - 1))) return fail(WAR_EINVAL, "tune.window=%d", window);
    if (defer < 1 || defer > 32) return fail(WAR_EINVAL, "tune.defer=%d (1..32)", defer);
    if (variant < 0 || variant > 31) return fail(WAR_EINVAL, "tune.variant=%d (0..31)", variant);
    variant &= 3;   // no cycle memo: its table would be allocated memory
    if (block_m > M) block_m = M > 0 ? M : 1;

    NoallocHost& h = host();
    std::lock_guard<std::mutex> lk(h.mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= MAX_DEVICES) return fail(WAR_EINVAL, "device %d above the %d this entry point tracks", dev, MAX_DEVICES);
    if (!h.dev_scratch[dev]) {   // set-up, once per device, with that device current
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress of the static scratch");
        h.dev_scratch[dev] = (unsigned char*)p;
    }
    DevAcc* d_acc = (DevAcc*)h.dev_scratch[dev];
    Unit* d_units = (Unit*)(h.dev_scratch[dev] + sizeof(DevAcc));

    u64 main_base = 0, main_count = 0, per_order = 1;
    const int n_extra = plan_fixed(job, block_m, main_base, main_count, per_order, h.units, WAR_NOALLOC_UNITS);
    if (n_extra < 0)
        return fail(WAR_EINVAL, "the job needs more than the %d extra work units war_enumerate_noalloc holds "
                    "(use war_enumerate, or split the range)", WAR_NOALLOC_UNITS);

    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    const int shape = (job->flags & WAR_F_SHAPE) && canon ? 1 : 0;
    int maxb = batched_max_blocks_per_sm(canon, job->rule, shape, (job->flags & WAR_F_DISTINCT) != 0,
                                         (job->flags & WAR_F_SAMPLE) != 0, threads, games, job->hbins, variant);
    if (maxb < 1) return fail(WAR_EINVAL, "launch shape threads=%d games=%d does not fit an SM", threads, games);
    const int bps = (tune && tune->blocks_per_sm) ? std::min(tune->blocks_per_sm, maxb) : maxb;

    BatchArgs a;
    memset(&a, 0, sizeof a);
    fill_fact(a.fact);
    a.n = job->n; a.m = block_m; a.hbins = job->hbins; a.dbins = job->dbins;
    a.blk = out->blk; a.W = window; a.defer = defer;
    a.tk.k16 = 16u; a.tk.km16 = (u32)-16; a.tk.k2p28 = 1u << 28; a.tk.k4 = 4u; a.tk.one = 1u;
    a.tk.c0 = 2 * job->n - 4; a.tk.end2 = (u32)(4 * job->n * job->n);
    a.half = (job->flags & WAR_F_HALF) ? 1 : 0;
    a.sample = (job->flags & WAR_F_SAMPLE) ? 1 : 0;
    a.distinct = (job->flags & WAR_F_DISTINCT) && canon ? 1 : 0;
    a.seed = job->seed;
    a.thr = ((u64)job->sample_ppm << 32) / 1000000u;
    a.units = d_units;
    BatchShape bs;
    bs.threads = threads; bs.games = games; bs.blocks = bps * sms; bs.variant = variant;

    cudaStream_t s = ctx().user_stream;   // the caller's stream (war_set_stream) or the default stream
    if (n_extra > 0 &&
        (e = cudaMemcpyAsync(d_units, h.units, sizeof(Unit) * (size_t)n_extra, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_fail(e, "copy units to the static scratch");
    // each launch plays fewer than 2^32 games (the kernel's 32-bit counters)
    const u64 per_unit = fact(block_m) * per_order;
    const u64 max_units = std::max<u64>(1, ((1ull << 32) - (1ull << 24)) / per_unit);
    const auto t0 = std::chrono::steady_clock::now();
    u64 done_main = 0;
    bool extras_done = n_extra == 0;
    while (done_main < main_count || !extras_done) {
        const u64 take = std::min<u64>(max_units, main_count - done_main);
        const bool last = done_main + take >= main_count;
        a.main_base = main_base + done_main;
        a.main_count = take;
        a.n_units = take + (last ? (u64)n_extra : 0);
        if ((e = cudaMemsetAsync(d_acc, 0, sizeof(DevAcc), s)) != cudaSuccess) return cuda_fail(e, "clear the static scratch");
        if ((e = launch_batched(a, canon, job->rule, shape, bs, d_acc, s)) != cudaSuccess) return cuda_fail(e, "kernel launch");
        if ((e = cudaMemcpyAsync(&h.acc, d_acc, sizeof(DevAcc), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
            return cuda_fail(e, "read back the static scratch");
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "kernel execution");
        if (h.acc.status) return fail(WAR_ECAP, "%llu game(s) passed the turn cap", (unsigned long long)h.acc.status);
        merge_acc(h.acc, out, job->hbins, job->dbins);
        out->units += a.n_units;
        done_main += take;
        if (last) extras_done = true;
    }
    out->kernel_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return WAR_OK;
}
