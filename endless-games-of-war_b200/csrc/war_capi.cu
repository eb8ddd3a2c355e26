// war_capi.cu — the extern "C" entry points of libwar.so (include/war.h): argument checks, the plan
// of work units, launches on the library's stream, and readback of the accumulators.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include "war_kernels.cuh"
#include "war_host.h"

namespace war {

static std::atomic<u64> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

static thread_local std::string t_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(WAR_ECUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

u64 fact(int i) {
    u64 f = 1;
    for (int k = 2; k <= i; k++) f *= (u64)k;
    return f;
}

u64 space_size(int n, int mode) {
    if (mode == WAR_CANON) return n < 2 ? 0 : fact(n - 1) * (u64)(n - 1);
    return fact(n);
}

int check_job(const war_job* j) {
    if (!j) return fail(WAR_EINVAL, "job is NULL");
    if (j->n < 1 || j->n > WAR_MAX_N) return fail(WAR_EINVAL, "n=%d outside 1..%d", j->n, WAR_MAX_N);
    if (j->mode != WAR_DEALS && j->mode != WAR_CANON) return fail(WAR_EINVAL, "mode=%d", j->mode);
    if (j->rule != 0 && j->rule != 1) return fail(WAR_EINVAL, "rule=%d", j->rule);
    if (j->hbins < 0 || j->hbins > WAR_HBINS_MAX) return fail(WAR_EINVAL, "hbins=%d outside 0..%d", j->hbins, WAR_HBINS_MAX);
    if (j->dbins < 0 || j->dbins > WAR_DBINS_MAX) return fail(WAR_EINVAL, "dbins=%d outside 0..%d", j->dbins, WAR_DBINS_MAX);
    if (j->flags & ~(WAR_F_HALF | WAR_F_DISTINCT | WAR_F_SHAPE | WAR_F_SAMPLE | WAR_F_MEMO_KEEP))
        return fail(WAR_EINVAL, "flags=0x%x", j->flags);
    if ((j->flags & WAR_F_HALF) && (j->mode != WAR_DEALS || (j->n & 1)))
        return fail(WAR_EINVAL, "WAR_F_HALF needs deals with even n");
    if (j->sample_ppm > 1000000u) return fail(WAR_EINVAL, "sample_ppm=%u above 10^6", j->sample_ppm);
    if (j->blk < 0 || j->blk > 512) return fail(WAR_EINVAL, "blk=%d", j->blk);
    u64 total = space_size(j->n, j->mode);
    if (j->lo > j->hi || j->hi > total)
        return fail(WAR_EINVAL, "range [%llu, %llu) outside the space of %llu", (unsigned long long)j->lo,
                    (unsigned long long)j->hi, (unsigned long long)total);
    return WAR_OK;
}

// ---- the library context ------------------------------------------------------------------------

Ctx& ctx() {
    static Ctx c;
    return c;
}

int ensure_ready() {
    Ctx& c = ctx();
    if (c.ready) return WAR_OK;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(WAR_ENODEV, "no CUDA device (%s)", cudaGetErrorString(e));
    if ((e = cudaGetDevice(&c.device)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    cudaDeviceProp p;
    if ((e = cudaGetDeviceProperties(&p, c.device)) != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
    c.sm_count = p.multiProcessorCount;
    if ((e = cudaStreamCreateWithFlags(&c.own_stream, cudaStreamNonBlocking)) != cudaSuccess) return cuda_fail(e, "stream");
    if ((e = cudaMalloc(&c.d_acc, sizeof(DevAcc))) != cudaSuccess) return cuda_fail(e, "cudaMalloc acc");
    if ((e = cudaMalloc(&c.d_units, sizeof(Unit) * Ctx::UNIT_CAP)) != cudaSuccess) return cuda_fail(e, "cudaMalloc units");
    if ((e = cudaMallocHost(&c.h_acc, sizeof(DevAcc))) != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
    if ((e = cudaEventCreate(&c.ev0)) != cudaSuccess) return cuda_fail(e, "event");
    if ((e = cudaEventCreate(&c.ev1)) != cudaSuccess) return cuda_fail(e, "event");
    c.ready = true;
    return WAR_OK;
}

cudaStream_t cur_stream() {
    Ctx& c = ctx();
    return c.user_stream ? c.user_stream : c.own_stream;
}

// Adds the device accumulators of one launch (already copied to h) into a result.
void merge_acc(const DevAcc& h, war_result* r, int hbins, int dbins) {
    r->cyc += h.cyc; r->done += h.done; r->turns += h.turns;
    if (h.maxfin > r->maxfin) r->maxfin = h.maxfin;
    r->shape_nonstd += h.shape_nonstd; r->shape_unchecked += h.shape_unchecked;
    r->oncycle += h.oncycle; r->distinct_min += h.distinct_min;
    r->s_count += h.s_count; r->s_cyc += h.s_cyc; r->s_lamsum += h.s_lamsum; r->s_lensum += h.s_lensum;
    if (h.s_maxfin > r->s_maxfin) r->s_maxfin = h.s_maxfin;
    r->units += h.units;
    r->memo_lookups += h.memo_lookups; r->memo_hits += h.memo_hits; r->memo_stores += h.memo_stores;
    r->undetermined += h.undetermined;
    for (int i = 0; i < hbins; i++) r->hist[i] += h.hist[i];
    for (int i = 0; i < dbins; i++) r->dhist[i] += h.dhist[i];
    for (int i = 0; i < WAR_EBINS; i++) r->endhist[i] += h.endhist[i];
}

void fill_fact(u64* f) {
    for (int i = 0; i <= 16; i++) f[i] = fact(i);
}

// ---- the plan: a rank range as work units ---------------------------------------------------------

// Splits orders [x, y) into aligned blocks of j! orders (j <= m), largest first.
void decompose(u64 x, u64 y, int m, u32 k0, u32 k1, std::vector<Unit>& out) {
    while (x < y) {
        int j = m;
        while (j > 0 && (x % fact(j) != 0 || x + fact(j) > y)) j--;
        Unit u; u.r = x; u.j = (u32)j; u.k0 = k0; u.k1 = k1; u.pad = 0;
        out.push_back(u);
        x += fact(j);
    }
}

void make_plan(const war_job* job, int m, Plan& p) {
    const int n = job->n;
    p.m = m;
    p.extra.clear();
    p.main_base = 0; p.main_count = 0;
    u64 A, B;   // full orders
    if (job->mode == WAR_DEALS) {
        A = job->lo; B = job->hi;
        p.games_per_order = 1;
    } else {
        const u64 s = (u64)(n - 1);
        p.games_per_order = s;
        u64 lo = job->lo, hi = job->hi;
        if (lo >= hi) return;
        u64 pa = lo / s, pb = hi / s;
        if (pa == pb) {   // inside one order
            Unit u; u.r = pa; u.j = 0; u.k0 = (u32)(lo % s); u.k1 = (u32)(hi % s); u.pad = 0;
            p.extra.push_back(u);
            return;
        }
        A = pa; B = pb;
        if (lo % s) {
            Unit u; u.r = pa; u.j = 0; u.k0 = (u32)(lo % s); u.k1 = (u32)s; u.pad = 0;
            p.extra.push_back(u);
            A = pa + 1;
        }
        if (hi % s) {
            Unit u; u.r = pb; u.j = 0; u.k0 = 0; u.k1 = (u32)(hi % s); u.pad = 0;
            p.extra.push_back(u);
        }
    }
    if (A >= B) return;
    const u32 k1 = job->mode == WAR_CANON ? (u32)(n - 1) : 0u;
    const u64 fm = fact(m);
    u64 A2 = (A + fm - 1) / fm * fm, B2 = B / fm * fm;
    if (A2 < B2) {
        decompose(A, A2, m, 0, k1, p.extra);
        p.main_base = A2 / fm;
        p.main_count = (B2 - A2) / fm;
        decompose(B2, B, m, 0, k1, p.extra);
    } else {
        decompose(A, B, m, 0, k1, p.extra);
    }
}

int resolve_tune(const war_job* job, const war_tune* in, Tune& t) {
    const bool canon = job->mode == WAR_CANON;
    t.threads = (in && in->threads) ? in->threads : 256;
    t.games = (in && in->games) ? in->games : 1;
    t.block_m = (in && in->block_m) ? in->block_m : (canon ? 5 : 6);
    t.window = (in && in->window) ? in->window : (canon ? 128 : 32);
    t.defer = (in && in->defer) ? in->defer : 1;
    t.variant = in ? in->variant : 0;
    t.memo_bits = (in && in->memo_bits) ? in->memo_bits : 24;
    t.chunk = (in && in->chunk) ? in->chunk : 1;
    if (t.threads < 64 || t.threads > 1024 || (t.threads & 31)) return fail(WAR_EINVAL, "tune.threads=%d", t.threads);
    if (t.games != 1 && t.games != 2 && t.games != 4) return fail(WAR_EINVAL, "tune.games=%d (1, 2 or 4)", t.games);
    if (t.chunk < 1 || t.chunk > 4096) return fail(WAR_EINVAL, "tune.chunk=%d (1..4096)", t.chunk);
    if (t.block_m < 1 || t.block_m > 8) return fail(WAR_EINVAL, "tune.block_m=%d (1..8)", t.block_m);
    if (t.window < 1 || t.window > (1 << 16) || (t.window & (t.window - 1))) return fail(WAR_EINVAL, "tune.window=%d", t.window);
    if (t.defer < 1 || t.defer > 32) return fail(WAR_EINVAL, "tune.defer=%d (1..32)", t.defer);
    if (t.variant < 0 || t.variant > 31) return fail(WAR_EINVAL, "tune.variant=%d (0..31)", t.variant);
    if (t.memo_bits < 12 || t.memo_bits > 31) return fail(WAR_EINVAL, "tune.memo_bits=%d (12..31)", t.memo_bits);
    // the cycle memo needs latched records and n >= 4; its landmark form serves n <= 15, the all-states
    // form n <= 14, the path form n <= 16; canonical scans take the path form only
    const int memo_nmax = (t.variant & 28) == 28 ? 16 : ((t.variant & 8) ? 14 : 15);
    if ((t.variant & 4) && (!(t.variant & 2) || job->n < 4 || job->n > memo_nmax)) t.variant &= 3;
    if (canon && !(t.variant & 16)) t.variant &= 3;
    if (!(t.variant & 4)) t.variant &= 7;
    if (!(t.variant & 8)) t.variant &= 15;
    const int M = canon ? job->n - 1 : job->n;
    if (t.block_m > M) t.block_m = M > 0 ? M : 1;
    int st = ensure_ready();
    if (st) return st;
    int maxb = batched_max_blocks_per_sm(canon, job->rule, (job->flags & WAR_F_SHAPE) != 0,
                                         (job->flags & WAR_F_DISTINCT) != 0, (job->flags & WAR_F_SAMPLE) != 0,
                                         t.threads, t.games, job->hbins, t.variant);
    if (maxb < 1) return fail(WAR_EINVAL, "launch shape threads=%d games=%d does not fit an SM", t.threads, t.games);
    t.blocks_per_sm = (in && in->blocks_per_sm) ? std::min(in->blocks_per_sm, maxb) : maxb;
    return WAR_OK;
}

int floyd_sample_run(const war_job* job, war_result* out) {
    Ctx& c = ctx();
    cudaError_t e;
    if (job->sample_ppm >= 1000000u) {   // every position: Floyd over the job's own enumeration, no buffer
        FloydArgs a;
        memset(&a, 0, sizeof a);
        fill_fact(a.fact);
        a.n = job->n; a.canon = job->mode == WAR_CANON; a.rule = job->rule;
        a.half = (job->flags & WAR_F_HALF) ? 1 : 0;
        a.per = 256;
        a.seed = job->seed;
        a.thr = 1ull << 32;
        a.start = job->lo; a.total = job->hi;
        const int blocks = c.sm_count * floyd_enum_blocks_per_sm(a.canon, a.rule);
        int st = run_launch([&](cudaStream_t x) { return launch_floyd_enum(a, blocks, c.d_acc, x); }, &out->kernel_ms);
        if (st) return st;
        merge_acc(*c.h_acc, out, 0, 0);
        return WAR_OK;
    }
    if (!c.d_sample) {
        c.sample_cap = 1u << 22;   // 4M positions, 64 MB
        if ((e = cudaMalloc(&c.d_sample, sizeof(ulonglong2) * c.sample_cap)) != cudaSuccess) {
            c.d_sample = nullptr;
            return cuda_fail(e, "cudaMalloc sample buffer");
        }
    }
    FloydArgs a;
    memset(&a, 0, sizeof a);
    fill_fact(a.fact);
    a.n = job->n; a.canon = job->mode == WAR_CANON; a.rule = job->rule;
    a.half = (job->flags & WAR_F_HALF) ? 1 : 0;
    a.per = 256;
    a.seed = job->seed;
    a.thr = ((u64)job->sample_ppm << 32) / 1000000u;
    // pieces whose expected sample fills at most a quarter of the buffer
    double rate = job->sample_ppm / 1e6;
    u64 piece = (u64)std::max(1.0, (double)(c.sample_cap / 4) / std::max(rate, 1e-12));
    piece = std::min<u64>(piece, 1ull << 40);
    const int threads = 256;
    for (u64 s = job->lo; s < job->hi; s += piece) {
        u64 e_ = std::min<u64>(job->hi, s + piece);
        a.start = s; a.total = e_;
        u64 nth = (e_ - s + a.per - 1) / a.per;
        int st = run_launch([&](cudaStream_t x) {
            cudaError_t r = cudaSuccess;
            for (u64 t0 = 0; t0 < nth && r == cudaSuccess; t0 += (1ull << 22)) {
                FloydArgs b = a;
                b.start = s + t0 * (u64)a.per;
                r = launch_sample_scan(b, threads, std::min<u64>(1ull << 22, nth - t0), c.d_sample, c.sample_cap, c.d_acc, x);
            }
            if (r == cudaSuccess) r = launch_floyd_play(c.d_sample, c.sample_cap, job->n, job->rule, c.sm_count * 8, 256, c.d_acc, x);
            return r;
        }, &out->kernel_ms);
        if (st) return st;
        if (c.h_acc->units > c.sample_cap)
            return fail(WAR_ENOMEM, "sample buffer overflow: %llu positions in a piece", (unsigned long long)c.h_acc->units);
        DevAcc h = *c.h_acc;
        h.units = 0;
        merge_acc(h, out, 0, 0);
    }
    return WAR_OK;
}

}  // namespace war

using namespace war;

extern "C" {

int war_last_error(char* buf, size_t len) {
    if (buf && len) {
        size_t k = std::min(len - 1, t_err.size());
        memcpy(buf, t_err.data(), k);
        buf[k] = 0;
    }
    return (int)t_err.size();
}

uint64_t war_launch_count(void) { return g_launches.load(); }

int war_sample_pick(uint64_t seed, uint32_t ppm, uint64_t w1s, uint64_t w2s) {
    u64 thr = ((u64)ppm << 32) / 1000000u;
    return war_pick(seed, thr, w1s, w2s) ? 1 : 0;
}

int war_plan(const war_job* job, int32_t block_m, uint64_t* main_base, uint64_t* main_count, war_unit* extra,
             int32_t cap) {
    int st = check_job(job);
    if (st) return st;
    if (block_m < 1 || block_m > 8) return fail(WAR_EINVAL, "block_m=%d (1..8)", block_m);
    if (!main_base || !main_count || cap < 0 || (cap && !extra)) return fail(WAR_EINVAL, "bad output arguments");
    const int M = job->mode == WAR_CANON ? job->n - 1 : job->n;
    Plan p;
    make_plan(job, std::min(block_m, std::max(M, 1)), p);
    *main_base = p.main_base;
    *main_count = p.main_count;
    for (size_t i = 0; i < p.extra.size() && (int)i < cap; i++) {
        extra[i].r = p.extra[i].r; extra[i].j = p.extra[i].j; extra[i].k0 = p.extra[i].k0;
        extra[i].k1 = p.extra[i].k1; extra[i].pad = 0;
    }
    return (int)p.extra.size();
}

int war_device_info_get(war_device_info* info) {
    if (!info) return fail(WAR_EINVAL, "info is NULL");
    memset(info, 0, sizeof(*info));
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(WAR_ENODEV, "no CUDA device (%s)", cudaGetErrorString(e));
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp p;
    if ((e = cudaGetDeviceProperties(&p, dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
    info->device = dev;
    info->sm_count = p.multiProcessorCount;
    info->cc_major = p.major;
    info->cc_minor = p.minor;
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev);
    info->clock_mhz = clk / 1000;
    info->max_threads_per_sm = p.maxThreadsPerMultiProcessor;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    info->mem_free = fr;
    info->mem_total = tot;
    snprintf(info->name, sizeof info->name, "%s", p.name);
    return WAR_OK;
}

int war_set_stream(void* s) {
    int st = ensure_ready();
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    ctx().user_stream = (cudaStream_t)s;
    return WAR_OK;
}

int war_count_launch(int32_t n, uint64_t start, uint64_t total, int32_t per, int32_t half_rule, int32_t threads,
                     uint64_t nthreads, uint64_t* cyc, uint64_t* done, uint64_t* maxfin, uint64_t* hist,
                     int32_t hbins) {
    if (n < 1 || n > WAR_MAX_N) return fail(WAR_EINVAL, "n=%d", n);
    if (per < 1 || threads < 32 || threads > 1024 || (threads & 31)) return fail(WAR_EINVAL, "per=%d threads=%d", per, threads);
    if (hbins < 0 || hbins > WAR_HBINS_MAX || (hbins && !hist)) return fail(WAR_EINVAL, "hbins=%d", hbins);
    if (!cyc || !done || !maxfin) return fail(WAR_EINVAL, "NULL accumulator");
    if (total > fact(n)) return fail(WAR_EINVAL, "total above n!");
    if ((half_rule & 1) && (n & 1)) return fail(WAR_EINVAL, "half needs even n");
    int st = ensure_ready();
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    PlainArgs a;
    memset(&a, 0, sizeof a);
    fill_fact(a.fact);
    a.start = start; a.total = total; a.n = n; a.per = per;
    a.half = half_rule & 1; a.hbins = hbins;
    double ms = 0;
    st = run_launch([&](cudaStream_t s) { return launch_plain(a, 0, (half_rule >> 1) & 1, threads, nthreads, ctx().d_acc, s); }, &ms);
    if (st) return st;
    const DevAcc& h = *ctx().h_acc;
    *cyc += h.cyc; *done += h.done;
    if (h.maxfin > *maxfin) *maxfin = h.maxfin;
    for (int i = 0; i < hbins; i++) hist[i] += h.hist[i];
    return WAR_OK;
}

int war_canon_launch(int32_t n, uint64_t start, uint64_t total, int32_t per, int32_t blk, int32_t threads,
                     uint64_t nthreads, uint64_t* cyc, uint64_t* done, uint64_t* maxfin, uint64_t* hist,
                     int32_t hbins, uint64_t* shape, int32_t rule, uint64_t* dhist, int32_t dbins) {
    if (n < 2 || n > WAR_MAX_N) return fail(WAR_EINVAL, "n=%d", n);
    if (per < 1 || threads < 32 || threads > 1024 || (threads & 31)) return fail(WAR_EINVAL, "per=%d threads=%d", per, threads);
    if (hbins < 0 || hbins > WAR_HBINS_MAX || (hbins && !hist)) return fail(WAR_EINVAL, "hbins=%d", hbins);
    if (dbins < 0 || dbins > WAR_DBINS_MAX || (dbins && !dhist)) return fail(WAR_EINVAL, "dbins=%d", dbins);
    if (blk < 0 || blk > 512 || (blk && !shape)) return fail(WAR_EINVAL, "blk=%d", blk);
    if (!cyc || !done || !maxfin) return fail(WAR_EINVAL, "NULL accumulator");
    if (rule != 0 && rule != 1) return fail(WAR_EINVAL, "rule=%d", rule);
    if (total > fact(n - 1)) return fail(WAR_EINVAL, "total above (n-1)!");
    int st = ensure_ready();
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    PlainArgs a;
    memset(&a, 0, sizeof a);
    fill_fact(a.fact);
    a.start = start; a.total = total; a.n = n; a.per = per;
    a.hbins = hbins; a.dbins = dbins; a.blk = blk; a.distinct = dbins > 0;
    a.pos_lo = 0; a.pos_hi = ~0ull;
    double ms = 0;
    st = run_launch([&](cudaStream_t s) { return launch_plain(a, 1, rule, threads, nthreads, ctx().d_acc, s); }, &ms);
    if (st) return st;
    const DevAcc& h = *ctx().h_acc;
    *cyc += h.cyc; *done += h.done;
    if (h.maxfin > *maxfin) *maxfin = h.maxfin;
    for (int i = 0; i < hbins; i++) hist[i] += h.hist[i];
    for (int i = 0; i < dbins; i++) dhist[i] += h.dhist[i];
    if (blk) { shape[0] += h.shape_nonstd; shape[1] += h.shape_unchecked; }
    return WAR_OK;
}

static void init_result(const war_job* job, war_result* out) {
    memset(out, 0, sizeof(*out));
    out->hbins = job->hbins;
    out->dbins = job->dbins;
    out->blk = (job->flags & WAR_F_SHAPE) ? (job->blk ? job->blk : (job->n & -job->n)) : 0;
}

int war_enumerate_plain(const war_job* job, war_result* out) {
    int st = check_job(job);
    if (st) return st;
    if (!out) return fail(WAR_EINVAL, "out is NULL");
    init_result(job, out);
    if (job->lo == job->hi) return WAR_OK;
    if ((st = ensure_ready())) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    const int n = job->n, per = 256, threads = 256;
    PlainArgs a;
    memset(&a, 0, sizeof a);
    fill_fact(a.fact);
    a.n = n; a.per = per; a.hbins = job->hbins; a.dbins = job->dbins;
    a.half = (job->flags & WAR_F_HALF) ? 1 : 0;
    a.blk = out->blk;
    a.distinct = (job->flags & WAR_F_DISTINCT) ? 1 : 0;
    a.sample = (job->flags & WAR_F_SAMPLE) ? 1 : 0;
    a.seed = job->seed;
    a.thr = ((u64)job->sample_ppm << 32) / 1000000u;
    if (job->mode == WAR_DEALS) {
        // gpu/war_gpu.py:310-328: spans of batch_threads * per ranks
        const u64 bt = 1ull << 18, span = bt * per;
        for (u64 s = job->lo; s < job->hi; s += span) {
            u64 nth = std::min<u64>(bt, (job->hi - s + per - 1) / per);
            a.start = s; a.total = job->hi;
            st = run_launch([&](cudaStream_t x) { return launch_plain(a, 0, job->rule, threads, nth, ctx().d_acc, x); }, &out->kernel_ms);
            if (st) return st;
            merge_acc(*ctx().h_acc, out, job->hbins, job->dbins);
        }
        return WAR_OK;
    }
    // canon: orders of the n-1 other cards, clipped to the position range (gpu/war_gpu.py:276-280)
    const u64 s = (u64)(n - 1);
    u64 bt = std::max<u64>(1ull << 12, (1ull << 18) / s);
    bt = std::max<u64>(threads, bt / threads * threads);
    const u64 span = bt * per;
    a.pos_lo = job->lo; a.pos_hi = job->hi;
    u64 o0 = job->lo / s, o1 = (job->hi + s - 1) / s;
    for (u64 o = o0; o < o1; o += span) {
        u64 nth = std::min<u64>(bt, (o1 - o + per - 1) / per);
        a.start = o; a.total = o1;
        st = run_launch([&](cudaStream_t x) { return launch_plain(a, 1, job->rule, threads, nth, ctx().d_acc, x); }, &out->kernel_ms);
        if (st) return st;
        merge_acc(*ctx().h_acc, out, job->hbins, job->dbins);
    }
    return WAR_OK;
}

// The context's memo table for a job: 2^bits words, cleared unless the job asks to keep the table the
// previous job of the same n, rule and entry layout left.  kind names the layout: 1 the held-out engine;
// for the main engine 4 * form + 2 * shape, with form 1 (landmarks, key | lam << shift), 2 (all cycle
// states, same packing) or 3 (path entries, (key * C) << bits | value) and shape = 1 when cycle values
// carry the loop-shape code.  Two layouts never share a table: an entry of one form read as another could
// name a different state.
static int prepare_memo(Ctx& c, const war_job* job, int bits, int kind, u64** table) {
    cudaError_t e;
    const size_t bytes = sizeof(u64) << bits;
    const bool keep = (job->flags & WAR_F_MEMO_KEEP) && c.memo_bits == bits && c.memo_n == job->n &&
                      c.memo_rule == job->rule && c.memo_kind == kind;
    if (c.memo_bits != bits) {
        if (c.d_memo) cudaFree(c.d_memo);
        c.d_memo = nullptr;
        c.memo_bits = 0;
        if ((e = cudaMalloc(&c.d_memo, bytes)) != cudaSuccess) {
            c.d_memo = nullptr;
            return cuda_fail(e, "cudaMalloc cycle memo");
        }
        c.memo_bits = bits;
    }
    if (!keep && (e = cudaMemsetAsync(c.d_memo, 0, bytes, cur_stream())) != cudaSuccess) {
        c.memo_n = -1;
        return cuda_fail(e, "clear cycle memo");
    }
    c.memo_n = job->n;
    c.memo_rule = job->rule;
    c.memo_kind = kind;
    *table = c.d_memo;
    return WAR_OK;
}

int war_enumerate_held(const war_job* job, const war_tune* tune, war_result* out) {
    if (!job) return fail(WAR_EINVAL, "job is NULL");
    if (!out) return fail(WAR_EINVAL, "out is NULL");
    if (job->mode != WAR_DEALS || job->n < 2 || job->n > 17)
        return fail(WAR_EINVAL, "the held-out engine plays deals of 2..17 cards (n=%d, mode=%d)", job->n, job->mode);
    if (job->rule != 0 && job->rule != 1) return fail(WAR_EINVAL, "rule=%d", job->rule);
    if (job->flags & ~WAR_F_MEMO_KEEP) return fail(WAR_EINVAL, "flags=0x%x: none apply to the held-out engine", job->flags);
    if (job->hbins < 0 || job->hbins > WAR_HBINS_MAX) return fail(WAR_EINVAL, "hbins=%d", job->hbins);
    if (job->lo > job->hi || job->hi > fact(job->n))
        return fail(WAR_EINVAL, "range [%llu, %llu) outside the %d! deals", (unsigned long long)job->lo,
                    (unsigned long long)job->hi, job->n);
    memset(out, 0, sizeof *out);
    out->hbins = job->hbins;
    if (job->lo == job->hi) return WAR_OK;
    int st;
    if ((st = ensure_ready())) return st;
    const bool memo = tune && (tune->variant & 4);   // the path memo (any variant with bit 2)
    const int threads = (tune && tune->threads) ? tune->threads : (memo ? 256 : 512);
    const int block_m = std::min(job->n, (tune && tune->block_m) ? tune->block_m : 6);
    const int W = (tune && tune->window) ? tune->window : 32;
    const int defer = (tune && tune->defer) ? tune->defer : (memo ? 16 : 32);
    const int memo_bits = (tune && tune->memo_bits) ? tune->memo_bits : 28;
    if (memo && (memo_bits < 12 || memo_bits > 31)) return fail(WAR_EINVAL, "tune.memo_bits=%d (12..31)", memo_bits);
    if (threads < 64 || threads > 1024 || (threads & 31)) return fail(WAR_EINVAL, "tune.threads=%d", threads);
    if (block_m < 1 || block_m > 8) return fail(WAR_EINVAL, "tune.block_m=%d (1..8)", block_m);
    if (W < 1 || W > (1 << 16) || (W & (W - 1))) return fail(WAR_EINVAL, "tune.window=%d", W);
    if (defer < 1 || defer > 32) return fail(WAR_EINVAL, "tune.defer=%d (1..32)", defer);
    // the turn (variant & 3): 0 the counts packed in one word with multiply-add card arithmetic (the default),
    // 1 multiply-adds on separate counts, 2 packed counts in logic/shift form, 3 the plain branching turn of
    // gpu/war17.py; bit 3 tests the tortoise checkpoint after every turn instead of saving it at the services
    static const int form_of_variant[4] = {3, 1, 2, 0};
    const int form = form_of_variant[tune ? (tune->variant & 3) : 0];
    HeldArgs a;
    memset(&a, 0, sizeof a);
    a.W = W; a.defer = defer; a.form = form; a.svc_off = (tune && (tune->variant & 8)) ? 1 : 0;
    const int maxb = held_max_blocks_per_sm(job->rule, threads, job->hbins, memo, form, held_svc(a));
    if (maxb < 1) return fail(WAR_EINVAL, "launch shape threads=%d does not fit an SM%s", threads,
                              memo ? " (at most 512 with the memo)" : "");
    const int bps = (tune && tune->blocks_per_sm) ? std::min(tune->blocks_per_sm, maxb) : maxb;
    std::lock_guard<std::mutex> lk(ctx().mu);
    Ctx& c = ctx();
    Plan p;
    make_plan(job, block_m, p);
    if (p.extra.size() > Ctx::UNIT_CAP) return fail(WAR_EINVAL, "plan has %zu extra units", p.extra.size());
    cudaError_t e;
    if (!p.extra.empty() &&
        (e = cudaMemcpyAsync(c.d_units, p.extra.data(), sizeof(Unit) * p.extra.size(), cudaMemcpyHostToDevice,
                             cur_stream())) != cudaSuccess)
        return cuda_fail(e, "copy units");
    for (int i = 0; i <= 17; i++) a.fact[i] = fact(i);
    a.n = job->n; a.m = block_m; a.rule = job->rule; a.hbins = job->hbins;
    a.units = c.d_units;
    a.tk.k16 = 16u; a.tk.km16 = (u32)-16; a.tk.k2p28 = 1u << 28; a.tk.k4 = 4u; a.tk.one = 1u;
    if (memo) {
        if ((st = prepare_memo(c, job, memo_bits, 1, &a.memo))) return st;
        a.memo_bits = (u32)memo_bits;
    }
    // each launch plays fewer than 2^32 - 2^24 games (32-bit per-lane counters)
    const u64 per_unit = fact(block_m);
    const u64 max_units = std::max<u64>(1, ((1ull << 32) - (1ull << 24)) / per_unit);
    u64 done_main = 0;
    bool extras_done = p.extra.empty();
    while (done_main < p.main_count || !extras_done) {
        const u64 take = std::min<u64>(max_units, p.main_count - done_main);
        const bool last = done_main + take >= p.main_count;
        a.main_base = p.main_base + done_main;
        a.main_count = take;
        a.n_units = take + (last ? p.extra.size() : 0);
        st = run_launch([&](cudaStream_t x) { return launch_held(a, threads, bps * c.sm_count, c.d_acc, x); },
                        &out->kernel_ms);
        if (st) return st;
        merge_acc(*c.h_acc, out, job->hbins, 0);
        out->units += a.n_units;
        done_main += take;
        if (last) extras_done = true;
    }
    return WAR_OK;
}

int war_enumerate(const war_job* job, const war_tune* tune, war_result* out) {
    if (job && job->n == 17 && job->mode == WAR_DEALS) return war_enumerate_held(job, tune, out);   // 17 cards
    int st = check_job(job);
    if (st) return st;
    if (!out) return fail(WAR_EINVAL, "out is NULL");
    init_result(job, out);
    if (job->lo == job->hi) return WAR_OK;
    if (job->mode == WAR_DEALS && job->n == 1) {
        // the single 1-card deal: player 2 has no card, the game is over before it starts (gpu/war_gpu.py:80)
        out->done = 1;
        out->endhist[0] = 1;
        if ((job->flags & WAR_F_SAMPLE) && war_sample_pick(job->seed, job->sample_ppm, 0x10ull, 0x1ull)) {
            out->s_count = 1;
        }
        return WAR_OK;
    }
    Tune t;
    if ((st = resolve_tune(job, tune, t))) return st;
    if ((st = ensure_ready())) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    Ctx& c = ctx();
    Plan p;
    make_plan(job, t.block_m, p);
    if (p.extra.size() > Ctx::UNIT_CAP) return fail(WAR_EINVAL, "plan has %zu extra units", p.extra.size());
    cudaError_t e;
    if (!p.extra.empty()) {
        if ((e = cudaMemcpyAsync(c.d_units, p.extra.data(), sizeof(Unit) * p.extra.size(), cudaMemcpyHostToDevice,
                                 cur_stream())) != cudaSuccess)
            return cuda_fail(e, "copy units");
    }
    BatchArgs a;
    memset(&a, 0, sizeof a);
    fill_fact(a.fact);
    a.n = job->n; a.m = t.block_m; a.hbins = job->hbins; a.dbins = job->dbins;
    a.blk = out->blk; a.W = t.window; a.defer = t.defer;
    a.tk.k16 = 16u; a.tk.km16 = (u32)-16; a.tk.k2p28 = 1u << 28; a.tk.k4 = 4u; a.tk.one = 1u;
    a.tk.c0 = 2 * job->n - 4; a.tk.end2 = (u32)(4 * job->n * job->n);
    a.half = (job->flags & WAR_F_HALF) ? 1 : 0;
    a.sample = (job->flags & WAR_F_SAMPLE) ? 1 : 0;
    a.distinct = (job->flags & WAR_F_DISTINCT) && job->mode == WAR_CANON ? 1 : 0;
    a.seed = job->seed;
    a.thr = ((u64)job->sample_ppm << 32) / 1000000u;
    a.units = c.d_units;
    a.chunk = (u32)t.chunk;
    if (t.variant & 4) {   // the cycle memo
        // its entry layout: the form the variant selects, and the shape-carrying values of a canonical scan
        // with the loop-shape test
        const int form = (t.variant & 24) == 24 ? 3 : ((t.variant & 8) ? 2 : 1);
        const int kind = 4 * form + ((job->mode == WAR_CANON && (job->flags & WAR_F_SHAPE)) ? 2 : 0);
        if ((st = prepare_memo(c, job, t.memo_bits, kind, &a.memo))) return st;
        a.memo_bits = (u32)t.memo_bits;
    }
    // Each launch plays fewer than 2^32 games, so the 32-bit per-block and per-lane counters cannot wrap.
    const u64 per_unit = fact(t.block_m) * p.games_per_order;
    const u64 max_units = std::max<u64>(1, ((1ull << 32) - (1ull << 24)) / per_unit);
    BatchShape bs;
    bs.threads = t.threads; bs.games = t.games; bs.blocks = t.blocks_per_sm * c.sm_count; bs.variant = t.variant;
    const int shape = (job->flags & WAR_F_SHAPE) && job->mode == WAR_CANON ? 1 : 0;
    u64 done_main = 0;
    bool extras_done = p.extra.empty();
    while (done_main < p.main_count || !extras_done) {
        u64 take = std::min<u64>(max_units, p.main_count - done_main);
        bool last = done_main + take >= p.main_count;
        a.main_base = p.main_base + done_main;
        a.main_count = take;
        a.n_units = take + (last ? p.extra.size() : 0);
        st = run_launch([&](cudaStream_t x) { return launch_batched(a, job->mode == WAR_CANON, job->rule, shape, bs, c.d_acc, x); },
                        &out->kernel_ms);
        if (st) return st;
        merge_acc(*c.h_acc, out, job->hbins, job->dbins);
        out->units += a.n_units;
        done_main += take;
        if (last) extras_done = true;
    }
    return WAR_OK;
}

int war_floyd_sample(const war_job* job, war_result* out) {
    int st = check_job(job);
    if (st) return st;
    if (!out) return fail(WAR_EINVAL, "out is NULL");
    init_result(job, out);
    if (job->lo == job->hi || job->sample_ppm == 0) return WAR_OK;
    if (job->mode == WAR_DEALS && job->n == 1) {
        if (war_sample_pick(job->seed, job->sample_ppm, 0x10ull, 0x1ull)) out->s_count = 1;
        return WAR_OK;
    }
    if ((st = ensure_ready())) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    return floyd_sample_run(job, out);
}

}  // extern "C"
