// war_wide.cu — the 5-bit-pile engine: deals of up to 20 cards (gpu/war24.py).
//
// Past 16 cards a pile no longer fits one 64-bit word of 4-bit cards.  gpu/war24.py keeps 5-bit cards in
// two 64-bit words (lo, hi) with explicit lengths and counts every deal of n <= 20 cards (deal ranks are
// 64-bit) with one of two cycle tests under a step cap (gpu/war24.py:31-125).  This engine plays the same
// games with the refill design of the 4-bit engine:
//
// * Sentinel piles of 5-bit cards.  A pile of len cards is a 128-bit value (two u64): card i (0 = top) in
//   bits 5i..5i+4 and a single 1 bit at bit 5*len, so the length is part of the words and two positions are
//   equal exactly when their four words are.  A turn pops both tops (a 128-bit shift right by 5), compares
//   them and XORs (pair ^ 0x401) << pos into the winner's words, where pos is the winner's sentinel after
//   the pop: the pair replaces the sentinel and a new sentinel appears 10 bits higher.  No branches; the
//   variable 128-bit shift is two clamped 64-bit shifts (PTX shl/shr give 0 for amounts of 64 or more).
// * Refill.  A persistent grid of SMs x resident blocks; each lane plays one game at a time and every K
//   turns the warp services its lanes together: a decided game is recorded and the lane takes its next deal.
//   Outcomes are latched, so the turn loop has no branch on them.
// * Enumeration.  Work units of j! consecutive lexicographic ranks (a fixed prefix and every order of the
//   last j positions) come from one atomic counter; a lane unranks the unit's first deal once and walks the
//   unit in Heap's order (one transposition per deal).  The deck is held split: player 1's cards (even
//   deck positions) in one word and player 2's (odd positions) in another, 5 bits per card, so a deal is
//   the two words plus their sentinels.
// * Detectors (template DET), each with the step cap after which a game counts as undetermined:
//   Brent with the tortoise saved at turns W, 3W, 7W, ... (the default; its cycle length feeds the
//   histogram), Floyd's tortoise and hare (gpu/war24.py:85-97), and the streak test for odd n
//   (gpu/war24.py:98-125): anchor where the next winner holds an even number of cards, then expect the
//   players to alternate for lcm(n+1, W, L-1) turns and compare with the anchor.  Every detector gives the
//   same counts whenever nothing reaches the cap; the step count of an ending game is its length.
#include <algorithm>
#include <cstring>
#include <mutex>
#include "war_kernels.cuh"
#include "war_host.h"

namespace war {

enum { DET_BRENT = 0, DET_FLOYD = 1, DET_STREAK = 2 };
enum { K_NONE = 0, K_END = 1, K_CYC = 2, K_UND = 3 };

__device__ __forceinline__ u64 shr64(u64 x, u32 s) {
    u64 r;
    asm("shr.b64 %0, %1, %2;" : "=l"(r) : "l"(x), "r"(s));
    return r;
}

// One turn on 128-bit sentinel piles (a0, a1) and (b0, b1); la = player 1's length, n1 = n - 1.  Returns
// true if player 1 won.  Rule 0 puts the winning card, then the losing card, under the winner's pile
// (gpu/war24.py:42-47); rule 1 the losing card first.
template <int RULE>
__device__ __forceinline__ bool turn5(u64& a0, u64& a1, u64& b0, u64& b1, u32& la, u32 n1) {
    const u32 c1 = (u32)a0 & 31u, c2 = (u32)b0 & 31u;
    a0 = (a0 >> 5) | (a1 << 59); a1 >>= 5;
    b0 = (b0 >> 5) | (b1 << 59); b1 >>= 5;
    const bool p1 = c1 > c2;
    const u32 hi = max(c1, c2), lo = min(c1, c2);
    const u32 pair = RULE ? (lo | (hi << 5)) : (hi | (lo << 5));
    const u32 pos = 5u * (p1 ? la - 1u : n1 - la);
    const u64 v = (u64)(pair ^ 0x401u);
    const u64 x0 = shl64(v, pos), x1 = shl64(v, pos - 64u) | shr64(v, 64u - pos);
    const u64 m = p1 ? ~0ull : 0ull;
    a0 ^= x0 & m; a1 ^= x1 & m;
    b0 ^= x0 & ~m; b1 ^= x1 & ~m;
    la = p1 ? la + 1u : la - 1u;
    return p1;
}

// The work units of a launch, as in the 4-bit engine (BatchArgs), with the 5-bit engine's own fields.
struct WideArgs {
    u64 fact[21];
    u64 main_base, main_count, n_units;
    const Unit* units;
    int n, m, rule, hbins, W, defer;
    u32 cap;            // step cap: a game undecided after this many turns is undetermined
    u32 lamtab[32];     // streak: lcm(n+1, ws, n-ws-1) for an even next-winner pile ws with n-ws >= 2, else 0
};

__device__ __forceinline__ u32 wide_heap_full(u32 j) {   // Heap counter value of a unit's last order
    u32 f = 0;
    for (u32 i = 1; i < j; i++) f |= i << (4u * i);
    return f;
}

struct WEnum {
    u64 A, B;           // the current deal: player 1's cards (even positions), player 2's (odd), 5 bits each
    u32 ctr, full, base;
    bool live;
};

// Swaps deck positions x and y of the split deck.
__device__ __forceinline__ void swap5(u64& A, u64& B, u32 x, u32 y) {
    const u32 sx = 5u * (x >> 1), sy = 5u * (y >> 1);
    const bool bx = x & 1u, by = y & 1u;
    const u64 t = (((bx ? B : A) >> sx) ^ ((by ? B : A) >> sy)) & 31ull;
    const u64 tx = t << sx, ty = t << sy;
    A ^= (bx ? 0ull : tx) ^ (by ? 0ull : ty);
    B ^= (bx ? tx : 0ull) ^ (by ? ty : 0ull);
}

__device__ __forceinline__ bool wide_fetch(WEnum& E, const WideArgs& a, u64* counter) {
    const u64 u = atomicAdd(counter, 1ull);
    if (u >= a.n_units) return false;
    u64 r;
    u32 j;
    if (u < a.main_count) {
        j = (u32)a.m; r = (a.main_base + u) * a.fact[a.m];
    } else {
        const Unit U = a.units[u - a.main_count];
        r = U.r; j = U.j;
    }
    // lexicographic unrank (gpu/war24.py:60-74) straight into the split deck
    const int n = a.n;
    u32 avail = (1u << n) - 1u;
    u64 A = 0, B = 0;
    for (int i = 0; i < n; i++) {
        const u64 f = a.fact[n - 1 - i];
        const u32 d = (u32)(r / f);
        r -= (u64)d * f;
        u32 mm = avail;
        for (u32 k = 0; k < d; k++) mm &= mm - 1u;
        const u32 v = (u32)(__ffs((int)mm) - 1);
        avail &= ~(1u << v);
        if (i & 1) B |= (u64)v << (5 * (i >> 1));
        else A |= (u64)v << (5 * (i >> 1));
    }
    E.A = A; E.B = B;
    E.ctr = 0;
    E.full = wide_heap_full(j);
    E.base = (u32)n - j;
    E.live = true;
    return true;
}

// Heap's algorithm, one output (as heap_step of the 4-bit engine); false after the unit's last deal.
__device__ __forceinline__ bool wide_heap_step(WEnum& E) {
    const u32 x = E.ctr ^ E.full;
    if (x == 0u) return false;
    const u32 i = (u32)(__ffs((int)x) - 1) >> 2;
    const u32 ci = (E.ctr >> (4u * i)) & 15u;
    const u32 o = (i & 1u) ? ci : 0u;
    swap5(E.A, E.B, E.base + i, E.base + o);
    E.ctr = ((E.ctr >> (4u * i)) + 1u) << (4u * i);
    return true;
}

// SVC (Brent only): W is a multiple of the service period, so an undecided game (which starts at a service and
// plays `period` turns between services) reaches each tortoise checkpoint W, 3W, 7W, ... exactly at a service,
// and the checkpoint is saved there instead of being tested after every turn.
template <int RULE, int DET, bool SVC>
__global__ void __launch_bounds__(1024) wide_kernel(const __grid_constant__ WideArgs a, DevAcc* __restrict__ acc) {
    extern __shared__ u32 sh[];
    u32* shh = sh;                    // cycle-length histogram (Brent)
    u32* she = sh + a.hbins;          // ending-length histogram
    u32* slam = she + WAR_EBINS;      // streak periods by pile size
    for (int b = threadIdx.x; b < a.hbins + WAR_EBINS; b += blockDim.x) sh[b] = 0;
    if (threadIdx.x < 32) slam[threadIdx.x] = a.lamtab[threadIdx.x];
    __syncthreads();

    const u32 n = (u32)a.n, n1 = n - 1u, W = (u32)a.W, cap = a.cap;
    const u32 hb1 = a.hbins > 0 ? (u32)(a.hbins - 1) : 0u;
    const int period = a.defer > 4 ? (a.defer + 3) & ~3 : 4;
    const u32 lenA = (n + 1u) / 2u, lenB = n / 2u;
    const u64 sA = 1ull << (5u * lenA), sB = 1ull << (5u * lenB);
    u64* counter = &acc->work_next;

    WEnum E;
    E.live = false;
    // the game: piles, player 1's length, turns played, outcome
    u64 a0 = 0, a1 = 0, b0 = 0, b1 = 0;
    u32 la = 0, rounds = 0, kind = K_NONE;
    bool active = false;
    // detector state: tortoise (Brent, Floyd) or anchor (streak)
    u64 t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    u32 tla = 0, next = 0, lam = 0, since = 0, prevw = 2u;
    bool anch = false;
    // per-lane totals
    u32 cyc = 0, done = 0, maxfin = 0, und = 0;
    u64 turns = 0;

    auto start = [&]() {
        if (!E.live && !wide_fetch(E, a, counter)) { active = false; kind = K_END; return; }
        a0 = E.A | sA; a1 = 0; b0 = E.B | sB; b1 = 0; la = lenA;
        E.live = wide_heap_step(E);
        active = true;
        done++;
        rounds = 0; kind = K_NONE;
        t0 = a0; t1 = a1; t2 = b0; t3 = b1; tla = la;
        next = W; lam = 0; since = 0; prevw = 2u; anch = false;
    };
    start();
    bool running = __any_sync(WAR_FULL_MASK, active);

    while (running) {
        for (int k = 0; k < period; k++) {
            const bool open = kind == K_NONE;
            if (DET == DET_FLOYD) {
                // two hare turns, one tortoise turn (gpu/war24.py:88-96)
                turn5<RULE>(a0, a1, b0, b1, la, n1);
                const bool e1 = (la == 0u) | (la == n);
                turn5<RULE>(a0, a1, b0, b1, la, n1);
                const bool e2 = (la == 0u) | (la == n);
                turn5<RULE>(t0, t1, t2, t3, tla, n1);
                const bool cy = (a0 == t0) & (a1 == t1) & (b0 == t2) & (b1 == t3);
                const u32 r2 = rounds + (e1 ? 1u : 2u);
                const u32 kk = (e1 | e2) ? (u32)K_END : (cy ? (u32)K_CYC : (r2 > cap ? (u32)K_UND : (u32)K_NONE));
                rounds = open ? r2 : rounds;
                kind = open ? kk : kind;
            } else if (DET == DET_STREAK) {
                // anchor where the next winner holds an even number of cards (gpu/war24.py:104-112)
                if (!anch) {
                    const u32 ws = ((u32)a0 & 31u) > ((u32)b0 & 31u) ? la : n - la;
                    // (a lane whose game is decided keeps stepping it until the service, so its pile
                    // length may leave 0..n: the mask keeps the read inside the 32-entry table)
                    const u32 lt = slam[ws & 31u];
                    if (lt) { anch = true; since = 0; prevw = 2u; lam = lt; t0 = a0; t1 = a1; t2 = b0; t3 = b1; }
                }
                const u32 w = turn5<RULE>(a0, a1, b0, b1, la, n1) ? 1u : 0u;
                bool cy = false;
                if (anch) {   // the players must alternate for lam turns (gpu/war24.py:114-123)
                    if (w == prevw) anch = false;
                    else {
                        prevw = w;
                        if (++since == lam) {
                            cy = (a0 == t0) & (a1 == t1) & (b0 == t2) & (b1 == t3);
                            anch = false;
                        }
                    }
                }
                const u32 r1 = rounds + 1u;
                const bool en = (la == 0u) | (la == n);
                const u32 kk = cy ? (u32)K_CYC : (en ? (u32)K_END : (r1 > cap ? (u32)K_UND : (u32)K_NONE));
                rounds = open ? r1 : rounds;
                kind = open ? kk : kind;
            } else {
                turn5<RULE>(a0, a1, b0, b1, la, n1);
                const u32 r1 = rounds + 1u;
                const bool en = (la == 0u) | (la == n);
                const bool cy = (a0 == t0) & (a1 == t1) & (b0 == t2) & (b1 == t3);
                const u32 kk = en ? (u32)K_END : (cy ? (u32)K_CYC : (r1 > cap ? (u32)K_UND : (u32)K_NONE));
                rounds = open ? r1 : rounds;
                kind = open ? kk : kind;
                if (!SVC && open && kk == K_NONE && r1 == next) {   // Brent: tortoise saved at W, 3W, 7W, ...
                    t0 = a0; t1 = a1; t2 = b0; t3 = b1; next = 2u * next + W;
                }
            }
        }
        if (DET == DET_BRENT && SVC && kind == K_NONE && rounds == next) {   // the checkpoint, at the service
            t0 = a0; t1 = a1; t2 = b0; t3 = b1; next = 2u * next + W;
        }
        // service: record every decided game, refill its lane
        const bool fin = active & (kind != K_NONE);
        if (__any_sync(WAR_FULL_MASK, fin)) {
            if (fin) {
                turns += rounds;
                if (kind == K_CYC) {
                    cyc++;
                    if (DET == DET_BRENT && a.hbins) {
                        const u32 l = rounds - ((next - W) >> 1);
                        atomicAdd(&shh[l < hb1 ? l : hb1], 1u);
                    }
                } else if (kind == K_END) {
                    if (rounds > maxfin) maxfin = rounds;
                    atomicAdd(&she[rounds < WAR_EBINS - 1 ? rounds : WAR_EBINS - 1], 1u);
                } else {
                    und++;
                }
                start();
            }
            running = __any_sync(WAR_FULL_MASK, active);
        }
    }

    const u64 v_cyc = warp_sum(cyc), v_done = warp_sum(done), v_turns = warp_sum(turns), v_max = warp_max(maxfin);
    const u64 v_und = warp_sum(und);
    if ((threadIdx.x & 31) == 0) {
        if (v_cyc) atomicAdd(&acc->cyc, v_cyc);
        if (v_done) atomicAdd(&acc->done, v_done);
        if (v_turns) atomicAdd(&acc->turns, v_turns);
        if (v_max) atomicMax(&acc->maxfin, v_max);
        if (v_und) atomicAdd(&acc->undetermined, v_und);
    }
    __syncthreads();
    flush_hist(shh, acc->hist, a.hbins);
    flush_hist(she, acc->endhist, WAR_EBINS);
}

typedef void (*WideFn)(const WideArgs, DevAcc*);

static WideFn wide_pick(int det, int rule, bool svc) {
    if (det == DET_FLOYD) return rule ? wide_kernel<1, DET_FLOYD, false> : wide_kernel<0, DET_FLOYD, false>;
    if (det == DET_STREAK) return wide_kernel<0, DET_STREAK, false>;
    if (svc) return rule ? wide_kernel<1, DET_BRENT, true> : wide_kernel<0, DET_BRENT, true>;
    return rule ? wide_kernel<1, DET_BRENT, false> : wide_kernel<0, DET_BRENT, false>;
}

// Brent's checkpoints fall on services when W is a multiple of the service period.
static bool wide_svc(int W, int defer) {
    const int period = defer > 4 ? (defer + 3) & ~3 : 4;
    return W % period == 0;
}

static size_t wide_shmem(int hbins) { return sizeof(u32) * (size_t)(hbins + WAR_EBINS + 32); }

static int wide_max_blocks(int det, int rule, bool svc, int threads, int hbins) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, wide_pick(det, rule, svc), threads, wide_shmem(hbins)) !=
        cudaSuccess)
        return 0;
    return nb;
}

}  // namespace war

using namespace war;

extern "C" int war_enumerate_wide(const war_job* job, const war_wide_cfg* cfg, war_result* out) {
    if (!job) return fail(WAR_EINVAL, "job is NULL");
    if (!out) return fail(WAR_EINVAL, "out is NULL");
    war_wide_cfg c;
    memset(&c, 0, sizeof c);
    if (cfg) c = *cfg;
    if (job->mode != WAR_DEALS || job->n < 2 || job->n > 20)
        return fail(WAR_EINVAL, "the 5-bit engine plays deals of 2..20 cards (n=%d, mode=%d)", job->n, job->mode);
    if (job->rule != 0 && job->rule != 1) return fail(WAR_EINVAL, "rule=%d", job->rule);
    if (job->flags & ~WAR_F_MEMO_KEEP) return fail(WAR_EINVAL, "flags=0x%x: none apply to the 5-bit engine", job->flags);
    if (c.det < 0 || c.det > 2) return fail(WAR_EINVAL, "det=%d (0 Brent, 1 Floyd, 2 streak)", c.det);
    if (c.det == DET_STREAK && (!(job->n & 1) || job->rule))
        return fail(WAR_EINVAL, "the streak test holds for odd n and the winner's card first (n=%d, rule=%d)", job->n,
                    job->rule);
    if (job->hbins < 0 || job->hbins > WAR_HBINS_MAX) return fail(WAR_EINVAL, "hbins=%d", job->hbins);
    u64 fn = 1;
    for (int i = 2; i <= job->n; i++) fn *= (u64)i;
    if (job->lo > job->hi || job->hi > fn)
        return fail(WAR_EINVAL, "range [%llu, %llu) outside the %d! deals", (unsigned long long)job->lo,
                    (unsigned long long)job->hi, job->n);
    const u32 cap = c.cap ? c.cap : (1u << 22);
    if (cap > (1u << 30)) return fail(WAR_EINVAL, "cap=%u (at most 2^30)", cap);
    const int threads = c.threads ? c.threads : 256;
    const int block_m = std::min(job->n, c.block_m ? c.block_m : 6);
    const int W = c.window ? c.window : 32;
    const int defer = c.defer ? c.defer : 16;
    if (threads < 64 || threads > 1024 || (threads & 31)) return fail(WAR_EINVAL, "cfg.threads=%d", threads);
    if (block_m < 1 || block_m > 8) return fail(WAR_EINVAL, "cfg.block_m=%d (1..8)", block_m);
    if (W < 1 || W > (1 << 16) || (W & (W - 1))) return fail(WAR_EINVAL, "cfg.window=%d", W);
    if (defer < 1 || defer > 64) return fail(WAR_EINVAL, "cfg.defer=%d (1..64)", defer);
    const int hbins = c.det == DET_BRENT ? job->hbins : 0;
    memset(out, 0, sizeof *out);
    out->hbins = hbins;
    if (job->lo == job->hi) return WAR_OK;
    int st;
    if ((st = ensure_ready())) return st;
    const bool svc = wide_svc(W, defer);
    const int maxb = wide_max_blocks(c.det, job->rule, svc, threads, hbins);
    if (maxb < 1) return fail(WAR_EINVAL, "launch shape threads=%d does not fit an SM", threads);
    const int bps = c.blocks_per_sm ? std::min(c.blocks_per_sm, maxb) : maxb;
    std::lock_guard<std::mutex> lk(ctx().mu);
    Ctx& cx = ctx();
    Plan p;
    make_plan(job, block_m, p);
    if (p.extra.size() > Ctx::UNIT_CAP) return fail(WAR_EINVAL, "plan has %zu extra units", p.extra.size());
    cudaError_t e;
    if (!p.extra.empty() &&
        (e = cudaMemcpyAsync(cx.d_units, p.extra.data(), sizeof(Unit) * p.extra.size(), cudaMemcpyHostToDevice,
                             cur_stream())) != cudaSuccess)
        return cuda_fail(e, "copy units");
    WideArgs a;
    memset(&a, 0, sizeof a);
    a.fact[0] = 1;
    for (int i = 1; i <= 20; i++) a.fact[i] = a.fact[i - 1] * (u64)i;
    a.n = job->n; a.m = block_m; a.rule = job->rule; a.hbins = hbins; a.W = W; a.defer = defer; a.cap = cap;
    a.units = cx.d_units;
    for (int ws = 2; ws + 2 <= job->n; ws += 2) {   // gpu/war24.py:109: lcm(n+1, lcm(W, L-1))
        auto gcd = [](u64 x, u64 y) { while (y) { u64 t = x % y; x = y; y = t; } return x; };
        const u64 l1 = (u64)ws / gcd(ws, job->n - ws - 1) * (u64)(job->n - ws - 1);
        a.lamtab[ws] = (u32)((u64)(job->n + 1) / gcd(job->n + 1, l1) * l1);
    }
    // each launch plays fewer than 2^32 - 2^24 games (32-bit per-lane counters)
    const u64 per_unit = a.fact[block_m];
    const u64 max_units = std::max<u64>(1, ((1ull << 32) - (1ull << 24)) / per_unit);
    const WideFn fnp = wide_pick(c.det, job->rule, svc);
    const size_t shmem = wide_shmem(hbins);
    u64 done_main = 0;
    bool extras_done = p.extra.empty();
    while (done_main < p.main_count || !extras_done) {
        const u64 take = std::min<u64>(max_units, p.main_count - done_main);
        const bool last = done_main + take >= p.main_count;
        a.main_base = p.main_base + done_main;
        a.main_count = take;
        a.n_units = take + (last ? p.extra.size() : 0);
        st = run_launch([&](cudaStream_t x) {
            fnp<<<bps * cx.sm_count, threads, shmem, x>>>(a, cx.d_acc);
            note_launch();
            return cudaGetLastError();
        }, &out->kernel_ms);
        if (st) return st;
        merge_acc(*cx.h_acc, out, hbins, 0);
        out->units += a.n_units;
        done_main += take;
        if (last) extras_done = true;
    }
    return WAR_OK;
}
