// war_plain.cu — the plain kernels: the reference's method (gpu/war_gpu.py:121-259) restated for
// sm_100a.  Each thread takes `per` consecutive lexicographic ranks, unranks the first one and steps
// with next-permutation; every game runs Brent with the reference's checkpoint schedule, so the turn
// totals equal the reference's.  Differences from the reference kernel: the permutation lives in a
// register as packed nibbles (no local-memory byte array), piles are sentinel piles (war_core.cuh),
// the loop-shape test runs on the fly without a bit buffer, and per-thread totals are reduced with
// warp shuffles before one global atomic per warp.
#include "war_kernels.cuh"

namespace war {

// Brent from a starting position (war_sim, gpu/war_gpu.py:77-96) with the first tortoise window W
// (W = 1: the reference's schedule; tortoise saved at steps 1, 3, 7, ...).  Returns 1 for a cycle
// (lam = exact cycle length, the piles hold the state at detection), 0 for a game that ends
// (rounds = its length), 2 if the turn cap was hit.
template <int RULE>
__device__ __forceinline__ int brent_play(u64& w1, u64& w2, u32& q, u32 n4, u32 k4m4, u32 W, u32& rounds, u32& lam,
                                          u32& tstep) {
    u64 t1 = w1, t2 = w2;
    u32 next = W;
    rounds = 0;
    tstep = 0;
    for (;;) {
        war_turn<RULE>(w1, w2, q, k4m4);
        rounds++;
        if (q == 0u || q == n4) return 0;
        if (w1 == t1 && w2 == t2) { lam = rounds - tstep; return 1; }
        if (rounds == next) {
            if (next > WAR_TURN_CAP) return 2;
            t1 = w1; t2 = w2; tstep = next; next = 2u * next + W;
        }
    }
}

template <int RULE>
__global__ void __launch_bounds__(256) plain_deals_kernel(const PlainArgs a, DevAcc* __restrict__ acc) {
    extern __shared__ u32 sh[];
    u32* shh = sh;                // cycle-length bins
    u32* she = sh + a.hbins;      // ending-length bins
    for (int b = threadIdx.x; b < a.hbins + WAR_EBINS; b += blockDim.x) sh[b] = 0;
    __syncthreads();

    const u32 n = (u32)a.n, n4 = 4u * n, k4m4 = 4u * (n - 1u);
    const u32 l1 = (n + 1u) / 2u, l2 = n / 2u;
    const u64 s1 = sentinel_bit(l1), s2 = sentinel_bit(l2);
    u64 tid = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u64 idx = a.start + tid * (u64)a.per;
    u64 cnt = 0;
    if (idx < a.total) { cnt = a.total - idx; if (cnt > (u64)a.per) cnt = (u64)a.per; }

    u64 cyc = 0, done = 0, maxfin = 0, turns = 0, capped = 0;
    u64 sc = 0, scy = 0, slam = 0, slen = 0, smax = 0;
    if (cnt) {
        u64 p = unrank_packed(idx, (int)n, a.fact);
        const u64 pat = 0x1111111111111111ull * (u64)(n - 1u);
        for (u64 k = 0; k < cnt; k++) {
            bool take = true;
            if (a.half) {   // gpu/war_gpu.py:151-154: card n-1 must sit at an even deck position
                u64 x = p ^ pat;
                u64 z = (x - 0x1111111111111111ull) & ~x & 0x8888888888888888ull;
                take = ((__ffsll((long long)z) - 1) >> 2 & 1) == 0;
            }
            if (take) {
                const u64 w1s = compact_even_nibbles(p) | s1, w2s = compact_even_nibbles(p >> 4) | s2;
                u64 w1 = w1s, w2 = w2s;
                u32 q = 4u * l1, rounds = 0, lam = 0, tstep = 0;
                int r = (n == 1u) ? 0 : brent_play<RULE>(w1, w2, q, n4, k4m4, 1u, rounds, lam, tstep);
                done++;
                turns += rounds;
                if (r == 1) {
                    cyc++;
                    if (a.hbins) atomicAdd(&shh[lam < (u32)(a.hbins - 1) ? lam : (u32)(a.hbins - 1)], 1u);
                } else if (r == 0) {
                    if (rounds > maxfin) maxfin = rounds;
                    atomicAdd(&she[rounds < WAR_EBINS - 1 ? rounds : WAR_EBINS - 1], 1u);
                } else {
                    capped++;
                }
                if (a.sample && war_pick(a.seed, a.thr, w1s, w2s)) {
                    sc++;
                    if (r == 1) { scy++; slam += lam; }
                    else { slen += rounds; if (rounds > smax) smax = rounds; }
                }
            }
            if (k + 1 < cnt) p = next_perm_packed(p, (int)n);
        }
    }
    cyc = warp_sum(cyc); done = warp_sum(done); turns = warp_sum(turns); maxfin = warp_max(maxfin);
    capped = warp_sum(capped);
    if (a.sample) { sc = warp_sum(sc); scy = warp_sum(scy); slam = warp_sum(slam); slen = warp_sum(slen); smax = warp_max(smax); }
    if ((threadIdx.x & 31) == 0) {
        if (cyc) atomicAdd(&acc->cyc, cyc);
        if (done) atomicAdd(&acc->done, done);
        if (turns) atomicAdd(&acc->turns, turns);
        if (maxfin) atomicMax(&acc->maxfin, maxfin);
        if (capped) atomicAdd(&acc->status, capped);
        if (sc) {
            atomicAdd(&acc->s_count, sc); atomicAdd(&acc->s_cyc, scy); atomicAdd(&acc->s_lamsum, slam);
            atomicAdd(&acc->s_lensum, slen); atomicMax(&acc->s_maxfin, smax);
        }
    }
    __syncthreads();
    flush_hist(shh, acc->hist, a.hbins);
    flush_hist(she, acc->endhist, WAR_EBINS);
}

template <int RULE>
__global__ void __launch_bounds__(256) plain_canon_kernel(const PlainArgs a, DevAcc* __restrict__ acc) {
    extern __shared__ u32 sh[];
    u32* shh = sh;
    u32* she = sh + a.hbins;
    for (int b = threadIdx.x; b < a.hbins + WAR_EBINS; b += blockDim.x) sh[b] = 0;
    __syncthreads();

    const u32 n = (u32)a.n, n4 = 4u * n, k4m4 = 4u * (n - 1u), m = n - 1u;
    u64 tid = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u64 idx = a.start + tid * (u64)a.per;
    u64 cnt = 0;
    if (idx < a.total) { cnt = a.total - idx; if (cnt > (u64)a.per) cnt = (u64)a.per; }

    u64 cyc = 0, done = 0, maxfin = 0, turns = 0, capped = 0, nonstd = 0, unchk = 0, oncyc = 0, dmin = 0;
    u64 sc = 0, scy = 0, slam = 0, slen = 0, smax = 0;
    if (cnt) {
        u64 qp = unrank_packed(idx, (int)m, a.fact);
        for (u64 it = 0; it < cnt; it++) {
            const u64 r0 = (idx + it) * (u64)m;
            for (u32 k = 0; k < m; k++) {
                if (r0 + k < a.pos_lo || r0 + k >= a.pos_hi) continue;
                u64 w1s, w2s; u32 qs;
                canon_position(qp, n, k, w1s, w2s, qs);
                u64 w1 = w1s, w2 = w2s; u32 q = qs, rounds = 0, lam = 0, tstep = 0;
                int r = brent_play<RULE>(w1, w2, q, n4, k4m4, 1u, rounds, lam, tstep);
                done++;
                turns += rounds;
                if (r == 1) {
                    cyc++;
                    if (a.dbins || a.distinct) {   // gpu/war_gpu.py:217-235
                        CycleWalk cw = cycle_walk<RULE>(w1s, w2s, qs, n, lam);
                        if (cw.on) {
                            oncyc++;
                            if (cw.is_min) dmin++;
                            if (a.dbins) {
                                u64 d = cw.sym ? cw.c1 : cw.c1 + cw.c2;
                                atomicAdd(&acc->dhist[d < (u64)(a.dbins - 1) ? d : (u64)(a.dbins - 1)], 1ull);
                            }
                        }
                    }
                    if (a.hbins) atomicAdd(&shh[lam < (u32)(a.hbins - 1) ? lam : (u32)(a.hbins - 1)], 1u);
                    if (a.blk) {   // gpu/war_gpu.py:238-242
                        int shp = loop_shape_walk<RULE>(w1, w2, q, k4m4, lam, (u32)a.blk);
                        if (shp == 1) nonstd++;
                        else if (shp == 2) unchk++;
                    }
                } else if (r == 0) {
                    if (rounds > maxfin) maxfin = rounds;
                    atomicAdd(&she[rounds < WAR_EBINS - 1 ? rounds : WAR_EBINS - 1], 1u);
                } else {
                    capped++;
                }
                if (a.sample && war_pick(a.seed, a.thr, w1s, w2s)) {
                    sc++;
                    if (r == 1) { scy++; slam += lam; }
                    else { slen += rounds; if (rounds > smax) smax = rounds; }
                }
            }
            if (it + 1 < cnt) qp = next_perm_packed(qp, (int)m);
        }
    }
    cyc = warp_sum(cyc); done = warp_sum(done); turns = warp_sum(turns); maxfin = warp_max(maxfin);
    capped = warp_sum(capped); nonstd = warp_sum(nonstd); unchk = warp_sum(unchk);
    oncyc = warp_sum(oncyc); dmin = warp_sum(dmin);
    if (a.sample) { sc = warp_sum(sc); scy = warp_sum(scy); slam = warp_sum(slam); slen = warp_sum(slen); smax = warp_max(smax); }
    if ((threadIdx.x & 31) == 0) {
        if (cyc) atomicAdd(&acc->cyc, cyc);
        if (done) atomicAdd(&acc->done, done);
        if (turns) atomicAdd(&acc->turns, turns);
        if (maxfin) atomicMax(&acc->maxfin, maxfin);
        if (capped) atomicAdd(&acc->status, capped);
        if (nonstd) atomicAdd(&acc->shape_nonstd, nonstd);
        if (unchk) atomicAdd(&acc->shape_unchecked, unchk);
        if (oncyc) atomicAdd(&acc->oncycle, oncyc);
        if (dmin) atomicAdd(&acc->distinct_min, dmin);
        if (sc) {
            atomicAdd(&acc->s_count, sc); atomicAdd(&acc->s_cyc, scy); atomicAdd(&acc->s_lamsum, slam);
            atomicAdd(&acc->s_lensum, slen); atomicMax(&acc->s_maxfin, smax);
        }
    }
    __syncthreads();
    flush_hist(shh, acc->hist, a.hbins);
    flush_hist(she, acc->endhist, WAR_EBINS);
}

cudaError_t launch_plain(const PlainArgs& a, int canon, int rule, int threads, u64 nthreads, DevAcc* acc,
                         cudaStream_t st) {
    if (nthreads == 0) return cudaSuccess;
    u64 blocks = (nthreads + (u64)threads - 1) / (u64)threads;
    size_t shmem = sizeof(u32) * (size_t)(a.hbins + WAR_EBINS);
    if (canon) {
        if (rule) plain_canon_kernel<1><<<(unsigned)blocks, threads, shmem, st>>>(a, acc);
        else plain_canon_kernel<0><<<(unsigned)blocks, threads, shmem, st>>>(a, acc);
    } else {
        if (rule) plain_deals_kernel<1><<<(unsigned)blocks, threads, shmem, st>>>(a, acc);
        else plain_deals_kernel<0><<<(unsigned)blocks, threads, shmem, st>>>(a, acc);
    }
    note_launch();
    return cudaGetLastError();
}

}  // namespace war
