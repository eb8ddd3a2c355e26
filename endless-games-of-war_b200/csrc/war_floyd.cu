// war_floyd.cu — the Floyd cross-check on a seeded sample.
//
// The reference confirms war_gpu.py with a second program that detects cycles with Floyd's tortoise
// and hare (gpu/war_gpu_floyd.py:95-105).  Here the check runs on a seeded sample of the job: a scan
// kernel walks the job's ranks in lexicographic order with its own unrank / next-permutation (not the
// refill kernel's Heap order), keeps the positions whose hash is in the sample, and appends them to a
// buffer; a second kernel plays every buffered position with Floyd, refilling lanes from the buffer.
// The resulting sample aggregates (count, cycling, sum of cycle lengths, sum and maximum of ending
// lengths) must equal those the Brent kernels accumulate for the same sample.
#include "war_kernels.cuh"

namespace war {

// Scan: thread t takes per consecutive ranks from a.start + t*per (rank space of the job: deals, or
// positions = order * (n-1) + split).  Sampled starting positions are appended to buf (sentinel piles).
__global__ void __launch_bounds__(256) sample_scan_kernel(const FloydArgs a, ulonglong2* __restrict__ buf,
                                                          u64 cap, DevAcc* __restrict__ acc) {
    const u32 n = (u32)a.n;
    u64 tid = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u64 idx = a.start + tid * (u64)a.per;
    u64 cnt = 0;
    if (idx < a.total) { cnt = a.total - idx; if (cnt > (u64)a.per) cnt = (u64)a.per; }
    if (cnt == 0) return;
    if (!a.canon) {
        const u64 s1 = sentinel_bit((n + 1u) / 2u), s2 = sentinel_bit(n / 2u);
        const u64 pat = 0x1111111111111111ull * (u64)(n - 1u);
        u64 p = unrank_packed(idx, (int)n, a.fact);
        for (u64 k = 0; k < cnt; k++) {
            bool take = true;
            if (a.half) {
                u64 x = p ^ pat;
                u64 z = (x - 0x1111111111111111ull) & ~x & 0x8888888888888888ull;
                take = (((u32)(__ffsll((long long)z) - 1) >> 2) & 1u) == 0u;
            }
            if (take && n > 1u) {
                u64 w1 = compact_even_nibbles(p) | s1, w2 = compact_even_nibbles(p >> 4) | s2;
                if (war_pick(a.seed, a.thr, w1, w2)) {
                    u64 slot = atomicAdd(&acc->units, 1ull);
                    if (slot < cap) buf[slot] = make_ulonglong2(w1, w2);
                }
            }
            if (k + 1 < cnt) p = next_perm_packed(p, (int)n);
        }
    } else {
        const u32 m = n - 1u;
        u64 perm = idx / m;
        u32 k = (u32)(idx % m);
        u64 qp = unrank_packed(perm, (int)m, a.fact);
        for (u64 i = 0; i < cnt; i++) {
            u64 w1, w2; u32 q;
            canon_position(qp, n, k, w1, w2, q);
            if (war_pick(a.seed, a.thr, w1, w2)) {
                u64 slot = atomicAdd(&acc->units, 1ull);
                if (slot < cap) buf[slot] = make_ulonglong2(w1, w2);
            }
            if (++k == m) { k = 0; if (i + 1 < cnt) qp = next_perm_packed(qp, (int)m); }
        }
    }
}

// 4 * (length of a sentinel pile)
__device__ __forceinline__ u32 pile_q(u64 w) { return 4u * ((63u - (u32)__clzll((long long)w)) >> 2); }

// Floyd over the buffered positions.  Each lane keeps one game: phase 0 moves the hare two turns and
// the tortoise one until the game ends or they meet; phase 1 walks the loop once from the meeting
// point to measure its length.  Lanes refill from the buffer through an atomic counter.
template <int RULE>
__global__ void __launch_bounds__(256) floyd_kernel(const ulonglong2* __restrict__ buf, u64 cap, int n_,
                                                    DevAcc* __restrict__ acc) {
    const u32 n = (u32)n_, n4 = 4u * n, k4m4 = 4u * (n - 1u);
    const u64 count = acc->units < cap ? acc->units : cap;   // positions the scan appended
    u64 h1 = 1, h2 = 1, t1 = 1, t2 = 1, m1 = 1, m2 = 1;
    u32 hq = 0, tq = 0, steps = 0, lam = 0, phase = 0;
    bool active = false;
    u64 sc = 0, scy = 0, slam = 0, slen = 0, smax = 0;
    auto refill = [&]() {
        u64 i = atomicAdd(&acc->work_next, 1ull);
        active = i < count;
        if (active) {
            ulonglong2 e = buf[i];
            h1 = t1 = e.x; h2 = t2 = e.y;
            hq = tq = pile_q(e.x);
            steps = 0; lam = 0; phase = 0;
        }
    };
    refill();
    for (;;) {
        bool fin = false, cyc = false;
        if (active && (steps > WAR_TURN_CAP || lam > WAR_TURN_CAP)) {   // never expected: abandon and flag
            atomicAdd(&acc->status, 1ull);
            refill();
        }
        if (active) {
            if (phase == 0u) {
                war_turn<RULE>(h1, h2, hq, k4m4); steps++;
                if (hq == 0u || hq == n4) fin = true;
                else {
                    war_turn<RULE>(h1, h2, hq, k4m4); steps++;
                    if (hq == 0u || hq == n4) fin = true;
                    else {
                        war_turn<RULE>(t1, t2, tq, k4m4);
                        if (t1 == h1 && t2 == h2) { phase = 1u; m1 = h1; m2 = h2; lam = 0; }
                    }
                }
            } else {
                war_turn<RULE>(h1, h2, hq, k4m4);
                lam++;
                if (h1 == m1 && h2 == m2) { fin = true; cyc = true; }
            }
        }
        if (fin) {
            sc++;
            if (cyc) { scy++; slam += lam; }
            else { slen += steps; if (steps > smax) smax = steps; }
            refill();
        }
        if (!__any_sync(WAR_FULL_MASK, active)) break;
    }
    sc = warp_sum(sc); scy = warp_sum(scy); slam = warp_sum(slam); slen = warp_sum(slen); smax = warp_max(smax);
    if ((threadIdx.x & 31) == 0 && sc) {
        atomicAdd(&acc->s_count, sc); atomicAdd(&acc->s_cyc, scy); atomicAdd(&acc->s_lamsum, slam);
        atomicAdd(&acc->s_lensum, slen); atomicMax(&acc->s_maxfin, smax);
    }
}

// Floyd over the whole job, for a sample rate of 100% (the full-range cross-check of gpu/war_gpu_floyd.py:
// the reference's second program plays every deal with Floyd, data/long_runs.txt:35).  No buffer: lanes take
// chunks of `per` consecutive ranks from an atomic counter, unrank the first (the plain kernel's
// lexicographic unrank, not the refill kernel's Heap order), step with next-permutation, and play each
// position with Floyd's tortoise and hare, taking the next position as soon as a game is decided.  The
// sample predicate still applies below a rate of 100%, so any sample can be played this way as well.
template <int RULE, bool CANON>
__global__ void __launch_bounds__(256) floyd_enum_kernel(const FloydArgs a, DevAcc* __restrict__ acc) {
    const u32 n = (u32)a.n, n4 = 4u * n, k4m4 = 4u * (n - 1u), m = CANON ? n - 1u : n;
    const bool all = a.thr >= (1ull << 32);
    const u64 s1 = sentinel_bit((n + 1u) / 2u), s2 = sentinel_bit(n / 2u);
    const u64 pat = 0x1111111111111111ull * (u64)(n - 1u);
    u64 r = 0, rend = 0, p = 0;   // the lane's chunk: next rank r of [.., rend), p its order
    u32 k = 0;                    // canonical split of rank r
    bool fresh = true;            // p must be unranked from r (first rank of a chunk)
    // next position of the lane's chunks into (h1, h2, hq); false when the job is exhausted
    auto next = [&](u64& w1, u64& w2, u32& q) -> bool {
        for (;;) {
            if (r >= rend) {
                const u64 c = atomicAdd(&acc->work_next, 1ull);
                r = a.start + c * (u64)a.per;
                if (c >= (a.total - a.start + (u64)a.per - 1) / (u64)a.per || r >= a.total) { r = rend = 0; return false; }
                rend = min(a.total, r + (u64)a.per);
                fresh = true;
            }
            if (fresh) {
                if (CANON) { p = unrank_packed(r / m, (int)m, a.fact); k = (u32)(r % m); }
                else p = unrank_packed(r, (int)n, a.fact);
                fresh = false;
            }
            bool take = true;
            if (CANON) {
                canon_position(p, n, k, w1, w2, q);
                if (++k == m) { k = 0; p = next_perm_packed(p, (int)m); }
            } else {
                if (a.half) {
                    const u64 x = p ^ pat;
                    const u64 z = (x - 0x1111111111111111ull) & ~x & 0x8888888888888888ull;
                    take = (((u32)(__ffsll((long long)z) - 1) >> 2) & 1u) == 0u;
                }
                w1 = compact_even_nibbles(p) | s1;
                w2 = compact_even_nibbles(p >> 4) | s2;
                q = 4u * ((n + 1u) / 2u);
                p = next_perm_packed(p, (int)n);
            }
            r++;
            if (take && (all || war_pick(a.seed, a.thr, w1, w2))) return true;
        }
    };
    u64 h1 = 1, h2 = 1, t1 = 1, t2 = 1, m1 = 1, m2 = 1;
    u32 hq = 0, tq = 0, steps = 0, lam = 0, phase = 0;
    u64 sc = 0, scy = 0, slam = 0, slen = 0, smax = 0;
    bool active = next(h1, h2, hq);
    t1 = h1; t2 = h2; tq = hq;
    for (;;) {
        if (active) {
            bool fin = false, cyc = false;
            if (steps > WAR_TURN_CAP || lam > WAR_TURN_CAP) {   // never expected: abandon and flag
                atomicAdd(&acc->status, 1ull);
                fin = true;
            } else if (phase == 0u) {
                war_turn<RULE>(h1, h2, hq, k4m4); steps++;
                if (hq == 0u || hq == n4) fin = true;
                else {
                    war_turn<RULE>(h1, h2, hq, k4m4); steps++;
                    if (hq == 0u || hq == n4) fin = true;
                    else {
                        war_turn<RULE>(t1, t2, tq, k4m4);
                        if (t1 == h1 && t2 == h2) { phase = 1u; m1 = h1; m2 = h2; lam = 0; }
                    }
                }
            } else {
                war_turn<RULE>(h1, h2, hq, k4m4);
                lam++;
                if (h1 == m1 && h2 == m2) { fin = true; cyc = true; }
            }
            if (fin) {
                sc++;
                if (cyc) { scy++; slam += lam; }
                else { slen += steps; if (steps > smax) smax = steps; }
                active = next(h1, h2, hq);
                t1 = h1; t2 = h2; tq = hq; steps = 0; lam = 0; phase = 0;
            }
        }
        if (!__any_sync(WAR_FULL_MASK, active)) break;
    }
    sc = warp_sum(sc); scy = warp_sum(scy); slam = warp_sum(slam); slen = warp_sum(slen); smax = warp_max(smax);
    if ((threadIdx.x & 31) == 0 && sc) {
        atomicAdd(&acc->s_count, sc); atomicAdd(&acc->s_cyc, scy); atomicAdd(&acc->s_lamsum, slam);
        atomicAdd(&acc->s_lensum, slen); atomicMax(&acc->s_maxfin, smax);
    }
}

cudaError_t launch_floyd_enum(const FloydArgs& a, int blocks, DevAcc* acc, cudaStream_t st) {
    if (a.canon) {
        if (a.rule) floyd_enum_kernel<1, true><<<blocks, 256, 0, st>>>(a, acc);
        else floyd_enum_kernel<0, true><<<blocks, 256, 0, st>>>(a, acc);
    } else {
        if (a.rule) floyd_enum_kernel<1, false><<<blocks, 256, 0, st>>>(a, acc);
        else floyd_enum_kernel<0, false><<<blocks, 256, 0, st>>>(a, acc);
    }
    note_launch();
    return cudaGetLastError();
}

int floyd_enum_blocks_per_sm(int canon, int rule) {
    int nb = 0;
    const void* fn = canon ? (rule ? (const void*)floyd_enum_kernel<1, true> : (const void*)floyd_enum_kernel<0, true>)
                           : (rule ? (const void*)floyd_enum_kernel<1, false> : (const void*)floyd_enum_kernel<0, false>);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, 256, 0) != cudaSuccess) return 1;
    return nb > 0 ? nb : 1;
}

cudaError_t launch_sample_scan(const FloydArgs& a, int threads, u64 nthreads, ulonglong2* buf, u64 cap, DevAcc* acc,
                               cudaStream_t st) {
    if (nthreads == 0) return cudaSuccess;
    u64 blocks = (nthreads + (u64)threads - 1) / (u64)threads;
    sample_scan_kernel<<<(unsigned)blocks, threads, 0, st>>>(a, buf, cap, acc);
    note_launch();
    return cudaGetLastError();
}

cudaError_t launch_floyd_play(const ulonglong2* buf, u64 cap, int n, int rule, int blocks, int threads, DevAcc* acc,
                              cudaStream_t st) {
    if (rule) floyd_kernel<1><<<blocks, threads, 0, st>>>(buf, cap, n, acc);
    else floyd_kernel<0><<<blocks, threads, 0, st>>>(buf, cap, n, acc);
    note_launch();
    return cudaGetLastError();
}

}  // namespace war
