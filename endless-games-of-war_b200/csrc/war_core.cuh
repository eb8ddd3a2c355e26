// war_core.cuh — device building blocks shared by every kernel of libwar.so.
//
// Pile layout ("sentinel piles"): a pile of len cards is a uint64 with card i (0 = top) in nibble i
// and a single 1 bit at bit 4*len, just above the last card.  The reference keeps the same 4-bit
// cards with the top card in the low nibble plus explicit lengths (gpu/war_gpu.py:38-45, :98-107);
// here the sentinel makes the length part of the word, so two piles compare equal exactly when the
// positions are equal, and Brent's test (gpu/war_gpu.py:91) is two 64-bit compares.  Player 1's
// length is tracked as q = 4*len1 to place the pushed pair; player 2's is n - len1.
#pragma once
#include <stdint.h>
#include "../../include/war.h"

typedef unsigned long long u64;
typedef unsigned int u32;

#define WAR_FULL_MASK 0xffffffffu

// Variable 64-bit left shift with PTX semantics: shift amounts above 63 give 0 (the amount is
// clamped, PTX ISA shl).  Used where a retired lane may shift by an out-of-range amount.
__device__ __forceinline__ u64 shl64(u64 x, u32 s) {
    u64 r;
    asm("shl.b64 %0, %1, %2;" : "=l"(r) : "l"(x), "r"(s));
    return r;
}

// One turn (WAR_STEP, gpu/war_gpu.py:38-45) on sentinel piles.  k4m4 = 4*(n-1).  Returns 1 if
// player 1 won.  Rule 0 puts the winning card then the losing card under the winner's pile, rule 1
// the losing card first.  The pair (first card in the low nibble) goes where the winner's sentinel
// was after the pop; XOR with pair ^ 0x101 writes both cards, clears the old sentinel bit and sets
// the new one 8 bits higher.
template <int RULE>
__device__ __forceinline__ bool war_turn(u64& w1, u64& w2, u32& q, u32 k4m4) {
    u32 c1 = (u32)w1 & 15u, c2 = (u32)w2 & 15u;
    w1 >>= 4;
    w2 >>= 4;
    bool p1 = c1 > c2;
    u32 hi = max(c1, c2), lo = min(c1, c2);
    u32 pair = RULE ? (lo | (hi << 4)) : (hi | (lo << 4));
    u32 pos = p1 ? q - 4u : k4m4 - q;
    u64 x = shl64((u64)(pair ^ 0x101u), pos);
    u64 m = p1 ? ~0ull : 0ull;
    w1 ^= x & m;
    w2 ^= x & ~m;
    q = p1 ? q + 4u : q - 4u;
    return p1;
}

// Constants of war_turn_fma, passed in from kernel arguments so that the compiler keeps them as
// multiplier operands instead of folding them into shifts.
struct TurnK {
    u32 k16;    // 16
    u32 km16;   // -16
    u32 k2p28;  // 2^28
    u32 k4;     // 4
    u32 one;    // 1
    int c0;     // 2n - 4
    u32 end2;   // (2n)^2
};

// The same turn as war_turn, written so that about half of its integer operations are multiply-adds
// (the FMA pipe) rather than logic / shift operations (the ALU pipe, half rate on sm_100):
//   pop:   lo' = funnel(lo, hi) >> 4, hi' = mulhi(hi, 2^28) = hi >> 4, card = lo - 16*lo' (mod 2^32)
//   pair:  c1 + 16*c2 and c2 + 16*c1 by IMAD, one select
//   push:  the winner's word gains (pair + 0xFF) << pos (the sentinel bit at pos becomes the pair and
//          a new sentinel 8 bits up; the same bits as war_turn's XOR), added as w += x*b with b in {0,1}
//          by mad.wide, so no select or mask is needed
//   length: qq = 4*len1 - 2n, pos = s*qq + (2n-4) and qq += 4s with s = +1 (player 1 won) or -1;
//          the game is over when qq*qq == (2n)^2.
template <int RULE>
__device__ __forceinline__ bool war_turn_fma(u64& w1, u64& w2, u32& qq, const TurnK& K) {
    const u32 l1 = (u32)w1, h1 = (u32)(w1 >> 32), l2 = (u32)w2, h2 = (u32)(w2 >> 32);
    const u32 nl1 = __funnelshift_r(l1, h1, 4), nl2 = __funnelshift_r(l2, h2, 4);
    const u32 nh1 = __umulhi(h1, K.k2p28), nh2 = __umulhi(h2, K.k2p28);
    const u32 c1 = l1 + nl1 * K.km16, c2 = l2 + nl2 * K.km16;
    const bool p1 = c1 > c2;
    const u32 pa = RULE ? c2 + c1 * K.k16 : c1 + c2 * K.k16;   // player 1 won
    const u32 pb = RULE ? c1 + c2 * K.k16 : c2 + c1 * K.k16;   // player 2 won
    const u32 term = (p1 ? pa : pb) + 0xFFu;
    const int s = p1 ? 1 : -1;
    const u32 pos = (u32)(s * (int)qq + K.c0);
    const u64 x = shl64((u64)term, pos);
    const u32 xl = (u32)x, xh = (u32)(x >> 32);
    const u32 b1 = p1 ? 1u : 0u, b2 = K.one - b1;
    u64 a1 = ((u64)nh1 << 32) | nl1, a2 = ((u64)nh2 << 32) | nl2;
    a1 = (u64)xl * b1 + a1;
    a2 = (u64)xl * b2 + a2;
    const u32 a1h = (u32)(a1 >> 32) + xh * b1, a2h = (u32)(a2 >> 32) + xh * b2;
    w1 = ((u64)a1h << 32) | (u32)a1;
    w2 = ((u64)a2h << 32) | (u32)a2;
    qq = qq + (u32)s * K.k4;
    return p1;
}

// The same turn with the rule chosen at run time (serving kernel, checks).
__device__ __forceinline__ bool war_turn_rt(u64& w1, u64& w2, u32& q, u32 k4m4, int rule) {
    return rule ? war_turn<1>(w1, w2, q, k4m4) : war_turn<0>(w1, w2, q, k4m4);
}

// Splitmix64 finaliser and the seeded sample predicate (war_sample_pick in include/war.h).
__host__ __device__ __forceinline__ u64 war_mix64(u64 x) {
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}
__host__ __device__ __forceinline__ bool war_pick(u64 seed, u64 thr, u64 w1s, u64 w2s) {
    u64 x = war_mix64(seed ^ (w1s * 0x9E3779B97F4A7C15ull) ^ (w2s * 0xC2B2AE3D27D4EB4Full));
    return (x >> 32) < thr;
}

// Nibble i of a packed permutation.
__device__ __forceinline__ u32 nib(u64 p, u32 i) { return (u32)(p >> (4u * i)) & 15u; }

// Swaps nibbles at bit offsets sa and sb (multiples of 4, < 64).
__device__ __forceinline__ u64 swap_nibbles(u64 p, u32 sa, u32 sb) {
    u64 t = ((p >> sa) ^ (p >> sb)) & 15ull;
    return p ^ ((t << sa) | (t << sb));
}

// Lexicographic unrank (gpu/war_gpu.py:135-146): the permutation of 0..m-1 with rank r, packed with
// position i in nibble i.  fact[i] = i!.
__device__ __forceinline__ u64 unrank_packed(u64 r, int m, const u64* fact) {
    u32 avail = (1u << m) - 1u;
    u64 p = 0;
    for (int i = 0; i < m; i++) {
        u64 f = fact[m - 1 - i];
        u32 d = (u32)(r / f);
        r -= (u64)d * f;
        u32 mm = avail;
        for (u32 k = 0; k < d; k++) mm &= mm - 1u;   // drop the d lowest unused cards
        u32 v = (u32)(__ffs((int)mm) - 1);
        p |= (u64)v << (4 * i);
        avail &= ~(1u << v);
    }
    return p;
}

// Lexicographic successor (gpu/war_gpu.py:109-119) on a packed permutation of m cards.
__device__ __forceinline__ u64 next_perm_packed(u64 p, int m) {
    int i = m - 2;
    while (i >= 0 && nib(p, i) >= nib(p, i + 1)) i--;
    if (i < 0) return p;
    int j = m - 1;
    u32 ai = nib(p, i);
    while (nib(p, j) <= ai) j--;
    p = swap_nibbles(p, 4u * i, 4u * j);
    for (int l = i + 1, r = m - 1; l < r; l++, r--) p = swap_nibbles(p, 4u * l, 4u * r);
    return p;
}

// Deal (war_cycles, gpu/war_gpu.py:98-107): even deck positions to player 1, odd to player 2, the
// first card on top.  Input: deck packed with position i in nibble i.  Output: card nibbles of each
// pile (no sentinel), by compacting the even and the odd nibbles.
__device__ __forceinline__ u64 compact_even_nibbles(u64 x) {
    x &= 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
    x = (x | (x >> 16)) & 0x00000000FFFFFFFFull;
    return x;
}

// The bit just above a pile of len cards; none for a 16-card word.
__host__ __device__ __forceinline__ u64 sentinel_bit(u32 len) { return len < 16 ? 1ull << (4 * len) : 0ull; }

// Canonical position (gpu/war_gpu.py:210-213) from the packed order q of the m = n-1 other cards and
// split k: player 1 = [n-1, q0..q(k-1)], player 2 = [qk..q(m-1)].  Sentinel piles.
__device__ __forceinline__ void canon_position(u64 q, u32 n, u32 k, u64& w1, u64& w2, u32& q4) {
    u32 m = n - 1;
    u64 lowk = k ? (q & (~0ull >> (64 - 4 * k))) : 0ull;
    w1 = (u64)(n - 1) | (lowk << 4) | (1ull << (4 * (k + 1)));
    w2 = (q >> (4 * k)) | (1ull << (4 * (m - k)));
    q4 = 4 * (k + 1);
}

// Reduction helpers.
__device__ __forceinline__ u64 warp_sum(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(WAR_FULL_MASK, v, o);
    return v;
}
__device__ __forceinline__ u64 warp_max(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u64 t = __shfl_xor_sync(WAR_FULL_MASK, v, o);
        v = t > v ? t : v;
    }
    return v;
}

// Device-side accumulators of one job (zeroed by the host before the launch).
struct DevAcc {
    u64 cyc, done, maxfin, turns, shape_nonstd, shape_unchecked, oncycle, distinct_min;
    u64 s_count, s_cyc, s_lamsum, s_lensum, s_maxfin, units;
    u64 memo_lookups, memo_hits, memo_stores;
    u64 work_next;   // persistent kernel: next work unit
    u64 status;      // nonzero: a game hit the turn cap
    u64 undetermined;   // 5-bit engine: games undecided at the step cap (counted, not an error)
    u64 hist[WAR_HBINS_MAX];
    u64 dhist[WAR_DBINS_MAX];
    u64 endhist[WAR_EBINS];
};

// Adds a block's shared histogram (u32 bins) to the global u64 bins.
__device__ __forceinline__ void flush_hist(const u32* sh, u64* g, int bins) {
    for (int b = threadIdx.x; b < bins; b += blockDim.x)
        if (sh[b]) atomicAdd(&g[b], (u64)sh[b]);
}
