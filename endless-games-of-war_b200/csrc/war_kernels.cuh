// war_kernels.cuh — kernel argument blocks, the cycle walks shared by the plain and batched kernels,
// and the launchers' declarations.
#pragma once
#include <cuda_runtime.h>
#include "war_core.cuh"

namespace war {

// A game that is still running when its tortoise would move past this step is abandoned and the job
// fails with WAR_ECAP.  Every game here is decided after at most a few thousand turns; the cap only
// bounds a faulty path.
constexpr u32 WAR_TURN_CAP = 1u << 24;

struct PlainArgs {
    u64 fact[17];
    u64 start, total;       // rank space of the launch: deals, or orders of the n-1 other cards (canon)
    u64 seed, thr;          // sample seed and threshold (war_pick)
    u64 pos_lo, pos_hi;     // canon: only positions order*(n-1)+split in [pos_lo, pos_hi) are played
    int n, per, half, hbins, dbins, blk, distinct, sample;
};

// A work unit of the persistent kernel: the orders r .. r + j! - 1 (lexicographic ranks of the
// M permuted cards; r is a multiple of j!), i.e. a fixed prefix and every order of the last j
// positions; canon units also restrict the split to k0 <= k < k1.
struct Unit {
    u64 r;
    u32 j, k0, k1, pad;
};

struct BatchArgs {
    u64 fact[17];
    u64 main_base;     // main units: orders [(main_base + u) * m!, + m!), u < main_count
    u64 main_count;
    u64 n_units;       // main_count + extra units
    const Unit* units; // extra units, handed out after the main ones
    u64 seed, thr;
    TurnK tk;          // constants of war_turn_fma
    int n, m, hbins, dbins, blk, W, half, sample, distinct, defer;
    u64* memo;         // cycle memo table (2^memo_bits words, 0 = empty), or null
    u32 memo_bits;
    u32 chunk;         // work units a lane takes from the counter at a time (0 or 1: one)
};

struct CycleWalk { u32 c1, c2; bool sym, on, is_min; };

// Key of cpu/distinct_cycles.c:84-92 for sentinel piles: player 1's length, then player 1's cards top
// first, then player 2's.  n <= 16 cards fit the 64-bit sequence; the length is compared first.
struct CKey { u32 len1; u64 seq; };
__device__ __forceinline__ CKey ckey(u64 a, u64 b, u32 la, u32 lb) {
    CKey k; k.len1 = la; k.seq = 0;
    for (u32 i = 0; i < la; i++) { k.seq = (k.seq << 4) | (a & 15ull); a >>= 4; }
    for (u32 i = 0; i < lb; i++) { k.seq = (k.seq << 4) | (b & 15ull); b >>= 4; }
    return k;
}
__device__ __forceinline__ bool ckey_lt(CKey x, CKey y) { return x.len1 < y.len1 || (x.len1 == y.len1 && x.seq < y.seq); }

// Walks lam turns from the start position (gpu/war_gpu.py:224-234): counts the states whose player-1
// top card is n-1 (c1) and whose player-2 top is n-1 (c2), notes whether the player-swapped start is
// passed (sym), whether the walk returns to the start (on: the start lies on its cycle), and whether
// the start is the minimum-key canonical state of its cycle, swapped states included
// (cpu/distinct_cycles.c:131-137).
template <int RULE>
__device__ __noinline__ CycleWalk cycle_walk(u64 w1s, u64 w2s, u32 qs, u32 n, u32 lam) {
    CycleWalk r; r.c1 = 0; r.c2 = 0; r.sym = false;
    const u32 k4m4 = 4u * (n - 1u);
    u64 v1 = w1s, v2 = w2s; u32 q = qs;
    CKey kmin; kmin.len1 = 0xFFFFFFFFu; kmin.seq = ~0ull;
    for (u32 t = 0; t < lam; t++) {
        u32 l1 = q >> 2, l2 = n - l1;
        if ((v1 & 15ull) == (u64)(n - 1u)) {
            r.c1++;
            CKey k = ckey(v1, v2, l1, l2);
            if (ckey_lt(k, kmin)) kmin = k;
        }
        if ((v2 & 15ull) == (u64)(n - 1u)) {
            r.c2++;
            CKey k = ckey(v2, v1, l2, l1);
            if (ckey_lt(k, kmin)) kmin = k;
        }
        if (v1 == w2s && v2 == w1s) r.sym = true;
        war_turn<RULE>(v1, v2, q, k4m4);
    }
    r.on = (v1 == w1s && v2 == w2s);
    CKey ks = ckey(w1s, w2s, qs >> 2, n - (qs >> 2));
    r.is_min = r.on && ks.len1 == kmin.len1 && ks.seq == kmin.seq;
    return r;
}

// Returns true if lam turns from the start come back to it (the start lies on its cycle).
template <int RULE>
__device__ __noinline__ bool on_cycle_walk(u64 w1s, u64 w2s, u32 qs, u32 n, u32 lam) {
    const u32 k4m4 = 4u * (n - 1u);
    u64 v1 = w1s, v2 = w2s; u32 q = qs;
    for (u32 t = 0; t < lam; t++) war_turn<RULE>(v1, v2, q, k4m4);
    return v1 == w1s && v2 == w2s;
}

// The Theorem-3 shape test of gpu/war_gpu.py:51-73 without a bit buffer: walks lam turns from a
// state on the loop and checks every cyclic run of wins by one player has length blk.
// 0 = that shape, 1 = not, 2 = loop longer than 512 turns (not checked, as in the reference).
template <int RULE>
__device__ __noinline__ int loop_shape_walk(u64 w1, u64 w2, u32 q, u32 k4m4, u32 lam, u32 blk) {
    if (lam > 512u) return 2;
    bool first = war_turn<RULE>(w1, w2, q, k4m4);
    bool prev = first, started = false, ok = true;
    u32 run = 1, first_run = 0;
    for (u32 i = 1; i < lam; i++) {
        bool b = war_turn<RULE>(w1, w2, q, k4m4);
        if (b == prev) { run++; continue; }
        if (!started) { first_run = run; started = true; }
        else ok = ok && (run == blk);
        run = 1;
        prev = b;
    }
    if (!started) return 1;
    if (prev == first) ok = ok && (run + first_run == blk);
    else ok = ok && (run == blk) && (first_run == blk);
    return ok ? 0 : 1;
}

// Counts kernels launched by this library (war_launch_count).
void note_launch();

cudaError_t launch_plain(const PlainArgs& a, int canon, int rule, int threads, u64 nthreads, DevAcc* acc,
                         cudaStream_t st);

struct BatchShape { int threads, blocks, games, variant; };
cudaError_t launch_batched(const BatchArgs& a, int canon, int rule, int shape, const BatchShape& bs, DevAcc* acc,
                           cudaStream_t st);
int batched_max_blocks_per_sm(int canon, int rule, int shape, int distinct, int sample, int threads, int games,
                              int hbins, int variant);

// Held-out-card engine (war_held.cu): deals of n <= 17 cards.
struct HeldArgs {
    u64 fact[18];
    u64 main_base, main_count, n_units;   // as in BatchArgs
    const Unit* units;
    int n, m, rule, hbins, W, defer;
    u64* memo;        // path memo (2^memo_bits words, 0 = empty), or null
    u32 memo_bits;
    int form;         // the turn: 0 h_turn, 1 h_turn_fma (multiply-add), 2 h_turn_packed (counts in one word),
                      // 3 h_turn_packed_fma
    int svc_off;      // test the tortoise checkpoint after every turn even where it could be saved at the services
    TurnK tk;         // its constants
};
cudaError_t launch_held(const HeldArgs& a, int threads, int blocks, DevAcc* acc, cudaStream_t st);
int held_max_blocks_per_sm(int rule, int threads, int hbins, bool memo, int form, bool svc);
bool held_svc(const HeldArgs& a);

struct FloydArgs {
    u64 fact[17];
    u64 start, total;       // rank range (deals: deal ranks; canon: position ranks)
    u64 seed, thr;
    int n, canon, rule, half, per;
};

}  // namespace war
