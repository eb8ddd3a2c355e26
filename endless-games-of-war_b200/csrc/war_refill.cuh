// war_refill.cuh — the refill loop shared by the persistent kernel (war_batched.cu) and the serving
// kernel (war_server.cu).
//
// The reference gives every thread 256 consecutive deals and plays them one after another, so a warp
// runs each deal slot as long as its longest game (gpu/war_gpu.py:149-165).  Here every lane keeps
// G games in flight and steps all of them every iteration; a lane whose game is decided records it and
// loads its next position at once, so uneven game lengths do not idle the warp.  The grid is
// persistent (SMs x resident blocks) and lanes pull work units from one global atomic counter.
//
// Enumeration inside a unit: a unit is the block of j! consecutive lexicographic ranks that share a
// prefix, i.e. every order of the last j positions.  The counts are sums and maxima over that SET, so
// the lane walks it in Heap's order (one transposition per step, the counter packed in nibbles)
// instead of lexicographic order; the set is the same.  Deals are held in a split layout: deck
// position p lives in slot (p>>1) + 8*(p&1), so player 1's cards are the low 32 bits and player 2's
// the high 32 bits and dealing is two ORs (war_cycles, gpu/war_gpu.py:98-107).
//
// Cycle detection is Brent (gpu/war_gpu.py:77-96) with the tortoise saved at steps W, 3W, 7W, ...;
// W = 1 is the reference's schedule.  With W >= lam the first window compares every state with the
// starting position itself, so a canonical start that lies on its cycle is recognised at no cost,
// and the distinct-cycle walk of gpu/war_gpu.py:224-234 runs only for those few positions.
#pragma once
#include "war_kernels.cuh"

namespace war {


struct Enum {
    u64 P;       // current order: split layout (deals) or packed q (canon)
    u32 ctr;     // Heap counter, digit i in nibble i
    u32 full;    // counter value of the unit's last order
    u32 base;    // first permuted position, M - j
    u32 k, k0, k1;
    bool live;   // P (and k) name the next unplayed position
};

// With a.chunk > 1 a lane takes that many consecutive units from the counter at a time.  Its cursor (the next
// unit of its chunk) lives in shared memory, one word per thread after the two histograms, so that the usual
// one-unit path keeps no register for it.  Chunks start at multiples of a.chunk, so the cursor needs a new
// chunk exactly when it is a multiple of a.chunk.
__device__ __forceinline__ u64* chunk_cursor(const BatchArgs& a) {
    extern __shared__ u32 war_dyn_sh[];
    const u32 off = ((u32)a.hbins + (u32)WAR_EBINS + 1u) & ~1u;   // 8-byte aligned
    return (u64*)(war_dyn_sh + off) + threadIdx.x;
}

template <bool CANON>
__device__ __forceinline__ u32 pos_shift(u32 p) {
    return CANON ? 4u * p : 4u * ((p >> 1) + ((p & 1u) << 3));
}

__device__ __forceinline__ u32 heap_full(u32 j) {
    u32 f = 0;
    for (u32 i = 1; i < j; i++) f |= i << (4u * i);
    return f;
}

template <bool CANON>
__device__ __forceinline__ bool fetch_unit(Enum& E, const BatchArgs& a, u64* counter) {
    u64 u;
    if (a.chunk <= 1u) {
        u = atomicAdd(counter, 1ull);
    } else {
        u64* cur = chunk_cursor(a);
        if (*cur % a.chunk == 0ull) *cur = atomicAdd(counter, (u64)a.chunk);   // the next chunk
        u = (*cur)++;
    }
    if (u >= a.n_units) return false;   // (the counter only grows: later units lie beyond the list too)
    u64 r;
    u32 j, k0, k1;
    if (u < a.main_count) {
        j = (u32)a.m; r = (a.main_base + u) * a.fact[a.m]; k0 = 0; k1 = (u32)a.n - 1u;
    } else {
        const Unit U = a.units[u - a.main_count];
        r = U.r; j = U.j; k0 = U.k0; k1 = U.k1;
    }
    const int M = CANON ? a.n - 1 : a.n;
    u64 p = unrank_packed(r, M, a.fact);
    if (!CANON) p = compact_even_nibbles(p) | (compact_even_nibbles(p >> 4) << 32);
    E.P = p;
    E.ctr = 0;
    E.full = heap_full(j);
    E.base = (u32)M - j;
    E.k0 = k0; E.k1 = k1; E.k = k0;
    E.live = true;
    return true;
}

// Heap's algorithm, one output: the lowest digit i with ctr[i] < i increments, the digits below it
// reset to 0, and position i swaps with position 0 (i even) or ctr[i] (i odd).  False after the last.
template <bool CANON>
__device__ __forceinline__ bool heap_step(Enum& E) {
    u32 x = E.ctr ^ E.full;
    if (x == 0u) return false;
    u32 i = (u32)(__ffs((int)x) - 1) >> 2;
    u32 ci = (E.ctr >> (4u * i)) & 15u;
    u32 o = (i & 1u) ? ci : 0u;
    E.P = swap_nibbles(E.P, pos_shift<CANON>(E.base + i), pos_shift<CANON>(E.base + o));
    E.ctr = ((E.ctr >> (4u * i)) + 1u) << (4u * i);
    return true;
}

struct DealConst { u64 s1, s2; u32 q0, pat32; };

// Next deal of the lane (deals mode); false when the lane has no work left.
__device__ __forceinline__ bool next_deal(Enum& E, const BatchArgs& a, u64* counter, const DealConst& c, u64& w1,
                                          u64& w2, u32& q) {
    for (;;) {
        if (!E.live && !fetch_unit<false>(E, a, counter)) return false;
        u64 D = E.P;
        E.live = heap_step<false>(E);
        if (a.half) {   // gpu/war_gpu.py:151-154: card n-1 dealt to player 1
            u32 x = (u32)D ^ c.pat32;
            if (((x - 0x11111111u) & ~x & 0x88888888u) == 0u) continue;
        }
        w1 = (D & 0xFFFFFFFFull) | c.s1;
        w2 = (D >> 32) | c.s2;
        q = c.q0;
        return true;
    }
}

// Next canonical position of the lane.
__device__ __forceinline__ bool next_canon(Enum& E, const BatchArgs& a, u64* counter, u64& w1, u64& w2, u32& q) {
    if (!E.live && !fetch_unit<true>(E, a, counter)) return false;
    canon_position(E.P, (u32)a.n, E.k, w1, w2, q);
    if (++E.k == E.k1) {
        E.k = E.k0;
        E.live = heap_step<true>(E);
    }
    return true;
}

// One game slot.  EXTRA keeps the start position and the sample bit (distinct walk, sample);
// SHAPE keeps the run tracker of the current tortoise window.
enum { ST_ACTIVE = 0, ST_WAITING = 1, ST_RETIRED = 2 };

template <bool EXTRA, bool SHAPE>
struct Game {
    u64 w1, w2, t1, t2;
    u32 q, rounds, next, st;
    // EXTRA
    u64 s1, s2; u32 sq; bool sampled;
    // SHAPE: run tracker since the last tortoise save
    u32 cur, first_run; bool first, prev, started, ok;
};

// The refill loop of one block: lanes take work units from *counter (shared by every block that works on
// the same unit list), play them and add the block's results to *acc.  sh: hbins + WAR_EBINS u32 words of
// shared memory.  Used by the persistent kernel (one job, all blocks) and by the serving kernel (one task
// of one job per block).
template <int RULE, int G, bool CANON, bool SHAPE, bool EXTRA, int TV>
__device__ __forceinline__ void refill_body(const BatchArgs& a, DevAcc* __restrict__ acc, u64* __restrict__ counter,
                                            u32* sh) {
    u32* shh = sh;
    u32* she = sh + a.hbins;
    for (int b = threadIdx.x; b < a.hbins + WAR_EBINS; b += blockDim.x) sh[b] = 0;
    __syncthreads();

    const u32 n = (u32)a.n, n4 = 4u * n, k4m4 = 4u * (n - 1u), W = (u32)a.W;
    const TurnK K = a.tk;
    // TV = 0: war_turn (q = 4*len1); TV = 1: war_turn_fma (q holds qq = 4*len1 - 2n)
    const u32 qshift = TV ? 2u * n : 0u;
    const u32 hb1 = a.hbins > 0 ? (u32)(a.hbins - 1) : 0u;
    DealConst dc;
    dc.s1 = sentinel_bit((n + 1u) / 2u);
    dc.s2 = sentinel_bit(n / 2u);
    dc.q0 = 4u * ((n + 1u) / 2u);
    dc.pat32 = 0x11111111u * (n - 1u);

    Enum E;
    E.live = false;
    if (a.chunk > 1u) *chunk_cursor(a) = 0ull;
    Game<EXTRA, SHAPE> g[G];
    // Per-lane totals.  A launch plays fewer than 2^32 games in all, so no lane's 32-bit turn total wraps.
    u32 cyc = 0, done = 0, maxfin = 0, capped = 0, turns = 0;
    u32 sc = 0, scy = 0, slam = 0, slen = 0, smax = 0, oncyc = 0, dmin = 0, nonstd = 0, unchk = 0;

    // Game slot states: ACTIVE (being played), WAITING (decided and recorded, frozen until the warp
    // refills), RETIRED (no work left).  A frozen slot holds two empty words and q far out of range, so
    // the turn step leaves it unchanged (the pushed pair shifts out, shl64 gives 0).
    // A frozen slot can never signal: its low words differ from its tortoise's, its next checkpoint is
    // never reached, and its length offset is odd and far from both ends.  Every turn moves the offset by
    // 4, so it stays odd: never 0 or 4n, and its square (multiply-add form) is odd, never (2n)^2.  With
    // both words empty the pushed pair lands beyond bit 63 and the words stay 0.
    auto freeze = [&](Game<EXTRA, SHAPE>& x) {
        x.w1 = 0ull; x.w2 = 0ull; x.q = 0x80000001u; x.t1 = 1ull; x.t2 = 1ull; x.next = 0xFFFFFFFFu;
    };
    auto start_game = [&](Game<EXTRA, SHAPE>& x) {
        bool ok = CANON ? next_canon(E, a, counter, x.w1, x.w2, x.q) : next_deal(E, a, counter, dc, x.w1, x.w2, x.q);
        x.st = ok ? ST_ACTIVE : ST_RETIRED;
        done += ok ? 1u : 0u;
        x.t1 = x.w1; x.t2 = x.w2; x.rounds = 0; x.next = W;
        if (EXTRA) {
            x.s1 = x.w1; x.s2 = x.w2; x.sq = x.q;
            x.sampled = a.sample && ok && war_pick(a.seed, a.thr, x.w1, x.w2);
        }
        if (SHAPE) x.cur = 0;
        x.q -= qshift;
        if (!ok) freeze(x);
    };

#pragma unroll
    for (int i = 0; i < G; i++) start_game(g[i]);

    // The warp leaves the loop once none of its lanes holds an active or waiting game.  That test runs
    // whenever a slot changes state (a game decided or abandoned at the cap), and once here for warps that
    // got no work at all.  Decided games wait, frozen, until `defer` lanes of the warp are waiting (or
    // none is playing); then all of them load their next position together, so the refill code runs
    // with many lanes at once instead of one.
    const int defer = a.defer > 0 ? a.defer : 1;
    bool alive0 = false;
#pragma unroll
    for (int i = 0; i < G; i++) alive0 |= g[i].st == ST_ACTIVE;
    bool running = __any_sync(WAR_FULL_MASK, alive0);

    while (running) {
        bool fin[G];
        bool anyfin = false;
#pragma unroll
        for (int i = 0; i < G; i++) {
            Game<EXTRA, SHAPE>& x = g[i];
            bool p1, en;
            if (TV == 1) {
                p1 = war_turn_fma<RULE>(x.w1, x.w2, x.q, K);
                x.rounds = x.rounds * K.one + K.one;
                en = x.q * x.q == K.end2;
            } else {
                p1 = war_turn<RULE>(x.w1, x.w2, x.q, k4m4);
                x.rounds++;
                en = (x.q == 0u) | (x.q == n4);
            }
            // Cycle candidate: the low words of both piles equal the tortoise's.  Exact equality of the
            // high words is checked when the game is recorded; a candidate that fails it plays on.
            bool cy = ((u32)x.w1 == (u32)x.t1) & ((u32)x.w2 == (u32)x.t2);
            if (SHAPE) {
                if (x.cur == 0u) { x.first = p1; x.prev = p1; x.cur = 1u; x.first_run = 0u; x.started = false; x.ok = true; }
                else if (p1 == x.prev) x.cur++;
                else {
                    if (!x.started) { x.first_run = x.cur; x.started = true; }
                    else x.ok = x.ok && (x.cur == (u32)a.blk);
                    x.cur = 1u; x.prev = p1;
                }
            }
            if (x.rounds == x.next && !(cy | en)) {   // a decided game keeps its tortoise (the record reads it)
                if (x.next > WAR_TURN_CAP) {
                    if (x.st == ST_ACTIVE) { capped++; x.st = ST_WAITING; freeze(x); anyfin = true; }
                } else {
                    x.t1 = x.w1; x.t2 = x.w2; x.next = 2u * x.next + W;
                    if (SHAPE) x.cur = 0u;
                }
            }
            fin[i] = cy | en;
            anyfin |= fin[i];
        }
        if (__any_sync(WAR_FULL_MASK, anyfin)) {
#pragma unroll
            for (int i = 0; i < G; i++) {
                Game<EXTRA, SHAPE>& x = g[i];
                bool rec = fin[i];
                if (rec) {
                    const bool en = TV ? (x.q * x.q == K.end2) : ((x.q == 0u) | (x.q == n4));
                    if (!en && !((x.w1 == x.t1) & (x.w2 == x.t2))) {
                        // low words matched by chance: play on, with the tortoise save this step skipped
                        rec = false;
                        if (x.rounds == x.next) {
                            x.t1 = x.w1; x.t2 = x.w2; x.next = 2u * x.next + W;
                            if (SHAPE) x.cur = 0u;
                        }
                    }
                }
                if (rec) {
                    const bool cy = (x.w1 == x.t1) & (x.w2 == x.t2);
                    turns += x.rounds;
                    const u32 lam = x.rounds - ((x.next - W) >> 1);
                    if (cy) {
                        cyc++;
                        if (a.hbins) atomicAdd(&shh[lam < hb1 ? lam : hb1], 1u);
                        if (CANON && EXTRA && a.distinct) {
                            const u32 tstep = (x.next - W) >> 1;
                            bool on = (tstep == 0u) ? true
                                    : (lam <= W ? false : on_cycle_walk<RULE>(x.s1, x.s2, x.sq, n, lam));
                            if (on) {
                                CycleWalk cw = cycle_walk<RULE>(x.s1, x.s2, x.sq, n, lam);
                                oncyc++;
                                if (cw.is_min) dmin++;
                                if (a.dbins) {
                                    u32 d = cw.sym ? cw.c1 : cw.c1 + cw.c2;
                                    u32 db1 = (u32)(a.dbins - 1);
                                    atomicAdd(&acc->dhist[d < db1 ? d : db1], 1ull);
                                }
                            }
                        }
                        if (SHAPE) {
                            if (lam > 512u) unchk++;
                            else {
                                bool ok = x.started && x.ok;
                                if (x.started) {
                                    if (x.prev == x.first) ok = ok && (x.cur + x.first_run == (u32)a.blk);
                                    else ok = ok && (x.cur == (u32)a.blk) && (x.first_run == (u32)a.blk);
                                }
                                if (!ok) nonstd++;
                            }
                        }
                    } else {
                        if (x.rounds > maxfin) maxfin = x.rounds;
                        atomicAdd(&she[x.rounds < WAR_EBINS - 1 ? x.rounds : WAR_EBINS - 1], 1u);
                    }
                    if (EXTRA && x.sampled) {
                        sc++;
                        if (cy) { scy++; slam += lam; }
                        else { slen += x.rounds; if (x.rounds > smax) smax = x.rounds; }
                    }
                    x.st = ST_WAITING;
                    freeze(x);
                }
            }
            bool waiting = false, playing = false;
#pragma unroll
            for (int i = 0; i < G; i++) { waiting |= g[i].st == ST_WAITING; playing |= g[i].st == ST_ACTIVE; }
            const u32 wb = __ballot_sync(WAR_FULL_MASK, waiting);
            const u32 pb = __ballot_sync(WAR_FULL_MASK, playing);
            if (__popc(wb) >= defer || pb == 0u) {
                if (waiting) {
#pragma unroll
                    for (int i = 0; i < G; i++)
                        if (g[i].st == ST_WAITING) start_game(g[i]);
                }
                playing = false;
#pragma unroll
                for (int i = 0; i < G; i++) playing |= g[i].st == ST_ACTIVE;
                running = __any_sync(WAR_FULL_MASK, playing);
            }
        }
    }

    u64 v_cyc = warp_sum(cyc), v_done = warp_sum(done), v_turns = warp_sum((u64)turns), v_max = warp_max(maxfin);
    u64 v_cap = warp_sum(capped);
    if ((threadIdx.x & 31) == 0) {
        if (v_cyc) atomicAdd(&acc->cyc, v_cyc);
        if (v_done) atomicAdd(&acc->done, v_done);
        if (v_turns) atomicAdd(&acc->turns, v_turns);
        if (v_max) atomicMax(&acc->maxfin, v_max);
        if (v_cap) atomicAdd(&acc->status, v_cap);
    }
    if (EXTRA) {
        u64 v_sc = warp_sum(sc), v_scy = warp_sum(scy), v_slam = warp_sum(slam), v_slen = warp_sum(slen);
        u64 v_smax = warp_max(smax), v_on = warp_sum(oncyc), v_dmin = warp_sum(dmin);
        if ((threadIdx.x & 31) == 0) {
            if (v_sc) {
                atomicAdd(&acc->s_count, v_sc); atomicAdd(&acc->s_cyc, v_scy); atomicAdd(&acc->s_lamsum, v_slam);
                atomicAdd(&acc->s_lensum, v_slen); atomicMax(&acc->s_maxfin, v_smax);
            }
            if (v_on) atomicAdd(&acc->oncycle, v_on);
            if (v_dmin) atomicAdd(&acc->distinct_min, v_dmin);
        }
    }
    if (SHAPE) {
        u64 v_ns = warp_sum(nonstd), v_un = warp_sum(unchk);
        if ((threadIdx.x & 31) == 0) {
            if (v_ns) atomicAdd(&acc->shape_nonstd, v_ns);
            if (v_un) atomicAdd(&acc->shape_unchecked, v_un);
        }
    }
    __syncthreads();
    flush_hist(shh, acc->hist, a.hbins);
    flush_hist(she, acc->endhist, WAR_EBINS);
}

// ---- cycle memo ---------------------------------------------------------------------------------------
// Every cycle of a game contains "landmark" states, where card n-1 is on top of its holder's pile (card
// n-1 never loses, and each pile is a queue, so every card reaches the top within one cycle).  The memo
// holds the landmarks of the cycles found so far in the job.  A game that passes a landmark in the memo
// is on that cycle: it never ends and its cycle length is the memo's, so it is decided then instead of
// when Brent's test fires.  Brent keeps running for every game, so a cycle missing from the memo (not
// found yet, or a full table) is still found exactly: the memo only decides games earlier.  War is the
// same game with the players swapped (the winner's card, then the loser's, goes under the winner's
// pile), so a landmark is stored once, with the holder of card n-1 as the first player.
//
// Entry (one 64-bit word): the holder's pile without its top card (which is n-1) followed by the other
// pile, as 4(n-2) bits of nibbles (the last card is the one missing), then the holder's pile length in
// 4 bits, then the cycle length in the remaining 64 - 4(n-1) bits.  The length field is at least 1, so
// no entry is 0, which marks an empty slot.  n <= 15, cycle lengths below 2^(64 - 4(n-1)).
//
// The table is direct-mapped and written with a fire-and-forget atomic maximum: a slot wanted by two
// landmarks keeps one whole entry of the two (the other is lost, which only means a later detection).
// Inserts therefore never wait for memory and lookups are one load, with no probe chain.
__device__ __forceinline__ u32 pile_len(u64 w) { return (63u - (u32)__clzll(w | 1ull)) >> 2; }

// The key of the landmark where pile h (top card n-1) is the holder's and pile o the other's.
__device__ __forceinline__ u64 memo_key(u64 h, u64 o, u32 n) {
    const u32 lh = pile_len(h);
    const u64 cat = (h ^ (1ull << (4u * lh))) | (o << (4u * lh));   // holder's cards, then the other's
    const u32 kb = 4u * (n - 2u);
    return ((cat >> 4) & ((1ull << kb) - 1ull)) | ((u64)lh << kb);
}

__device__ __forceinline__ u32 memo_slot(u64 key, u32 bits) {
    return (u32)((key * 0x9E3779B97F4A7C15ull) >> (64u - bits));   // the multiplier of path_entry
}

// The atomic is skipped when the slot already holds this entry or a larger one (it would change
// nothing), which keeps the games that find the same new cycle at once from queueing on its slots.
__device__ __forceinline__ void memo_put(u64* T, u32 bits, u64 key, u32 lsh, u32 lam) {
    unsigned long long* p = (unsigned long long*)T + memo_slot(key, bits);
    const unsigned long long val = key | ((u64)lam << lsh);
    if (__ldcg(p) < val) atomicMax(p, val);
}

// The all-states memo (MEMO_ALL) holds every state of a found cycle instead of its landmarks, so a game
// is looked up at its current state and needs nothing kept per turn.  Entry: the pile that is smaller as
// a 64-bit word first (either orientation gives the same key), its cards then the other pile's as 4(n-1)
// bits of nibbles (the last card is the one missing), its length in 4 bits, the cycle length in the top
// 64 - 4n bits.  n <= 14.  (The path memo's entries, below, keep the key implicitly and serve n <= 16.)
//
// The path memo (MEMO_PATH) adds, for every decided game, the states at which it was looked up and
// missed (the last two), with the game's outcome from there: "on a cycle of length lam" (value 2 lam) or
// "ends after r more turns" (value 2r + 1).  Deals of nearby ranks often merge into one another's paths
// after a few turns, so a later game is decided where it meets such a state.  All entries of these two
// memos are plain fire-and-forget stores that overwrite the slot (the most recent paths are the useful
// ones; an aligned 8-byte store never tears, and a lost entry only means a later decision).
//
// A path-memo entry does not hold its key.  H = key * C is a bijection of 64-bit words (C odd); the slot
// is the top `bits` bits of H and the entry holds the other 64 - bits bits of H above a value of `bits`
// bits, (H << bits) | value.  Slot and entry together give back H, hence the key, so an entry that
// matches names exactly the state looked up.  The key is the 4(n-1)-bit concatenation plus a 4-bit length
// (memo_key_state), which fits 64 bits up to n = 16, and the value field is wide (bits >= 12).
enum { MEMO_NONE = 0, MEMO_LANDMARK = 1, MEMO_ALL = 2, MEMO_PATH = 3 };

constexpr u64 MEMO_MUL = 0x9E3779B97F4A7C15ull;   // odd (memo_slot's multiplier): a bijection mod 2^64

__device__ __forceinline__ u64 path_entry(u64 key, u32 bits, u64 v) { return ((key * MEMO_MUL) << bits) | v; }

__device__ __forceinline__ u64 memo_key_state(u64 w1, u64 w2, u32 n) {
    const bool sw = w2 < w1;
    const u64 h = sw ? w2 : w1, o = sw ? w1 : w2;
    const u32 lh = pile_len(h);
    const u64 cat = (h ^ (1ull << (4u * lh))) | (o << (4u * lh));
    const u32 kb = 4u * (n - 1u);
    return (cat & ((1ull << kb) - 1ull)) | ((u64)lh << kb);
}

template <int MODE>
__device__ __forceinline__ u32 memo_lam_shift(u32 n) { return MODE >= MEMO_ALL ? 4u * n : 4u * (n - 1u); }

// Walks the cycle of length lam through the state (w1, w2, q4 = 4*len1) once and stores its landmarks
// (MEMO_LANDMARK) or all its states (MEMO_ALL, MEMO_PATH).
template <int RULE, int MODE>
__device__ __noinline__ void memo_store_cycle(u64* T, u32 bits, u64 w1, u64 w2, u32 q4, u32 n, u32 lam,
                                              u32 pv = 0u) {
    const u32 lsh = memo_lam_shift<MODE>(n);
    const u32 v = MODE == MEMO_PATH ? (pv ? pv : 2u * lam) : lam;   // pv: the path value, if not 2 lam
    if (lam == 0u || (u64)v >> (MODE == MEMO_PATH ? bits : 64u - lsh) != 0ull) return;
    const u32 k4m4 = 4u * (n - 1u);
    const u64 top = (u64)(n - 1u);
    for (u32 t = 0; t < lam; t++) {
        if (MODE == MEMO_PATH) {
            const u64 k = memo_key_state(w1, w2, n);
            __stcg((unsigned long long*)T + memo_slot(k, bits), (unsigned long long)path_entry(k, bits, v));
        } else if (MODE == MEMO_ALL) memo_put(T, bits, memo_key_state(w1, w2, n), lsh, lam);
        else if ((w1 & 15ull) == top) memo_put(T, bits, memo_key(w1, w2, n), lsh, lam);
        else if ((w2 & 15ull) == top) memo_put(T, bits, memo_key(w2, w1, n), lsh, lam);
        war_turn<RULE>(w1, w2, q4, k4m4);
    }
}

// The same refill loop with the outcome of each game latched instead of recorded at once.  Every
// iteration steps all G games of every lane without a branch or a warp vote; a game whose cycle or end
// is found sets its `done` flag, which freezes its turn count and its tortoise (the game itself keeps
// being stepped, harmlessly).  Every K = a.defer iterations (a multiple of 4) the warp services its
// slots: each done game is recorded and replaced by the lane's next position.  The record and refill
// code therefore runs once per K iterations with every lane that has a done game, instead of once per
// decided game with one lane.  The cycle test compares all four words (no candidate to verify later).
template <bool EXTRA, int MEMO>
struct LGame {
    u64 w1, w2, t1, t2;
    u32 q, rounds, next, st;
    bool done, kcy;     // decided; decided by a cycle (else by an end)
    u64 s1, s2; u32 sq; bool sampled;
    u64 m1, m2;         // MEMO_LANDMARK: the last landmark passed since the last lookup (m1 = 0: none)
    u32 mlam;           // MEMO: the memo's value for this game (0: decided by Brent or by its end)
    u64 ka, kb;         // MEMO_PATH: the keys of the last two states looked up and missed,
    u32 ta, tb;         // at these turns (0: none)
    u32 pend;           // canonical distinct scan: a memo value held until turn lam of its cycle (0: none)
};

// With MEMO_LANDMARK, each turn also keeps the state before it when card n-1 is on top (a landmark), and
// every service looks the kept landmark of each undecided game up in the memo; with MEMO_ALL every
// service looks up each undecided game's current state.  A game decided by Brent stores its cycle.
//
// SHAPE (canonical scans with the loop-shape test, path memo only): the Theorem-3 shape is a property of
// the cycle, so it travels in the memo with the cycle length — a cycle outcome is 8 lam + 2 code (code 0
// of the shape, 1 not, 2 loop too long to check) instead of 2 lam — and a cycle found by Brent is checked
// once with loop_shape_walk from its detection state, which lies on the loop.
template <int RULE, int G, bool CANON, bool EXTRA, int TV, int MEMO, bool SHAPE = false>
__device__ __forceinline__ void refill_latched(const BatchArgs& a, DevAcc* __restrict__ acc, u64* __restrict__ counter,
                                               u32* sh) {
    u32* shh = sh;
    u32* she = sh + a.hbins;
    for (int b = threadIdx.x; b < a.hbins + WAR_EBINS; b += blockDim.x) sh[b] = 0;
    __syncthreads();

    const u32 n = (u32)a.n, n4 = 4u * n, k4m4 = 4u * (n - 1u), W = (u32)a.W;
    const TurnK K = a.tk;
    const u32 qshift = TV ? 2u * n : 0u;
    const u32 hb1 = a.hbins > 0 ? (u32)(a.hbins - 1) : 0u;
    const int period = a.defer > 4 ? (a.defer + 3) & ~3 : 4;
    DealConst dc;
    dc.s1 = sentinel_bit((n + 1u) / 2u);
    dc.s2 = sentinel_bit(n / 2u);
    dc.q0 = 4u * ((n + 1u) / 2u);
    dc.pat32 = 0x11111111u * (n - 1u);

    Enum E;
    E.live = false;
    if (a.chunk > 1u) *chunk_cursor(a) = 0ull;
    LGame<EXTRA, MEMO> g[G];
    u32 cyc = 0, done = 0, maxfin = 0, capped = 0, turns = 0;
    u32 sc = 0, scy = 0, slam = 0, slen = 0, smax = 0, oncyc = 0, dmin = 0;
    u32 nonstd = 0, unchk = 0;             // SHAPE
    u32 mlook = 0, mhit = 0, mstore = 0;   // memo traffic
    const u32 nm1 = n - 1u;
    u64* const memo = MEMO ? a.memo : nullptr;
    const u32 mbits = a.memo_bits, lsh = memo_lam_shift<MEMO>(n);
    const u64 kmask = lsh < 64u ? (1ull << lsh) - 1ull : ~0ull;
    const u64 vmask = (1ull << mbits) - 1ull;   // value field of a path entry

    auto start_game = [&](LGame<EXTRA, MEMO>& x) {
        bool ok = CANON ? next_canon(E, a, counter, x.w1, x.w2, x.q) : next_deal(E, a, counter, dc, x.w1, x.w2, x.q);
        x.st = ok ? ST_ACTIVE : ST_RETIRED;
        done += ok ? 1u : 0u;
        x.t1 = x.w1; x.t2 = x.w2; x.rounds = 0; x.next = W;
        x.done = !ok; x.kcy = false;
        if (MEMO) { x.m1 = 0ull; x.m2 = 0ull; x.mlam = 0u; }
        if (MEMO == MEMO_PATH) { x.ta = 0u; x.tb = 0u; }
        if (MEMO) x.pend = 0u;
        if (EXTRA) {
            x.s1 = x.w1; x.s2 = x.w2; x.sq = x.q;
            x.sampled = a.sample && ok && war_pick(a.seed, a.thr, x.w1, x.w2);
        }
        x.q -= qshift;
    };

#pragma unroll
    for (int i = 0; i < G; i++) start_game(g[i]);
    bool alive0 = false;
#pragma unroll
    for (int i = 0; i < G; i++) alive0 |= g[i].st == ST_ACTIVE;
    bool running = __any_sync(WAR_FULL_MASK, alive0);

    while (running) {
        for (int k = 0; k < period; k += 4) {
#pragma unroll
            for (int u = 0; u < 4; u++) {
#pragma unroll
                for (int i = 0; i < G; i++) {
                    LGame<EXTRA, MEMO>& x = g[i];
                    if (MEMO == MEMO_LANDMARK) {
                        const u32 c1 = (u32)x.w1 & 15u, c2 = (u32)x.w2 & 15u;
                        const bool lm = max(c1, c2) == nm1;
                        x.m1 = lm ? x.w1 : x.m1;
                        x.m2 = lm ? x.w2 : x.m2;
                    }
                    bool en;
                    if (TV == 1) {
                        war_turn_fma<RULE>(x.w1, x.w2, x.q, K);
                        en = x.q * x.q == K.end2;
                    } else {
                        war_turn<RULE>(x.w1, x.w2, x.q, k4m4);
                        en = (x.q == 0u) | (x.q == n4);
                    }
                    if (!x.done) x.rounds += K.one;
                    const bool cy = (x.w1 == x.t1) & (x.w2 == x.t2);
                    const bool fin = (cy | en) & !x.done;
                    x.kcy = fin ? cy : x.kcy;
                    x.done = x.done | fin;
                }
            }
        }
        // Brent's checkpoint, at the service: a game starts at a service and plays `period` turns between
        // services while undecided, so when W is a multiple of the period the checkpoints W, 3W, 7W, ... all
        // fall on services and this is the reference's doubling schedule (with first window W) exactly; else
        // the tortoise is saved at the first service at or after the checkpoint.  next = 2 t + W keeps the turn
        // t of the last save ((next - W) / 2 names it; the gaps still double, so every cycle is found, and
        // the first return to the saved state is exactly one cycle length after it).
#pragma unroll
        for (int i = 0; i < G; i++) {
            LGame<EXTRA, MEMO>& x = g[i];
            if (!x.done && x.rounds >= x.next) {
                if (x.next > WAR_TURN_CAP) {   // abandon (never expected): counted, slot serviced as done
                    capped++; x.done = true; x.st = ST_WAITING;
                } else {
                    x.t1 = x.w1; x.t2 = x.w2; x.next = 2u * x.rounds + W;
                }
            }
        }
        if (MEMO && memo != nullptr) {   // look up the kept landmarks: the loads of all G games first
            u64 key[G], e[G];
            bool look[G];
#pragma unroll
            for (int i = 0; i < G; i++) {
                LGame<EXTRA, MEMO>& x = g[i];
                if (MEMO >= MEMO_ALL) {
                    look[i] = !x.done & (x.pend == 0u);
                    key[i] = memo_key_state(x.w1, x.w2, n);
                } else {
                    look[i] = !x.done & (x.m1 != 0ull);
                    const bool h1 = ((u32)x.m1 & 15u) == nm1;
                    key[i] = memo_key(h1 ? x.m1 : x.m2, h1 ? x.m2 : x.m1, n);
                    x.m1 = 0ull;
                }
                e[i] = look[i] ? __ldcg((const unsigned long long*)memo + memo_slot(key[i], mbits)) : 0ull;
            }
#pragma unroll
            for (int i = 0; i < G; i++) {
                LGame<EXTRA, MEMO>& x = g[i];
                mlook += look[i] ? 1u : 0u;
                // (an empty slot reads 0: no key of the explicit-key memos, and a value of 0 in a path entry)
                const bool match = MEMO == MEMO_PATH
                    ? (e[i] & vmask) != 0ull && ((e[i] ^ path_entry(key[i], mbits, 0ull)) >> mbits) == 0ull
                    : (e[i] & kmask) == key[i];
                if (look[i] && match) {
                    mhit++;
                    const u32 v = MEMO == MEMO_PATH ? (u32)(e[i] & vmask) : (u32)(e[i] >> lsh);
                    const bool vcy = MEMO == MEMO_PATH ? (v & 1u) == 0u : true;
                    const u32 vlam = MEMO == MEMO_PATH ? v >> (SHAPE ? 3 : 1) : v;
                    if (CANON && EXTRA && a.distinct && vcy && vlam <= W && x.rounds < vlam) {
                        // Whether the start lies on its cycle shows at turn vlam: Brent's first window
                        // compares every state up to W >= vlam with the start.  Play on until then.
                        x.pend = v;
                    } else {
                        x.done = true; x.kcy = vcy; x.mlam = v;
                    }
                } else if (CANON && EXTRA && x.pend != 0u && !x.done &&
                           x.rounds >= (MEMO == MEMO_PATH ? x.pend >> (SHAPE ? 3 : 1) : x.pend)) {
                    // turn lam passed without the start coming back: on the cycle, not through the start
                    x.done = true; x.kcy = true; x.mlam = x.pend;
                } else if (MEMO == MEMO_PATH && look[i]) {
                    x.kb = x.ka; x.tb = x.ta;
                    x.ka = key[i]; x.ta = x.rounds;
                }
            }
        }
        // service: record every decided game, refill its slot
        bool any = false;
#pragma unroll
        for (int i = 0; i < G; i++) any |= g[i].done & (g[i].st != ST_RETIRED);
        if (__any_sync(WAR_FULL_MASK, any)) {
#pragma unroll
            for (int i = 0; i < G; i++) {
                LGame<EXTRA, MEMO>& x = g[i];
                if (x.done & (x.st == ST_ACTIVE)) {
                    const bool cy = x.kcy;
                    turns += x.rounds;
                    // the memo's cycle length, or (path memo) the turns left after the memoised state
                    const u32 mcy = MEMO == MEMO_PATH ? (x.mlam & 1u ? 0u : x.mlam >> (SHAPE ? 3 : 1)) : x.mlam;
                    const u32 len = MEMO == MEMO_PATH && (x.mlam & 1u) ? x.rounds + (x.mlam >> 1) : x.rounds;
                    const u32 lam = (MEMO && mcy) ? mcy : x.rounds - ((x.next - W) >> 1);
                    // SHAPE: the loop's shape code, from the memo or checked now on the loop
                    u32 code = 0u;
                    if (SHAPE && cy) {
                        code = mcy ? (x.mlam >> 1) & 3u
                                   : (u32)loop_shape_walk<RULE>(x.w1, x.w2, TV ? x.q + qshift : x.q, k4m4, lam, (u32)a.blk);
                        if (code == 1u) nonstd++;
                        if (code == 2u) unchk++;
                    }
                    const u64 vcyc = SHAPE ? 8ull * lam + 2ull * code : 2ull * lam;   // the cycle outcome
                    if (MEMO == MEMO_PATH && memo != nullptr) {   // the states it missed, with its outcome
                        if (x.ta) {
                            const u64 v = cy ? vcyc : 2ull * (len - x.ta) + 1ull;
                            const u64 k = x.ka;
                            if (v <= vmask) {
                                __stcg((unsigned long long*)memo + memo_slot(k, mbits), path_entry(k, mbits, v));
                                mstore++;
                            }
                        }
                        if (x.tb) {
                            const u64 v = cy ? vcyc : 2ull * (len - x.tb) + 1ull;
                            const u64 k = x.kb;
                            if (v <= vmask) {
                                __stcg((unsigned long long*)memo + memo_slot(k, mbits), path_entry(k, mbits, v));
                                mstore++;
                            }
                        }
                    }
                    if (cy) {
                        cyc++;
                        if (MEMO && memo != nullptr && mcy == 0u) {   // found by Brent: store its cycle
                            memo_store_cycle<RULE, MEMO>(memo, mbits, x.w1, x.w2, TV ? x.q + qshift : x.q, n, lam,
                                                         SHAPE ? (u32)vcyc : 0u);
                            mstore += lam;
                        }
                        if (a.hbins) atomicAdd(&shh[lam < hb1 ? lam : hb1], 1u);
                        if (CANON && EXTRA && a.distinct) {
                            const u32 tstep = (x.next - W) >> 1;
                            // decided by the memo: the start was not seen again within lam <= W turns
                            // (else Brent's first window would have decided it), or lam > W: walk
                            bool on = (MEMO && mcy) ? (lam <= W ? false : on_cycle_walk<RULE>(x.s1, x.s2, x.sq, n, lam))
                                    : (tstep == 0u) ? true
                                    : (lam <= W ? false : on_cycle_walk<RULE>(x.s1, x.s2, x.sq, n, lam));
                            if (on) {
                                CycleWalk cw = cycle_walk<RULE>(x.s1, x.s2, x.sq, n, lam);
                                oncyc++;
                                if (cw.is_min) dmin++;
                                if (a.dbins) {
                                    u32 d = cw.sym ? cw.c1 : cw.c1 + cw.c2;
                                    u32 db1 = (u32)(a.dbins - 1);
                                    atomicAdd(&acc->dhist[d < db1 ? d : db1], 1ull);
                                }
                            }
                        }
                    } else {
                        if (len > maxfin) maxfin = len;
                        atomicAdd(&she[len < WAR_EBINS - 1 ? len : WAR_EBINS - 1], 1u);
                    }
                    if (EXTRA && x.sampled) {
                        sc++;
                        if (cy) { scy++; slam += lam; }
                        else { slen += len; if (len > smax) smax = len; }
                    }
                }
                if (x.done & (x.st != ST_RETIRED)) start_game(x);
            }
            bool playing = false;
#pragma unroll
            for (int i = 0; i < G; i++) playing |= g[i].st == ST_ACTIVE;
            running = __any_sync(WAR_FULL_MASK, playing);
        }
    }

    if (SHAPE) {
        u64 v_ns = warp_sum((u64)nonstd), v_un = warp_sum((u64)unchk);
        if ((threadIdx.x & 31) == 0) {
            if (v_ns) atomicAdd(&acc->shape_nonstd, v_ns);
            if (v_un) atomicAdd(&acc->shape_unchecked, v_un);
        }
    }
    if (MEMO) {
        u64 v_l = warp_sum((u64)mlook), v_h = warp_sum((u64)mhit), v_s = warp_sum((u64)mstore);
        if ((threadIdx.x & 31) == 0) {
            if (v_l) atomicAdd(&acc->memo_lookups, v_l);
            if (v_h) atomicAdd(&acc->memo_hits, v_h);
            if (v_s) atomicAdd(&acc->memo_stores, v_s);
        }
    }
    u64 v_cyc = warp_sum(cyc), v_done = warp_sum(done), v_turns = warp_sum((u64)turns), v_max = warp_max(maxfin);
    u64 v_cap = warp_sum(capped);
    if ((threadIdx.x & 31) == 0) {
        if (v_cyc) atomicAdd(&acc->cyc, v_cyc);
        if (v_done) atomicAdd(&acc->done, v_done);
        if (v_turns) atomicAdd(&acc->turns, v_turns);
        if (v_max) atomicMax(&acc->maxfin, v_max);
        if (v_cap) atomicAdd(&acc->status, v_cap);
    }
    if (EXTRA) {
        u64 v_sc = warp_sum(sc), v_scy = warp_sum(scy), v_slam = warp_sum(slam), v_slen = warp_sum(slen);
        u64 v_smax = warp_max(smax), v_on = warp_sum(oncyc), v_dmin = warp_sum(dmin);
        if ((threadIdx.x & 31) == 0) {
            if (v_sc) {
                atomicAdd(&acc->s_count, v_sc); atomicAdd(&acc->s_cyc, v_scy); atomicAdd(&acc->s_lamsum, v_slam);
                atomicAdd(&acc->s_lensum, v_slen); atomicMax(&acc->s_maxfin, v_smax);
            }
            if (v_on) atomicAdd(&acc->oncycle, v_on);
            if (v_dmin) atomicAdd(&acc->distinct_min, v_dmin);
        }
    }
    __syncthreads();
    flush_hist(shh, acc->hist, a.hbins);
    flush_hist(she, acc->endhist, WAR_EBINS);
}

// Dispatch: variant V selects the turn form (V & 1: multiply-add), the record scheme (V & 2: latched)
// and, for deals with the latched scheme, the cycle memo (V & 4: landmarks, V & 12: all states, V & 28:
// all states and paths); the loop-shape tracker needs the immediate scheme.
template <int RULE, int G, bool CANON, bool SHAPE, bool EXTRA, int V>
__device__ __forceinline__ void refill_dispatch(const BatchArgs& a, DevAcc* __restrict__ acc, u64* __restrict__ counter,
                                                u32* sh) {
    if constexpr (SHAPE && CANON && (V & 30) == 30)   // the loop-shape test with the path memo
        refill_latched<RULE, G, CANON, EXTRA, V & 1, MEMO_PATH, true>(a, acc, counter, sh);
    else if constexpr (SHAPE || (V & 2) == 0) refill_body<RULE, G, CANON, SHAPE, EXTRA, V & 1>(a, acc, counter, sh);
    else if constexpr ((V & 4) == 0 || (CANON && (V & 8) == 0)) refill_latched<RULE, G, CANON, EXTRA, V & 1, MEMO_NONE>(a, acc, counter, sh);
    else if constexpr ((V & 24) == 24) refill_latched<RULE, G, CANON, EXTRA, V & 1, MEMO_PATH>(a, acc, counter, sh);
    else if constexpr ((V & 8) != 0) refill_latched<RULE, G, CANON, EXTRA, V & 1, MEMO_ALL>(a, acc, counter, sh);
    else refill_latched<RULE, G, CANON, EXTRA, V & 1, MEMO_LANDMARK>(a, acc, counter, sh);
}

}  // namespace war
