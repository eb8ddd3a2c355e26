// war_held.cu — the held-out-card engine (war_enumerate_held): deals of up to 17 cards.
//
// With 17 cards a pile no longer fits 4-bit cards in one 64-bit word.  As gpu/war17.py:7-16 observes,
// card n-1 never loses, so it never changes hands and its holder never runs out of cards: it can be kept
// out of the packed piles.  The state is the holder's other cards wh (lh of them), the opponent's cards
// wo (lo), and the depth p of card n-1 in the holder's full pile (0 = on top); lh + lo = n - 1, so
// (wh, wo, lh, p) is the whole position and Brent compares exactly that (gpu/war17.py:62-71).  The game
// ends when the opponent has no card.  The default turn (h_turn_packed_fma) keeps lh and p in one word
// s = 4 lh + 256 p and leaves lo implied, so Brent compares (wh, wo, s).
//
// The kernel is the refill design of war_refill.cuh for this state: a persistent grid, one game per lane,
// outcomes latched every turn and recorded every `defer` turns by the whole warp, work units of aligned
// lexicographic rank blocks (fixed prefix, every order of the last j positions) from one global counter.
// A unit is enumerated as (position of card n-1, order of the other cards): the others stay in deck order
// in one word (16 nibbles at n = 17) and a unit permutes either the last j of them (card n-1 in the
// prefix) or the last j-1 of them for each of the j positions of card n-1 in the suffix — the same set of
// deals as the lexicographic block, so the counts are the same.  With a table (HeldArgs.memo) the engine
// takes the path memo of war_refill.cuh, with a key of its own state (h_key).
#include "war_refill.cuh"

namespace war {

__device__ __forceinline__ u64 shr64(u64 x, u32 s) {   // PTX shr: amounts above 63 give 0
    u64 r;
    asm("shr.b64 %0, %1, %2;" : "=l"(r) : "l"(x), "r"(s));
    return r;
}

__device__ __forceinline__ u32 h_heap_full(u32 j) {
    u32 f = 0;
    for (u32 i = 1; i < j; i++) f |= i << (4u * i);
    return f;
}

struct HEnum {
    u64 O;             // the cards other than n-1, in deck order (others index i in nibble i)
    u32 pos, pos_end;  // position of card n-1 in the deck; positions still to take it: [pos, pos_end)
    u32 base, J;       // Heap's algorithm permutes others indices [base, base + J)
    u32 ctr, full;     // Heap counter (digit i in nibble i) and its last value
    bool live;         // (O, pos) is the next unplayed deal
};

// Takes the next unit; false when there is none.  Unranks its first (lexicographic) order.
__device__ __forceinline__ bool h_fetch(HEnum& E, const HeldArgs& a, u64* counter) {
    const u64 u = atomicAdd(counter, 1ull);
    if (u >= a.n_units) return false;
    u64 r;
    u32 j;
    if (u < a.main_count) {
        j = (u32)a.m;
        r = (a.main_base + u) * a.fact[a.m];
    } else {
        const Unit U = a.units[u - a.main_count];
        r = U.r;
        j = U.j;
    }
    const u32 n = (u32)a.n;
    u32 avail = (1u << n) - 1u, cnt = 0, pos = 0;
    u64 O = 0;
    for (u32 i = 0; i < n; i++) {   // lexicographic unrank (gpu/war17.py:95-104)
        const u64 f = a.fact[n - 1u - i];
        const u32 d = (u32)(r / f);
        r -= (u64)d * f;
        u32 mm = avail;
        for (u32 k = 0; k < d; k++) mm &= mm - 1u;
        const u32 v = (u32)(__ffs((int)mm) - 1);
        avail &= ~(1u << v);
        if (v == n - 1u) pos = i;
        else { O |= (u64)v << (4u * cnt); cnt++; }
    }
    const u32 b = n - j;   // first permuted deck position
    E.O = O;
    if (pos < b) { E.pos = pos; E.pos_end = pos + 1u; E.base = b - 1u; E.J = j; }
    else { E.pos = b; E.pos_end = n; E.base = b; E.J = j - 1u; }
    E.ctr = 0;
    E.full = h_heap_full(E.J);
    E.live = true;
    return true;
}

// Advances to the next deal of the unit (Heap's algorithm over the J permuted others; when it has run
// through all their orders, card n-1 moves one position further).  False after the unit's last deal.
__device__ __forceinline__ bool h_step(HEnum& E) {
    const u32 x = E.ctr ^ E.full;
    if (x != 0u) {
        const u32 i = (u32)(__ffs((int)x) - 1) >> 2;
        const u32 ci = (E.ctr >> (4u * i)) & 15u;
        const u32 o = (i & 1u) ? ci : 0u;
        const u32 sa = 4u * (E.base + i), sb = 4u * (E.base + o);
        const u64 t = ((E.O >> sa) ^ (E.O >> sb)) & 15ull;
        E.O ^= (t << sa) | (t << sb);
        E.ctr = ((E.ctr >> (4u * i)) + 1u) << (4u * i);
        return true;
    }
    if (E.pos + 1u < E.pos_end) {   // every order of the others seen: next position of card n-1
        E.pos++;
        E.ctr = 0;
        return true;
    }
    return false;
}

// Player 1 gets the even deck positions, player 2 the odd ones, the first card on top (gpu/war17.py:48-60).
__device__ __forceinline__ void h_deal(u64 O, u32 pos, u32 n, u64& wh, u64& wo, u32& lh, u32& lo, u32& p) {
    const u32 L = pos;                                   // others dealt before card n-1
    const u64 low = L ? (O & (shr64(~0ull, 64u - 4u * L))) : 0ull;
    const u64 high = shr64(O, 4u * L);
    const u64 p1l = compact_even_nibbles(low), p2l = compact_even_nibbles(low >> 4);
    // after card n-1 the deck position of others index i is i + 1, so the parities swap
    const u64 he = compact_even_nibbles(high), ho = compact_even_nibbles(high >> 4);
    const u64 p1h = (L & 1u) ? he : ho, p2h = (L & 1u) ? ho : he;
    const u64 p1 = p1l | (p1h << (4u * ((L + 1u) >> 1))), p2 = p2l | (p2h << (4u * (L >> 1)));
    const u32 n1 = (n + 1u) >> 1, n2 = n >> 1;
    const bool h1 = (pos & 1u) == 0u;                    // player 1 holds card n-1
    wh = h1 ? p1 : p2;
    wo = h1 ? p2 : p1;
    lh = h1 ? n1 - 1u : n2 - 1u;
    lo = h1 ? n2 : n1;
    p = pos >> 1;
}

// One turn (gpu/war17.py:36-47, with the put-back order of rule 1 added).  Returns true when the game
// is over (the opponent has no card).
template <int RULE>
__device__ __forceinline__ bool h_turn(u64& wh, u64& wo, u32& lh, u32& lo, u32& p) {
    const u32 c = (u32)wo & 15u;
    wo >>= 4;
    lo--;
    if (p == 0u) {   // the holder plays card n-1 and wins the opponent's card
        wh |= shl64((u64)c, 4u * lh);
        lh++;
        p = RULE ? lh : lh - 1u;   // rule 0: n-1 above the captured card; rule 1: below it
    } else {
        const u32 h = (u32)wh & 15u;
        wh >>= 4;
        lh--;
        p--;
        const u32 hi = max(h, c), lw = min(h, c);
        const u32 pair = RULE ? (lw | (hi << 4)) : (hi | (lw << 4));
        if (h > c) { wh |= shl64((u64)pair, 4u * lh); lh += 2u; }
        else { wo |= shl64((u64)pair, 4u * lo); lo += 2u; }
    }
    return lo == 0u;
}

// The same turn without a branch and with the card arithmetic on the multiply-add pipe, the way
// war_turn_fma does it for the main engine: both tops are popped (funnel shift, multiply-high, card =
// lo - 16 lo'), the holder's pop is undone by a select when it plays card n-1, and the one or two cards
// that go under the winner's pile are added to its word by a multiply-add with a 0/1 weight (the nibbles
// above a pile are zero, so adding is placing).  K: the constants of war_turn_fma.
template <int RULE>
__device__ __forceinline__ bool h_turn_fma(u64& wh, u64& wo, u32& lh, u32& lo, u32& p, const TurnK& K) {
    const u32 ol = (u32)wo, oh = (u32)(wo >> 32), hl = (u32)wh, hh = (u32)(wh >> 32);
    const u32 nol = __funnelshift_r(ol, oh, 4), noh = __umulhi(oh, K.k2p28);
    const u32 nhl = __funnelshift_r(hl, hh, 4), nhh = __umulhi(hh, K.k2p28);
    const u32 c = ol + nol * K.km16;                   // the opponent's top card
    const u32 h = hl + nhl * K.km16;                   // the holder's top other card (played when p != 0)
    const bool z = p == 0u;                            // the holder plays card n-1
    const bool hw = z | (h > c);                       // the holder wins the turn
    const u32 hi = max(h, c), lw = min(h, c);
    const u32 pair = RULE ? lw + hi * K.k16 : hi + lw * K.k16;
    const u32 t = z ? c : pair;                        // what goes under the winner's pile
    const u32 lh1 = z ? lh : lh - 1u, lo1 = lo - 1u;   // counts after the pops
    const u32 pos = 4u * (hw ? lh1 : lo1);
    const u64 x = shl64((u64)t, pos);
    const u32 xl = (u32)x, xh = (u32)(x >> 32);
    const u32 bh = hw ? 1u : 0u, bo = K.one - bh;
    u64 ah = z ? wh : (((u64)nhh << 32) | nhl), ao = ((u64)noh << 32) | nol;
    ah = (u64)xl * bh + ah;
    ao = (u64)xl * bo + ao;
    wh = ((u64)((u32)(ah >> 32) + xh * bh) << 32) | (u32)ah;
    wo = ((u64)((u32)(ao >> 32) + xh * bo) << 32) | (u32)ao;
    p = z ? (RULE ? lh + 1u : lh) : p - 1u;
    lh = lh1 + (hw ? (z ? 1u : 2u) : 0u);
    lo = lo1 + (hw ? 0u : 2u);
    return lo == 0u;
}

// The same turn on a packed count word s = 4 lh + 256 p (lh < 64 cards, so the fields never overlap); the
// opponent's count is n - 1 - lh and is not kept.  Branch-free: when card n-1 is on top (s < 256) the
// holder's pop is undone by a select and only the opponent's card goes under its pile.  Brent's test then
// compares three words (wh, wo, s) instead of five, and the game is over exactly when the holder wins the
// opponent's last card (lh = n - 2 before the turn), so no count has to be tested after it.  n4m8 = 4n - 8.
template <int RULE>
__device__ __forceinline__ bool h_turn_packed(u64& wh, u64& wo, u32& s, u32 n4m8) {
    const u32 q = s & 255u;                  // 4 lh
    const bool z = s < 256u;                 // the holder plays card n-1
    const u32 c = (u32)wo & 15u, h = (u32)wh & 15u;
    const u64 ws = wh >> 4;
    wo >>= 4;
    const bool hw = z | (h > c);             // the holder wins the turn
    const u32 hi = max(h, c), lw = min(h, c);
    const u32 pair = RULE ? (lw | (hi << 4)) : (hi | (lw << 4));
    const u32 t = z ? c : pair;              // what goes under the winner's pile
    const u32 pos = hw ? (z ? q : q - 4u) : n4m8 - q;
    const u64 x = shl64((u64)t, pos);
    const u64 m = hw ? ~0ull : 0ull;
    wh = (z ? wh : ws) | (x & m);
    wo = wo | (x & ~m);
    // z: lh + 1 cards, card n-1 at depth lh (rule 0: above the captured card) or lh + 1 (rule 1);
    // else: one card popped from each pile, two added to the winner's, card n-1 one place higher
    s = z ? q * 65u + (4u + 256u * (u32)RULE) : s - 260u + (hw ? 8u : 0u);
    return hw & (q == n4m8);
}

// The packed-count turn with the card arithmetic of h_turn_fma: both tops popped by funnel shift and
// multiply-high, the cards as lo - 16 lo', the pair by multiply-add, and what goes under the winner's pile
// added by mad.wide with a 0/1 weight instead of masks, so about a third of the turn runs on the FMA pipe.
template <int RULE>
__device__ __forceinline__ bool h_turn_packed_fma(u64& wh, u64& wo, u32& s, u32 n4m8, const TurnK& K) {
    const u32 ol = (u32)wo, oh = (u32)(wo >> 32), hl = (u32)wh, hh = (u32)(wh >> 32);
    const u32 nol = __funnelshift_r(ol, oh, 4), noh = __umulhi(oh, K.k2p28);
    const u32 nhl = __funnelshift_r(hl, hh, 4), nhh = __umulhi(hh, K.k2p28);
    const u32 c = ol + nol * K.km16, h = hl + nhl * K.km16;   // the two top cards
    const u32 q = s & 255u;
    const bool z = s < 256u;
    const bool hw = z | (h > c);
    const u32 pa = RULE ? c + h * K.k16 : h + c * K.k16;      // the holder won with h
    const u32 pb = RULE ? h + c * K.k16 : c + h * K.k16;      // the opponent won
    const u32 t = z ? c : (hw ? pa : pb);
    const u32 pos = hw ? (z ? q : q - 4u) : n4m8 - q;
    const u64 x = shl64((u64)t, pos);
    const u32 xl = (u32)x, xh = (u32)(x >> 32);
    const u32 bh = hw ? 1u : 0u, bo = K.one - bh;
    u64 ah = z ? wh : (((u64)nhh << 32) | nhl), ao = ((u64)noh << 32) | nol;
    ah = (u64)xl * bh + ah;
    ao = (u64)xl * bo + ao;
    wh = ((u64)((u32)(ah >> 32) + xh * bh) << 32) | (u32)ah;
    wo = ((u64)((u32)(ao >> 32) + xh * bo) << 32) | (u32)ao;
    s = z ? q * 65u + (4u + 256u * (u32)RULE) : bh * 8u + (s - 260u);
    return hw & (q == n4m8);
}

// Path-memo key of a held-out state (the entry format of war_refill.cuh: the key itself is not stored, the
// slot and entry give it back).  The n-1 other cards in the order holder's then opponent's, the holder's
// count lh and the depth p; the last card is the one missing.  At 17 cards that is 15 nibbles + 8 bits =
// 68 bits, so there the key keeps 13 cards and the order of the last three (one of six, 3 bits): 63 bits.
__device__ __forceinline__ u64 h_key(u64 wh, u64 wo, u32 lh, u32 p, u32 n) {
    const u64 cat = wh | shl64(wo, 4u * lh);
    if (n < 17u) {
        const u32 kb = 4u * (n - 2u);
        return (cat & ((1ull << kb) - 1ull)) | ((u64)lh << kb) | ((u64)p << (kb + 4u));
    }
    const u32 c0 = (u32)(cat >> 52) & 15u, c1 = (u32)(cat >> 56) & 15u, c2 = (u32)(cat >> 60) & 15u;
    const u32 ord = 2u * ((u32)(c0 > c1) + (u32)(c0 > c2)) + (u32)(c1 > c2);
    return (cat & ((1ull << 52) - 1ull)) | ((u64)ord << 52) | ((u64)lh << 55) | ((u64)p << 59);
}

// Walks the cycle of length lam through the given state once and stores every state (value 2 lam).
template <int RULE>
__device__ __noinline__ void h_store_cycle(u64* T, u32 bits, u64 wh, u64 wo, u32 lh, u32 lo, u32 p, u32 n, u32 lam) {
    const u64 v = 2ull * lam;
    if (lam == 0u || (v >> bits) != 0ull) return;
    for (u32 t = 0; t < lam; t++) {
        const u64 k = h_key(wh, wo, lh, p, n);
        __stcg((unsigned long long*)T + memo_slot(k, bits), (unsigned long long)path_entry(k, bits, v));
        h_turn<RULE>(wh, wo, lh, lo, p);
    }
}

// FORM 0: h_turn (branches on card n-1 on top), 1: h_turn_fma, 2: h_turn_packed (the counts in one word),
// 3: h_turn_packed_fma.
// SVC: the window W is a multiple of the service period, so a game (which starts at a service and plays
// `period` turns between services while undecided) reaches each tortoise checkpoint W, 3W, 7W, ... exactly at
// a service; the checkpoint is then saved there instead of being tested after every turn.
template <int RULE, bool MEMO, int FORM, bool SVC>
__global__ void __launch_bounds__(MEMO ? 512 : 1024) held_kernel(const __grid_constant__ HeldArgs a,
                                                                DevAcc* __restrict__ acc) {
    extern __shared__ u32 sh[];
    u32* shh = sh;
    u32* she = sh + a.hbins;
    for (int b = threadIdx.x; b < a.hbins + WAR_EBINS; b += blockDim.x) sh[b] = 0;
    __syncthreads();

    const u32 n = (u32)a.n, W = (u32)a.W, n4m8 = 4u * n - 8u;
    const TurnK K = a.tk;
    const u32 hb1 = a.hbins > 0 ? (u32)(a.hbins - 1) : 0u;
    const int period = a.defer > 4 ? (a.defer + 3) & ~3 : 4;
    u64* counter = &acc->work_next;

    HEnum E;
    E.live = false;
    u64 wh = 0, wo = 0, th = 0, to = 0;
    u32 lh = 0, lo = 0, p = 0, tlh = 0, tp = 0, rounds = 0, next = 0;
    u32 s = 0, ts = 0;   // FORM 2, 3: 4 lh + 256 p
    bool done = true, kcy = false, active = false;
    u32 cyc = 0, ndone = 0, maxfin = 0, capped = 0, turns = 0;
    // the path memo (war_refill.cuh): lookups at every service, the game's last two misses stored with
    // its outcome, cycles found by Brent stored whole
    u64* const memo = MEMO ? a.memo : nullptr;
    const u32 mbits = a.memo_bits;
    const u64 vmask = memo ? (1ull << mbits) - 1ull : 0ull;
    u64 ka = 0, kb = 0;
    u32 ta = 0, tb = 0, mv = 0, mlook = 0, mhit = 0, mstore = 0;

    auto unpack = [&]() {   // FORM 2, 3: the counts of the current state
        if (FORM >= 2) { lh = (s & 255u) >> 2; p = s >> 8; lo = n - 1u - lh; }
    };
    auto save = [&]() {     // the tortoise checkpoint
        th = wh; to = wo;
        if (FORM >= 2) ts = s; else { tlh = lh; tp = p; }
        next = 2u * next + W;
    };
    auto start_game = [&]() {
        active = false;
        for (;;) {
            if (!E.live && !h_fetch(E, a, counter)) return;
            h_deal(E.O, E.pos, n, wh, wo, lh, lo, p);
            E.live = h_step(E);
            break;
        }
        active = true;
        ndone++;
        s = 4u * lh + 256u * p;
        th = wh; to = wo; tlh = lh; tp = p; ts = s;
        rounds = 0; next = W; kcy = false;
        ta = 0u; tb = 0u; mv = 0u;
        done = lo == 0u;   // n = 1 only (never here: n >= 2)
    };

    start_game();
    bool running = __any_sync(WAR_FULL_MASK, active);
    while (running) {
        for (int k = 0; k < period; k++) {
            if (FORM >= 2) {
                const bool en = FORM == 3 ? h_turn_packed_fma<RULE>(wh, wo, s, n4m8, K) : h_turn_packed<RULE>(wh, wo, s, n4m8);
                if (!done) rounds++;
                const bool cy = (wh == th) & (wo == to) & (s == ts);
                kcy = done ? kcy : (cy & !en);
                done = done | cy | en;
            } else {
                bool en = FORM == 1 ? h_turn_fma<RULE>(wh, wo, lh, lo, p, K) : h_turn<RULE>(wh, wo, lh, lo, p);
                if (!done) rounds++;
                const bool cy = (wh == th) & (wo == to) & (lh == tlh) & (p == tp);
                en = en | (lo == 0u);
                const bool fin = (cy | en) & !done;
                kcy = fin ? (cy & !en) : kcy;
                done = done | fin;
                if (lo == 0u) { lo = 1u; wo = 0ull; }   // a finished game keeps being stepped harmlessly
            }
            if (!SVC && rounds == next && !done) {
                if (next > WAR_TURN_CAP) { capped++; done = true; active = false; }
                else save();
            }
        }
        if (SVC && rounds == next && !done) {
            if (next > WAR_TURN_CAP) { capped++; done = true; active = false; }
            else save();
        }
        if (memo != nullptr) {
            unpack();
            const bool look = active & !done;
            const u64 key = h_key(wh, wo, lh, p, n);
            const u64 e = look ? __ldcg((const unsigned long long*)memo + memo_slot(key, mbits)) : 0ull;
            if (look) {
                mlook++;
                if ((e & vmask) != 0ull && ((e ^ path_entry(key, mbits, 0ull)) >> mbits) == 0ull) {
                    mhit++;
                    mv = (u32)(e & vmask);
                    done = true;
                    kcy = (mv & 1u) == 0u;
                } else {
                    kb = ka; tb = ta; ka = key; ta = rounds;
                }
            }
        }
        if (__any_sync(WAR_FULL_MASK, done & active)) {
            if (done & active) {
                turns += rounds;
                const u32 mcy = (mv != 0u && (mv & 1u) == 0u) ? mv >> 1 : 0u;   // the memo's cycle length
                const u32 len = (mv & 1u) ? rounds + (mv >> 1) : rounds;        // or the turns left
                const u32 lam = mcy ? mcy : rounds - ((next - W) >> 1);
                if (memo != nullptr) {
                    if (ta) {
                        const u64 v = kcy ? 2ull * lam : 2ull * (len - ta) + 1ull;
                        if (v <= vmask) { __stcg((unsigned long long*)memo + memo_slot(ka, mbits), path_entry(ka, mbits, v)); mstore++; }
                    }
                    if (tb) {
                        const u64 v = kcy ? 2ull * lam : 2ull * (len - tb) + 1ull;
                        if (v <= vmask) { __stcg((unsigned long long*)memo + memo_slot(kb, mbits), path_entry(kb, mbits, v)); mstore++; }
                    }
                    if (kcy && mcy == 0u) {   // found by Brent: store its cycle (the game is still on it)
                        unpack();
                        h_store_cycle<RULE>(memo, mbits, wh, wo, lh, lo, p, n, lam);
                        mstore += lam;
                    }
                }
                if (kcy) {
                    cyc++;
                    if (a.hbins) atomicAdd(&shh[lam < hb1 ? lam : hb1], 1u);
                } else {
                    if (len > maxfin) maxfin = len;
                    atomicAdd(&she[len < WAR_EBINS - 1 ? len : WAR_EBINS - 1], 1u);
                }
                start_game();
            }
            running = __any_sync(WAR_FULL_MASK, active);
        }
    }

    const u64 v_cyc = warp_sum(cyc), v_done = warp_sum(ndone), v_turns = warp_sum((u64)turns), v_max = warp_max(maxfin);
    const u64 v_cap = warp_sum(capped);
    const u64 v_l = warp_sum((u64)mlook), v_h = warp_sum((u64)mhit), v_s = warp_sum((u64)mstore);
    if ((threadIdx.x & 31) == 0) {
        if (v_l) atomicAdd(&acc->memo_lookups, v_l);
        if (v_h) atomicAdd(&acc->memo_hits, v_h);
        if (v_s) atomicAdd(&acc->memo_stores, v_s);
        if (v_cyc) atomicAdd(&acc->cyc, v_cyc);
        if (v_done) atomicAdd(&acc->done, v_done);
        if (v_turns) atomicAdd(&acc->turns, v_turns);
        if (v_max) atomicMax(&acc->maxfin, v_max);
        if (v_cap) atomicAdd(&acc->status, v_cap);
    }
    __syncthreads();
    flush_hist(shh, acc->hist, a.hbins);
    flush_hist(she, acc->endhist, WAR_EBINS);
}

typedef void (*HeldFn)(const HeldArgs, DevAcc*);

template <int RULE, bool MEMO>
static HeldFn held_pick_form(int form, bool svc) {
    if (form == 3) return svc ? held_kernel<RULE, MEMO, 3, true> : held_kernel<RULE, MEMO, 3, false>;
    if (form == 2) return svc ? held_kernel<RULE, MEMO, 2, true> : held_kernel<RULE, MEMO, 2, false>;
    if (form == 1) return svc ? held_kernel<RULE, MEMO, 1, true> : held_kernel<RULE, MEMO, 1, false>;
    return svc ? held_kernel<RULE, MEMO, 0, true> : held_kernel<RULE, MEMO, 0, false>;
}

// The checkpoint can be saved at the services when W is a multiple of the service period.
bool held_svc(const HeldArgs& a) {
    const int period = a.defer > 4 ? (a.defer + 3) & ~3 : 4;
    return !a.svc_off && a.W % period == 0;
}

static HeldFn held_pick(int rule, bool memo, int form, bool svc) {
    if (rule) return memo ? held_pick_form<1, true>(form, svc) : held_pick_form<1, false>(form, svc);
    return memo ? held_pick_form<0, true>(form, svc) : held_pick_form<0, false>(form, svc);
}

cudaError_t launch_held(const HeldArgs& a, int threads, int blocks, DevAcc* acc, cudaStream_t st) {
    const size_t shmem = sizeof(u32) * (size_t)(a.hbins + WAR_EBINS);
    held_pick(a.rule, a.memo != nullptr, a.form, held_svc(a))<<<blocks, threads, shmem, st>>>(a, acc);
    note_launch();
    return cudaGetLastError();
}

int held_max_blocks_per_sm(int rule, int threads, int hbins, bool memo, int form, bool svc) {
    if (memo && threads > 512) return 0;
    int nb = 0;
    const size_t shmem = sizeof(u32) * (size_t)(hbins + WAR_EBINS);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, held_pick(rule, memo, form, svc), threads, shmem);
    return e == cudaSuccess ? nb : 0;
}

}  // namespace war
