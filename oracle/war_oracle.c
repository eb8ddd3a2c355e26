/* war_oracle.c — THE ORACLE.  Test infrastructure only: the CPU restatement of the reference's
 * exhaustive War enumerator (gpu/war_gpu.py) that the tests, the smoke check and the benchmark's
 * CPU-baseline leg use as the checker.  Nothing in the product links or calls this file.
 *
 * It follows the reference step for step, in plain C with OpenMP over contiguous rank sub-ranges:
 *   turn              WAR_STEP            gpu/war_gpu.py:38-45  (same rule as cpu/war.cpp:17-23)
 *   brent             war_sim (Brent)     gpu/war_gpu.py:77-96  (checkpoint schedule of cpu/war.cpp:26-37)
 *   deal              war_cycles          gpu/war_gpu.py:98-107
 *   unrank            war_count unrank    gpu/war_gpu.py:135-146 (and war_canon :196-206)
 *   next_perm         next_perm           gpu/war_gpu.py:109-119
 *   half filter       --half              gpu/war_gpu.py:147-154
 *   canon position    war_canon           gpu/war_gpu.py:208-213
 *   distinct weights  war_canon           gpu/war_gpu.py:217-235
 *   min-key distinct  distinct_cycles     cpu/distinct_cycles.c:84-92, :128-141
 *   loop_shape        Theorem-3 test      gpu/war_gpu.py:51-73
 *   floyd             second detector     gpu/war_gpu_floyd.py:95-105 (tortoise/hare, hare steps = game length)
 *   held-out card     n <= 17 deals       gpu/war17.py:36-113 (oracle_enumerate_held)
 *   5-bit piles       n <= 20 deals       gpu/war24.py:31-139 (oracle_war24: Floyd, streak test, step cap)
 * Piles use the reference's layout: 4-bit cards in a uint64, top card in the low nibble, explicit
 * lengths.  Additions with no reference counterpart (turn totals, ending-length histogram, sample
 * aggregates) are computed from the same per-game results.
 *
 * Pinned against the reference's recorded outputs (data/checks.txt, data/long_runs.txt,
 * data/deals.tsv, data/canonical_positions.tsv, data/loser_first.tsv) by tests/test_oracle.py, and
 * against cpu/war.cpp built unmodified into oracle/_ref/ when that binary is present.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/war.h"

typedef struct { uint64_t w1, w2; int l1, l2; } St;

/* WAR_STEP, gpu/war_gpu.py:38-45.  Returns 1 if player 1 won the turn. */
static inline int turn(St* s, int rule) {
    uint64_t c1 = s->w1 & 15u, c2 = s->w2 & 15u;
    s->w1 >>= 4; s->l1--;
    s->w2 >>= 4; s->l2--;
    if (c1 > c2) {
        uint64_t a = rule ? c2 : c1, b = rule ? c1 : c2;
        s->w1 |= a << (4 * s->l1); s->l1++;
        s->w1 |= b << (4 * s->l1); s->l1++;
        return 1;
    }
    uint64_t a = rule ? c1 : c2, b = rule ? c2 : c1;
    s->w2 |= a << (4 * s->l2); s->l2++;
    s->w2 |= b << (4 * s->l2); s->l2++;
    return 0;
}

static inline int same(const St* a, const St* b) { return a->w1 == b->w1 && a->w2 == b->w2 && a->l1 == b->l1; }

/* war_sim, gpu/war_gpu.py:77-96.  Returns 1 if the game never ends; *rounds = turns played until the
 * end or until the repeat was found; *lam = exact cycle length; *meet = the state at detection. */
static int brent(St s, int rule, uint64_t* rounds_out, uint64_t* lam_out, St* meet) {
    if (s.l1 == 0 || s.l2 == 0) { *rounds_out = 0; return 0; }
    St t = s;
    uint64_t power = 1, lam = 0, rounds = 0;
    for (;;) {
        turn(&s, rule);
        rounds++;
        if (s.l1 == 0 || s.l2 == 0) { *rounds_out = rounds; return 0; }
        lam++;
        if (same(&s, &t)) { *rounds_out = rounds; *lam_out = lam; if (meet) *meet = s; return 1; }
        if (lam == power) { t = s; power <<= 1; lam = 0; }
    }
}

/* Floyd, as in gpu/war_gpu_floyd.py:95-105: the hare takes two turns per tortoise turn, the hare's
 * turn count is the game length when it ends; for a cycle the length is found by walking the loop
 * once from the meeting point. */
static int floyd(St s, int rule, uint64_t* rounds_out, uint64_t* lam_out) {
    if (s.l1 == 0 || s.l2 == 0) { *rounds_out = 0; return 0; }
    St t = s, h = s;
    uint64_t steps = 0;
    for (;;) {
        turn(&h, rule); steps++;
        if (h.l1 == 0 || h.l2 == 0) { *rounds_out = steps; return 0; }
        turn(&h, rule); steps++;
        if (h.l1 == 0 || h.l2 == 0) { *rounds_out = steps; return 0; }
        turn(&t, rule);
        if (same(&t, &h)) break;
    }
    St c = h; uint64_t lam = 0;
    do { turn(&c, rule); lam++; } while (!same(&c, &h));
    *rounds_out = steps; *lam_out = lam;
    return 1;
}

/* loop_shape, gpu/war_gpu.py:51-73: 0 = every cyclic run of wins has length blk, 1 = not,
 * 2 = loop longer than 512 turns (not checked). */
static int loop_shape(St s, uint64_t lam, int blk, int rule) {
    if (lam > 512) return 2;
    unsigned char bits[512];
    int L = (int)lam;
    for (int i = 0; i < L; i++) bits[i] = (unsigned char)turn(&s, rule);
    int st = -1;
    for (int i = 0; i < L; i++) if (bits[i] != bits[(i + L - 1) % L]) { st = i; break; }
    if (st < 0) return 1;
    int run = 1;
    for (int j = 1; j <= L; j++) {
        if (j < L && bits[(st + j) % L] == bits[(st + j - 1) % L]) { run++; continue; }
        if (run != blk) return 1;
        run = 1;
    }
    return 0;
}

/* Key of cpu/distinct_cycles.c:84-92, generalised to two words so that n = 16 fits: player 1's
 * length, then player 1's cards top first, then player 2's.  Compared lexicographically. */
typedef struct { uint32_t len1; uint64_t seq; } Key;
static inline Key key_of(uint64_t w1, int l1, uint64_t w2, int l2) {
    Key k; k.len1 = (uint32_t)l1; k.seq = 0;
    for (int i = 0; i < l1; i++) { k.seq = (k.seq << 4) | (w1 & 15u); w1 >>= 4; }
    for (int i = 0; i < l2; i++) { k.seq = (k.seq << 4) | (w2 & 15u); w2 >>= 4; }
    return k;
}
static inline int key_lt(Key a, Key b) { return a.len1 < b.len1 || (a.len1 == b.len1 && a.seq < b.seq); }
static inline int key_eq(Key a, Key b) { return a.len1 == b.len1 && a.seq == b.seq; }

/* The seeded sample predicate (war_sample_pick in include/war.h). */
static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27; x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}
int oracle_sample_pick(uint64_t seed, uint32_t ppm, uint64_t w1s, uint64_t w2s) {
    uint64_t x = mix64(seed ^ (w1s * 0x9E3779B97F4A7C15ull) ^ (w2s * 0xC2B2AE3D27D4EB4Full));
    uint64_t thr = ((uint64_t)ppm << 32) / 1000000u;
    return (x >> 32) < thr;
}

/* The 1 bit just above a pile of len cards (none for a full 16-card word). */
static inline uint64_t sentinel(int len) { return len < 16 ? 1ull << (4 * len) : 0ull; }

/* unrank, gpu/war_gpu.py:135-146: lexicographic permutation of 0..m-1 with rank idx. */
static void unrank(uint64_t idx, int m, unsigned char* a) {
    uint64_t f[17]; f[0] = 1;
    for (int i = 1; i <= 16; i++) f[i] = f[i - 1] * (uint64_t)i;
    unsigned avail = (1u << m) - 1u;
    uint64_t r = idx;
    for (int i = 0; i < m; i++) {
        uint64_t fi = f[m - 1 - i];
        int d = (int)(r / fi); r -= (uint64_t)d * fi;
        unsigned mm = avail;
        for (int k = 0; k < d; k++) mm &= mm - 1u;
        int v = __builtin_ctz(mm);
        a[i] = (unsigned char)v; avail &= ~(1u << v);
    }
}

/* next_perm, gpu/war_gpu.py:109-119 */
static int next_perm(unsigned char* a, int n) {
    int i = n - 2;
    while (i >= 0 && a[i] >= a[i + 1]) i--;
    if (i < 0) return 0;
    int j = n - 1;
    while (a[j] <= a[i]) j--;
    unsigned char t = a[i]; a[i] = a[j]; a[j] = t;
    for (int l = i + 1, r = n - 1; l < r; l++, r--) { t = a[l]; a[l] = a[r]; a[r] = t; }
    return 1;
}

typedef struct {
    int n, mode, rule, flags, hbins, dbins, blk;
    uint32_t ppm; uint64_t seed;
} Ctx;

/* Plays one position and folds its result into acc (per-thread accumulator). */
static void play(const Ctx* c, St s, war_result* acc) {
    uint64_t rounds = 0, lam = 0;
    St mt;
    int cyc = brent(s, c->rule, &rounds, &lam, &mt);
    acc->done++;
    acc->turns += rounds;
    if (cyc) {
        acc->cyc++;
        if (c->hbins) acc->hist[lam < (uint64_t)(c->hbins - 1) ? lam : (uint64_t)(c->hbins - 1)]++;
        if (c->mode == WAR_CANON && (c->flags & WAR_F_DISTINCT)) {
            /* gpu/war_gpu.py:224-234: walk lam turns from the start, counting canonical states */
            St v = s; uint64_t c1 = 0, c2 = 0; int sym = 0;
            Key kmin = {0xFFFFFFFFu, ~0ull};
            for (uint64_t t = 0; t < lam; t++) {
                if (v.l1 > 0 && (v.w1 & 15u) == (uint64_t)(c->n - 1)) {
                    c1++;
                    Key k = key_of(v.w1, v.l1, v.w2, v.l2);
                    if (key_lt(k, kmin)) kmin = k;
                }
                if (v.l2 > 0 && (v.w2 & 15u) == (uint64_t)(c->n - 1)) {
                    c2++;
                    Key k = key_of(v.w2, v.l2, v.w1, v.l1);   /* the swapped state, distinct_cycles.c:134 */
                    if (key_lt(k, kmin)) kmin = k;
                }
                if (v.w1 == s.w2 && v.w2 == s.w1 && v.l1 == s.l2) sym = 1;
                turn(&v, c->rule);
            }
            if (same(&v, &s)) {
                uint64_t d = sym ? c1 : c1 + c2;
                acc->oncycle++;
                if (c->dbins) acc->dhist[d < (uint64_t)(c->dbins - 1) ? d : (uint64_t)(c->dbins - 1)]++;
                if (key_eq(key_of(s.w1, s.l1, s.w2, s.l2), kmin)) acc->distinct_min++;
            }
        }
        if (c->mode == WAR_CANON && (c->flags & WAR_F_SHAPE) && c->blk) {
            int shp = loop_shape(mt, lam, c->blk, c->rule);
            if (shp == 1) acc->shape_nonstd++;
            else if (shp == 2) acc->shape_unchecked++;
        }
    } else {
        if (rounds > acc->maxfin) acc->maxfin = rounds;
        acc->endhist[rounds < WAR_EBINS - 1 ? rounds : WAR_EBINS - 1]++;
    }
    if (c->flags & WAR_F_SAMPLE) {
        uint64_t w1s = s.w1 | sentinel(s.l1), w2s = s.w2 | sentinel(s.l2);
        if (oracle_sample_pick(c->seed, c->ppm, w1s, w2s)) {
            acc->s_count++;
            if (cyc) { acc->s_cyc++; acc->s_lamsum += lam; }
            else { acc->s_lensum += rounds; if (rounds > acc->s_maxfin) acc->s_maxfin = rounds; }
        }
    }
}

/* Same sample, Floyd detector. */
static void play_floyd(const Ctx* c, St s, war_result* acc) {
    uint64_t w1s = s.w1 | sentinel(s.l1), w2s = s.w2 | sentinel(s.l2);
    if (!oracle_sample_pick(c->seed, c->ppm, w1s, w2s)) return;
    uint64_t rounds = 0, lam = 0;
    int cyc = floyd(s, c->rule, &rounds, &lam);
    acc->s_count++;
    if (cyc) { acc->s_cyc++; acc->s_lamsum += lam; }
    else { acc->s_lensum += rounds; if (rounds > acc->s_maxfin) acc->s_maxfin = rounds; }
}

static St deal_state(const unsigned char* p, int n) {     /* war_cycles, gpu/war_gpu.py:98-107 */
    St s; s.w1 = s.w2 = 0; s.l1 = s.l2 = 0;
    for (int i = 0; i < n; i++) {
        if ((i & 1) == 0) { s.w1 |= ((uint64_t)p[i]) << (4 * s.l1); s.l1++; }
        else { s.w2 |= ((uint64_t)p[i]) << (4 * s.l2); s.l2++; }
    }
    return s;
}

static St canon_state(const unsigned char* q, int n, int k) {   /* gpu/war_gpu.py:210-213 */
    int m = n - 1;
    St s; s.w1 = (uint64_t)(n - 1); s.l1 = 1; s.w2 = 0; s.l2 = 0;
    for (int i = 0; i < k; i++) { s.w1 |= ((uint64_t)q[i]) << (4 * s.l1); s.l1++; }
    for (int i = k; i < m; i++) { s.w2 |= ((uint64_t)q[i]) << (4 * s.l2); s.l2++; }
    return s;
}

static void merge(war_result* dst, const war_result* src) {
    dst->cyc += src->cyc; dst->done += src->done; dst->turns += src->turns;
    if (src->maxfin > dst->maxfin) dst->maxfin = src->maxfin;
    dst->shape_nonstd += src->shape_nonstd; dst->shape_unchecked += src->shape_unchecked;
    dst->oncycle += src->oncycle; dst->distinct_min += src->distinct_min;
    dst->s_count += src->s_count; dst->s_cyc += src->s_cyc; dst->s_lamsum += src->s_lamsum;
    dst->s_lensum += src->s_lensum;
    if (src->s_maxfin > dst->s_maxfin) dst->s_maxfin = src->s_maxfin;
    dst->undetermined += src->undetermined;
    for (int i = 0; i < WAR_HBINS_MAX; i++) dst->hist[i] += src->hist[i];
    for (int i = 0; i < WAR_DBINS_MAX; i++) dst->dhist[i] += src->dhist[i];
    for (int i = 0; i < WAR_EBINS; i++) dst->endhist[i] += src->endhist[i];
}

static uint64_t space_size(int n, int mode) {
    uint64_t f = 1;
    if (mode == WAR_CANON) {
        if (n < 2) return 0;
        for (int i = 2; i <= n - 1; i++) f *= (uint64_t)i;
        return f * (uint64_t)(n - 1);
    }
    for (int i = 2; i <= n; i++) f *= (uint64_t)i;
    return f;
}

/* Walks ranks [lo, hi) of the job in lexicographic order (deals) or (order, split) order (canon). */
static void walk(const Ctx* c, uint64_t lo, uint64_t hi, war_result* acc, int use_floyd) {
    if (lo >= hi) return;
    int n = c->n;
    unsigned char a[16];
    if (c->mode == WAR_DEALS) {
        unrank(lo, n, a);
        for (uint64_t r = lo; r < hi; r++) {
            int take = 1;
            if (c->flags & WAR_F_HALF) {           /* gpu/war_gpu.py:151-154 */
                int pos = 0; while (a[pos] != (unsigned char)(n - 1)) pos++;
                take = (pos & 1) == 0;
            }
            if (take) {
                St s = deal_state(a, n);
                if (use_floyd) play_floyd(c, s, acc); else play(c, s, acc);
            }
            if (r + 1 < hi) next_perm(a, n);
        }
    } else {
        int m = n - 1;
        uint64_t p = lo / (uint64_t)m; int k = (int)(lo % (uint64_t)m);
        unrank(p, m, a);
        for (uint64_t r = lo; r < hi; r++) {
            St s = canon_state(a, n, k);
            if (use_floyd) play_floyd(c, s, acc); else play(c, s, acc);
            if (++k == m) { k = 0; if (r + 1 < hi) next_perm(a, m); }
        }
    }
}

static int run_job(const war_job* job, int nthreads, war_result* out, int use_floyd) {
    if (!job || !out) return WAR_EINVAL;
    if (job->n < 1 || job->n > WAR_MAX_N || job->mode < 0 || job->mode > 1) return WAR_EINVAL;
    if (job->hbins < 0 || job->hbins > WAR_HBINS_MAX || job->dbins < 0 || job->dbins > WAR_DBINS_MAX) return WAR_EINVAL;
    uint64_t total = space_size(job->n, job->mode);
    if (job->lo > job->hi || job->hi > total) return WAR_EINVAL;
    Ctx c;
    c.n = job->n; c.mode = job->mode; c.rule = job->rule; c.flags = job->flags;
    c.hbins = job->hbins; c.dbins = job->dbins;
    c.blk = job->blk ? job->blk : (job->n & -job->n);
    c.ppm = job->sample_ppm; c.seed = job->seed;
    memset(out, 0, sizeof(*out));
    out->hbins = job->hbins; out->dbins = job->dbins; out->blk = (job->flags & WAR_F_SHAPE) ? c.blk : 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    uint64_t len = job->hi - job->lo;
    if ((uint64_t)nthreads > len / 64 + 1) nthreads = (int)(len / 64 + 1);
    war_result* parts = (war_result*)calloc((size_t)nthreads, sizeof(war_result));
    if (!parts) return WAR_ENOMEM;
    /* Contiguous pieces, many more than threads, handed out dynamically. */
    uint64_t pieces = (uint64_t)nthreads * 64u;
    if (pieces > len) pieces = len ? len : 1;
    #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (long long pc = 0; pc < (long long)pieces; pc++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        uint64_t a = job->lo + len * (uint64_t)pc / pieces;
        uint64_t b = job->lo + len * (uint64_t)(pc + 1) / pieces;
        walk(&c, a, b, &parts[tid], use_floyd);
    }
    for (int t = 0; t < nthreads; t++) merge(out, &parts[t]);
    free(parts);
    return WAR_OK;
}

/* Enumerate ranks [lo, hi) of the job with the reference's algorithm; nthreads <= 0 = all cores. */
int oracle_enumerate(const war_job* job, int nthreads, war_result* out) { return run_job(job, nthreads, out, 0); }

/* Floyd over the seeded sample of the job; fills only the s_* fields. */
int oracle_floyd_sample(const war_job* job, int nthreads, war_result* out) { return run_job(job, nthreads, out, 1); }

/* One position given as piles (reference layout).  Returns 1 if it cycles. */
int oracle_play_one(uint64_t w1, int l1, uint64_t w2, int l2, int rule, uint64_t* rounds, uint64_t* lam) {
    St s; s.w1 = w1; s.w2 = w2; s.l1 = l1; s.l2 = l2;
    *lam = 0;
    return brent(s, rule, rounds, lam, NULL);
}

/* ---- the held-out-card program, gpu/war17.py (deals of n <= 17) -------------------------------------
 * Card n-1 is kept out of the packed piles (gpu/war17.py:7-16); the holder's other cards, the opponent's
 * cards and the depth p of card n-1 in the holder's pile are the state; Brent on the whole state with the
 * reference's schedule (:62-71).  Rule 1 (loser's card first) is added the same way as in war_gpu.py. */
typedef struct { uint64_t wh, wo; int lh, lo, p; } HSt;

/* turn, gpu/war17.py:36-47.  Returns 1 when the opponent is out of cards. */
static inline int hturn(HSt* s, int rule) {
    if (s->p == 0) {
        uint64_t c = s->wo & 15u; s->wo >>= 4; s->lo--;
        if (rule) { s->wh |= c << (4 * s->lh); s->lh++; s->p = s->lh; }
        else { s->p = s->lh; s->wh |= c << (4 * s->lh); s->lh++; }
        return s->lo == 0;
    }
    uint64_t h = s->wh & 15u; s->wh >>= 4; s->lh--; s->p--;
    uint64_t o = s->wo & 15u; s->wo >>= 4; s->lo--;
    if (h > o) {
        uint64_t x = rule ? o : h, y = rule ? h : o;
        s->wh |= x << (4 * s->lh); s->lh++; s->wh |= y << (4 * s->lh); s->lh++;
    } else {
        uint64_t x = rule ? h : o, y = rule ? o : h;
        s->wo |= x << (4 * s->lo); s->lo++; s->wo |= y << (4 * s->lo); s->lo++;
    }
    return s->lo == 0;
}

/* deal_cycles, gpu/war17.py:50-71.  Returns 1 if the game never ends; *len = turns to the end, or the
 * turns played until the repeat was found; *lam = the cycle length. */
static int hdeal(const unsigned char* a, int n, int rule, uint64_t* len, uint64_t* lam_out) {
    uint64_t w1 = 0, w2 = 0; int l1 = 0, l2 = 0, holder = 0, p = 0;
    for (int i = 0; i < n; i++) {
        int pl = i & 1;
        if (a[i] == (unsigned char)(n - 1)) { holder = pl; p = pl ? l2 : l1; continue; }
        if (pl == 0) { w1 |= ((uint64_t)a[i]) << (4 * l1); l1++; }
        else { w2 |= ((uint64_t)a[i]) << (4 * l2); l2++; }
    }
    HSt s; s.wh = holder ? w2 : w1; s.wo = holder ? w1 : w2; s.lh = holder ? l2 : l1; s.lo = holder ? l1 : l2; s.p = p;
    if (s.lo == 0) { *len = 0; return 0; }
    HSt t = s;
    uint64_t power = 1, lam = 0, rounds = 0;
    for (;;) {
        rounds++;
        if (hturn(&s, rule)) { *len = rounds; return 0; }
        lam++;
        if (s.wh == t.wh && s.wo == t.wo && s.lh == t.lh && s.p == t.p) { *len = rounds; *lam_out = lam; return 1; }
        if (lam == power) { t = s; power <<= 1; lam = 0; }
    }
}

/* Ranks [lo, hi) of the n! deals (lexicographic, gpu/war17.py:95-113) with the held-out program. */
int oracle_enumerate_held(const war_job* job, int nthreads, war_result* out) {
    if (!job || !out || job->n < 2 || job->n > 17 || job->mode != WAR_DEALS) return WAR_EINVAL;
    if (job->hbins < 0 || job->hbins > WAR_HBINS_MAX) return WAR_EINVAL;
    const int n = job->n, rule = job->rule, hbins = job->hbins;
    uint64_t f[18]; f[0] = 1;
    for (int i = 1; i <= 17; i++) f[i] = f[i - 1] * (uint64_t)i;
    if (job->lo > job->hi || job->hi > f[n]) return WAR_EINVAL;
    memset(out, 0, sizeof(*out));
    out->hbins = hbins;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    uint64_t len = job->hi - job->lo;
    if ((uint64_t)nthreads > len / 64 + 1) nthreads = (int)(len / 64 + 1);
    war_result* parts = (war_result*)calloc((size_t)nthreads, sizeof(war_result));
    if (!parts) return WAR_ENOMEM;
    uint64_t pieces = (uint64_t)nthreads * 64u;
    if (pieces > len) pieces = len ? len : 1;
    #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (long long pc = 0; pc < (long long)pieces; pc++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        war_result* acc = &parts[tid];
        uint64_t lo = job->lo + len * (uint64_t)pc / pieces, hi = job->lo + len * (uint64_t)(pc + 1) / pieces;
        if (lo >= hi) continue;
        unsigned char a[17];
        unsigned avail = (1u << n) - 1u;
        uint64_t r = lo;
        for (int i = 0; i < n; i++) {
            uint64_t fi = f[n - 1 - i];
            int d = (int)(r / fi); r -= (uint64_t)d * fi;
            unsigned m = avail;
            for (int k = 0; k < d; k++) m &= m - 1u;
            int v = __builtin_ctz(m);
            a[i] = (unsigned char)v; avail &= ~(1u << v);
        }
        for (uint64_t q = lo; q < hi; q++) {
            uint64_t gl = 0, lam = 0;
            acc->done++;
            if (hdeal(a, n, rule, &gl, &lam)) {
                acc->cyc++;
                if (hbins) acc->hist[lam < (uint64_t)(hbins - 1) ? lam : (uint64_t)(hbins - 1)]++;
            } else {
                if (gl > acc->maxfin) acc->maxfin = gl;
                acc->endhist[gl < WAR_EBINS - 1 ? gl : WAR_EBINS - 1]++;
            }
            acc->turns += gl;
            if (q + 1 < hi) {   /* next_perm, gpu/war17.py:74-84 */
                int i = n - 2;
                while (i >= 0 && a[i] >= a[i + 1]) i--;
                if (i >= 0) {
                    int j = n - 1;
                    while (a[j] <= a[i]) j--;
                    unsigned char t = a[i]; a[i] = a[j]; a[j] = t;
                    for (int l = i + 1, rr = n - 1; l < rr; l++, rr--) { t = a[l]; a[l] = a[rr]; a[rr] = t; }
                }
            }
        }
    }
    for (int t = 0; t < nthreads; t++) merge(out, &parts[t]);
    free(parts);
    return WAR_OK;
}

/* ---- the 5-bit program of gpu/war24.py: deals of n <= 20 cards ------------------------------------------
 * Cards are 5 bits and a pile is two 64-bit words (lo, hi) with the top card in the lowest 5 bits and an
 * explicit length (gpu/war24.py:31-47); a deal's rank is its lexicographic rank among the n! orders, unranked
 * with the Lehmer code of :64-77 and stepped with the next permutation of :127-137.  Two detectors follow the
 * reference line by line, each with its step cap (:57) after which a game counts as undetermined:
 *   floyd   tortoise and hare, two hare turns per tortoise turn; cap tested after the tortoise turn (:82-95)
 *   streak  odd n: anchor where the next winner holds an even number of cards, then expect the players to
 *           alternate for lcm(n+1, W, L-1) turns and compare with the anchor (:96-125)
 * and a third, Brent with the tortoise saved at turns W, 3W, 7W, ... (the engine's default), which is this
 * repository's addition, like the loser-first rule (the reference plays rule 0 only).  The step count of an
 * ending game is its length in every detector. */
typedef struct { uint64_t lo, hi; } P5;
typedef struct { P5 a, b; int la; } S5;
enum { DET_BRENT = 0, DET_FLOYD = 1, DET_STREAK = 2 };

static inline unsigned pop5(P5* p) {                        /* popc5, gpu/war24.py:31-35 */
    unsigned c = (unsigned)(p->lo & 31u);
    p->lo = (p->lo >> 5) | (p->hi << 59); p->hi >>= 5;
    return c;
}
static inline void put5(P5* p, int L, uint64_t v, int bits) {   /* put, gpu/war24.py:36-41 */
    int q = 5 * L;
    uint64_t slo = (q < 64) ? (v << q) : 0ull;
    uint64_t shi = (q >= 64) ? (v << (q - 64)) : ((q + bits > 64) ? (v >> (64 - q)) : 0ull);
    p->lo |= slo; p->hi |= shi;
}
static inline int pstep5(S5* s, int n, int rule) {          /* pstep, gpu/war24.py:42-47 (+ rule 1) */
    int lb = n - s->la;
    unsigned ta = pop5(&s->a), tb = pop5(&s->b);
    if (ta > tb) {
        put5(&s->a, s->la - 1, rule ? ((uint64_t)tb | ((uint64_t)ta << 5)) : ((uint64_t)ta | ((uint64_t)tb << 5)), 10);
        s->la += 1; return 1;
    }
    put5(&s->b, lb - 1, rule ? ((uint64_t)ta | ((uint64_t)tb << 5)) : ((uint64_t)tb | ((uint64_t)ta << 5)), 10);
    s->la -= 1; return 0;
}
static inline int eq5(const S5* x, const S5* y) {
    return x->a.lo == y->a.lo && x->a.hi == y->a.hi && x->b.lo == y->b.lo && x->b.hi == y->b.hi && x->la == y->la;
}
static int gcd5(int a, int b) { while (b) { int t = a % b; a = b; b = t; } return a; }
static int lcm5(int a, int b) { return a / gcd5(a, b) * b; }

/* Returns 0 = ends, 1 = cycles, 2 = undetermined; *steps = turns played (the game's length if it ends). */
static int floyd5(S5 s, int n, int rule, uint64_t cap, uint64_t* steps_out) {      /* gpu/war24.py:85-97 */
    S5 t = s, h = s;
    uint64_t steps = 0;
    for (;;) {
        if (h.la == 0 || h.la == n) { *steps_out = steps; return 0; }
        pstep5(&h, n, rule); steps++;
        if (h.la == 0 || h.la == n) { *steps_out = steps; return 0; }
        pstep5(&h, n, rule); steps++;
        if (h.la == 0 || h.la == n) { *steps_out = steps; return 0; }
        pstep5(&t, n, rule);
        if (eq5(&t, &h)) { *steps_out = steps; return 1; }
        if (steps > cap) { *steps_out = steps; return 2; }
    }
}

static int streak5(S5 s, int n, int rule, uint64_t cap, uint64_t* steps_out) {      /* gpu/war24.py:98-125 */
    int anch = 0, lam = 0, since = 0, prevw = -1;
    S5 sv = s;
    uint64_t steps = 0;
    for (;;) {
        if (s.la == 0 || s.la == n) { *steps_out = steps; return 0; }
        if (steps > cap) { *steps_out = steps; return 2; }
        if (!anch) {
            unsigned ta = (unsigned)(s.a.lo & 31u), tb = (unsigned)(s.b.lo & 31u);
            int ws = (ta > tb) ? s.la : (n - s.la), ls = n - ws;
            if ((ws & 1) == 0 && ls >= 2) {
                anch = 1; since = 0; prevw = -1;
                lam = lcm5(n + 1, lcm5(ws, ls - 1));
                sv = s;
            }
        }
        int w = pstep5(&s, n, rule); steps++;
        if (anch) {
            if (w == prevw) anch = 0;
            else {
                prevw = w; since++;
                if (since == lam) {
                    if (eq5(&s, &sv)) { *steps_out = steps; return 1; }
                    anch = 0;
                }
            }
        }
    }
}

static int brent5(S5 s, int n, int rule, uint64_t cap, uint64_t W, uint64_t* steps_out, uint64_t* lam_out) {
    if (s.la == 0 || s.la == n) { *steps_out = 0; return 0; }
    S5 t = s;
    uint64_t rounds = 0, next = W, last = 0;
    for (;;) {
        pstep5(&s, n, rule); rounds++;
        if (s.la == 0 || s.la == n) { *steps_out = rounds; return 0; }
        if (eq5(&s, &t)) { *steps_out = rounds; *lam_out = rounds - last; return 1; }
        if (rounds > cap) { *steps_out = rounds; return 2; }
        if (rounds == next) { t = s; last = rounds; next = 2 * next + W; }
    }
}

/* Ranks [lo, hi) of the n! deals of gpu/war24.py (2 <= n <= 20).  det: 0 Brent (first window `window`),
 * 1 Floyd, 2 streak (odd n, rule 0).  cap: the step cap (0 = 2^22, gpu/war24.py:57).  Fills cyc, done,
 * maxfin, undetermined, turns (steps played), endhist and, with Brent, the cycle-length histogram. */
int oracle_war24(const war_job* job, int det, uint32_t window, uint64_t cap, int nthreads, war_result* out) {
    if (!job || !out || job->n < 2 || job->n > 20 || job->mode != WAR_DEALS) return WAR_EINVAL;
    if (det < 0 || det > 2 || (det == DET_STREAK && (!(job->n & 1) || job->rule))) return WAR_EINVAL;
    if (job->hbins < 0 || job->hbins > WAR_HBINS_MAX || window < 1) return WAR_EINVAL;
    const int n = job->n, rule = job->rule, hbins = det == DET_BRENT ? job->hbins : 0;
    if (cap == 0) cap = 1ull << 22;
    uint64_t f[21]; f[0] = 1;
    for (int i = 1; i <= 20; i++) f[i] = f[i - 1] * (uint64_t)i;
    if (job->lo > job->hi || job->hi > f[n]) return WAR_EINVAL;
    memset(out, 0, sizeof(*out));
    out->hbins = hbins;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    uint64_t len = job->hi - job->lo;
    if ((uint64_t)nthreads > len / 64 + 1) nthreads = (int)(len / 64 + 1);
    war_result* parts = (war_result*)calloc((size_t)nthreads, sizeof(war_result));
    if (!parts) return WAR_ENOMEM;
    uint64_t pieces = (uint64_t)nthreads * 64u;
    if (pieces > len) pieces = len ? len : 1;
    #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (long long pc = 0; pc < (long long)pieces; pc++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        war_result* acc = &parts[tid];
        uint64_t lo = job->lo + len * (uint64_t)pc / pieces, hi = job->lo + len * (uint64_t)(pc + 1) / pieces;
        if (lo >= hi) continue;
        unsigned char q[20];
        {   /* Lehmer unrank of lo, gpu/war24.py:60-74 */
            unsigned char avail[20];
            for (int i = 0; i < n; i++) avail[i] = (unsigned char)i;
            uint64_t r = lo;
            int left = n;
            for (int i = 0; i < n; i++) {
                uint64_t fi = f[left - 1];
                uint64_t d = left > 1 ? r / fi : 0;
                if (left > 1) r %= fi;
                q[i] = avail[d];
                for (int k = (int)d; k < left - 1; k++) avail[k] = avail[k + 1];
                left--;
            }
        }
        for (uint64_t x = lo; x < hi; x++) {
            S5 s;   /* the deal, gpu/war24.py:76-82: even positions to player 1, first card on top */
            s.a.lo = s.a.hi = s.b.lo = s.b.hi = 0;
            int la = 0, lb = 0;
            for (int i = 0; i < n; i++) {
                if ((i & 1) == 0) { put5(&s.a, la, q[i], 5); la++; }
                else { put5(&s.b, lb, q[i], 5); lb++; }
            }
            s.la = la;
            uint64_t steps = 0, lam = 0;
            int res = det == DET_FLOYD ? floyd5(s, n, rule, cap, &steps)
                    : det == DET_STREAK ? streak5(s, n, rule, cap, &steps)
                    : brent5(s, n, rule, cap, window, &steps, &lam);
            acc->done++;
            acc->turns += steps;
            if (res == 1) {
                acc->cyc++;
                if (hbins) acc->hist[lam < (uint64_t)(hbins - 1) ? lam : (uint64_t)(hbins - 1)]++;
            } else if (res == 2) {
                acc->undetermined++;
            } else {
                if (steps > acc->maxfin) acc->maxfin = steps;
                acc->endhist[steps < WAR_EBINS - 1 ? steps : WAR_EBINS - 1]++;
            }
            if (x + 1 < hi) next_perm(q, n);   /* gpu/war24.py:129-139 */
        }
    }
    for (int t = 0; t < nthreads; t++) merge(out, &parts[t]);
    free(parts);
    return WAR_OK;
}

uint64_t oracle_space_size(int n, int mode) { return space_size(n, mode); }
size_t oracle_result_size(void) { return sizeof(war_result); }
