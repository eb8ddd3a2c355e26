/* war.h — C ABI of libwar.so, the sm_100a engine that enumerates single-suit War deals and
 * canonical positions and counts the games that never end.
 *
 * The reference (OrygnsCode/endless-games-of-war) has no FFI: its hot path gpu/war_gpu.py keeps
 * the CUDA source in a string, compiles it with NVRTC through CuPy and launches the kernels
 * war_count / war_canon from Python (gpu/war_gpu.py:262-269, :309-328).  Each entry point below
 * says which part of that path it replaces.  Plain C types only: pointers, sizes, fixed-width
 * integers.  Every function returns a war_status (0 = ok, < 0 = error; the message is kept for
 * war_last_error).  Errors never abort the process.
 *
 * Ownership: callers own every host struct they pass (results included); the library owns all
 * device memory.  Threading: calls that launch work are serialised by an internal lock; a server
 * (war_server_*) runs its own host thread.
 *
 * Card values are 0..n-1 (0 lowest), deck position 0,2,4,.. goes to player 1 and 1,3,5,.. to
 * player 2, the first card dealt on top, as in gpu/war_gpu.py:3-5.  1 <= n <= 16 (deals: 17, see
 * war_enumerate_held).
 */
#ifndef WAR_B200_WAR_H
#define WAR_B200_WAR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WAR_MAX_N 16
#define WAR_HBINS_MAX 4096 /* cycle-length histogram bins (last bin = overflow), gpu/war_gpu.py:364 */
#define WAR_DBINS_MAX 4096 /* distinct-cycle weight bins, gpu/war_gpu.py:379 uses 4096 */
#define WAR_EBINS 1024     /* ending-game-length histogram bins (last bin = overflow) */

enum war_status {
    WAR_OK = 0,
    WAR_EINVAL = -1,   /* bad argument */
    WAR_ECUDA = -2,    /* CUDA runtime error (message in war_last_error) */
    WAR_ETIMEOUT = -3, /* a bounded wait ran out */
    WAR_ENOMEM = -4,   /* device or host memory exhausted / admission refused */
    WAR_EBUSY = -5,    /* server queue full */
    WAR_ENOTFOUND = -6,/* unknown job id */
    WAR_ECAP = -7,     /* a game exceeded the per-lane turn cap (never expected: Brent terminates) */
    WAR_ENODEV = -8,   /* no CUDA device */
    WAR_PENDING = 1    /* war_server_poll: job not finished yet */
};

enum war_mode { WAR_DEALS = 0, WAR_CANON = 1 };

enum war_flags {
    WAR_F_HALF = 1,     /* even n, deals: play only deals that give card n-1 to player 1 (gpu/war_gpu.py:147-154) */
    WAR_F_DISTINCT = 2, /* canon: distinct-cycle weights + min-key count (gpu/war_gpu.py:217-235, cpu/distinct_cycles.c:67-80) */
    WAR_F_SHAPE = 4,    /* canon: Theorem-3 loop-shape test, blk = n & -n (gpu/war_gpu.py:51-73, :290) */
    WAR_F_SAMPLE = 8,   /* accumulate the seeded sample aggregates used by the Floyd cross-check */
    WAR_F_MEMO_KEEP = 16 /* jobs with the cycle memo (war_tune.variant bit 2): start from the memo left by the
                            previous war_enumerate of the same n and rule instead of an empty one (its entries
                            are facts about n and the rule, not about the range); no other effect (no
                            reference counterpart) */
};

/* One enumeration job: the ranks [lo, hi) of one space.
 *  mode WAR_DEALS: rank r = lexicographic rank of the deck order (0 <= r < n!).
 *  mode WAR_CANON: rank r = perm_rank * (n-1) + k, where perm_rank is the lexicographic rank of the
 *  order q of the cards 0..n-2 and k in 0..n-2 is the split: player 1 = [n-1, q0..q(k-1)],
 *  player 2 = [qk..q(n-2)] (gpu/war_gpu.py:178-182, :208-213). */
typedef struct war_job {
    int32_t n;
    int32_t mode;      /* war_mode */
    int32_t rule;      /* 0 = winner's card first (Spivey), 1 = loser's card first (gpu/war_gpu.py:367-368) */
    int32_t flags;     /* war_flags */
    int32_t hbins;     /* 0..WAR_HBINS_MAX: cycle-length histogram bins, 0 = off */
    int32_t dbins;     /* 0..WAR_DBINS_MAX: distinct weight bins (canon + WAR_F_DISTINCT) */
    int32_t blk;       /* shape block length; 0 = n & -n (only with WAR_F_SHAPE) */
    uint32_t sample_ppm; /* sample rate for WAR_F_SAMPLE, parts per million */
    uint64_t lo, hi;   /* rank range */
    uint64_t seed;     /* sample seed */
} war_job;

/* Launch shape of the persistent refill kernel (war_enumerate).  Zero fields take defaults. */
typedef struct war_tune {
    int32_t threads;       /* threads per block (multiple of 32, 64..1024) */
    int32_t blocks_per_sm; /* resident blocks per SM for the persistent grid */
    int32_t games;         /* games in flight per thread: 1, 2, or 4 (4: variants 3 and 31 only, at most 256 threads) */
    int32_t block_m;       /* each work unit covers m! consecutive ranks (deals) or m! orders x splits (canon); 1..8 */
    int32_t window;        /* Brent first tortoise window (power of two); 1 = the reference's schedule */
    int32_t defer;         /* immediate records: lanes that wait, decided, before the warp refills them (1..32);
                              latched records: iterations between services (rounded up to a multiple of 4) */
    int32_t variant;       /* bit 0: multiply-add turn form (else logic/shift).
                              bit 1: outcomes latched and recorded every `defer` iterations (else at once).
                              bit 2 (needs bit 1 and n >= 4): the cycle memo, a table of facts "from this
                              state the game cycles with length L / ends after r turns" filled by the job's
                              own games; a game is decided at the first state it finds there (`turns` then
                              counts the turns played, fewer than the reference's schedule).  Alone: the
                              memo holds cycle landmarks kept per turn (n <= 15).  With bit 3: every state
                              of each found cycle, games looked up at their current state (n <= 14).  With
                              bits 3 and 4 (the "path memo"): also the states where decided games missed,
                              with their outcome (n <= 16; canonical scans take only this form).
                              Every form gives the same results; out-of-range forms fall back to none. */
    int32_t memo_bits;     /* cycle memo: log2 of its 8-byte slots (12..31); 0 = 24 (128 MiB) */
    int32_t chunk;         /* work units a lane takes from the work counter at a time (1..4096; 0 = 1): each lane
                              walks chunks of chunk x block_m! consecutive ranks (deals) */
} war_tune;

/* Aggregates of one job.  Matches what gpu/war_gpu.py run() returns (gpu/war_gpu.py:346-352) before
 * its --half doubling, plus the fields the reference does not have (turns, ending-length histogram,
 * min-key distinct count, sample aggregates). */
typedef struct war_result {
    uint64_t cyc;            /* games that never end */
    uint64_t done;           /* games played (deals or positions) */
    uint64_t maxfin;         /* longest game that ends, in turns */
    uint64_t turns;          /* turns executed by the cycle search (plain kernel: the reference's Brent schedule) */
    uint64_t shape_nonstd;   /* cycling positions whose loop is not of Theorem-3 shape */
    uint64_t shape_unchecked;/* cycling positions whose loop is longer than 512 */
    uint64_t oncycle;        /* canonical positions that lie on their own cycle */
    uint64_t distinct_min;   /* positions that are the minimum canonical state of their cycle (= distinct cycles) */
    uint64_t s_count, s_cyc, s_lamsum, s_lensum, s_maxfin; /* sample aggregates (WAR_F_SAMPLE) */
    uint64_t units;          /* work units processed (diagnostic) */
    uint64_t memo_lookups, memo_hits, memo_stores; /* cycle memo traffic (war_tune.variant bit 2; diagnostic) */
    uint64_t undetermined;   /* war_enumerate_wide: games still undecided at the step cap (gpu/war24.py:57, :103, :117) */
    double kernel_ms;        /* device time of the enumeration kernel(s), CUDA events */
    int32_t hbins, dbins, blk, status;
    uint64_t hist[WAR_HBINS_MAX];
    uint64_t dhist[WAR_DBINS_MAX];
    uint64_t endhist[WAR_EBINS];
} war_result;

/* ---- plain kernels: the reference's launches, restated for sm_100a -------------------------- */

/* Replaces one CuPy launch of the reference kernel war_count (gpu/war_gpu.py:121-124, launched at
 * :316-326): threads t = 0..nthreads-1 each take `per` consecutive ranks from start + t*per (clipped
 * to total), in lexicographic order.  half_rule = half | rule << 1 as at :324.  The accumulators are
 * HOST arrays that are added to, like the reference's device arrays (cyc, done, maxfin are 1 word,
 * hist has hbins words).  Blocks of `threads` threads; the call returns after the launch finished. */
int war_count_launch(int32_t n, uint64_t start, uint64_t total, int32_t per, int32_t half_rule,
                     int32_t threads, uint64_t nthreads, uint64_t* cyc, uint64_t* done,
                     uint64_t* maxfin, uint64_t* hist, int32_t hbins);

/* Replaces one CuPy launch of war_canon (gpu/war_gpu.py:183-186, launched at :318-326).  Ranks are
 * orders of the n-1 other cards (n-1 positions each).  shape has 2 words, dhist dbins words. */
int war_canon_launch(int32_t n, uint64_t start, uint64_t total, int32_t per, int32_t blk,
                     int32_t threads, uint64_t nthreads, uint64_t* cyc, uint64_t* done,
                     uint64_t* maxfin, uint64_t* hist, int32_t hbins, uint64_t* shape,
                     int32_t rule, uint64_t* dhist, int32_t dbins);

/* The plain kernel over a whole job with the full result (turns, ending-length histogram, min-key
 * count, sample aggregates).  Same per-thread rank blocks as war_count_launch (per = 256, 256
 * threads, spans of 2^18 threads; canon spans divided by n-1 as at gpu/war_gpu.py:276-277). */
int war_enumerate_plain(const war_job* job, war_result* out);

/* ---- batched persistent kernel --------------------------------------------------------------- */

/* Replaces run()'s launch loop (gpu/war_gpu.py:309-328) with one persistent launch: a grid of
 * SMs x blocks_per_sm blocks pulls work units from a global atomic counter, and every lane refills
 * with the next deal or position as soon as its game is decided.  tune may be NULL (defaults). */
int war_enumerate(const war_job* job, const war_tune* tune, war_result* out);

/* war_enumerate for callers that cannot allocate device memory: a host program whose own memory pool
 * has reserved the GPU (a cudaMalloc would fail or fragment it), or code on a latency-bound path that
 * cannot take cudaMalloc's implicit synchronisation.  No counterpart in the reference.  Same refill
 * kernel, arguments and results as war_enumerate for jobs of 1..16 cards (kernel_ms is host wall time
 * here), with two differences: 17-card deals, which war_enumerate hands to the held-out engine, are
 * refused with WAR_EINVAL, and the cycle memo is never used (tune.variant bits 2-4 are ignored, so
 * memo_lookups stays 0), because its table would be allocated memory.  The scratch (one job's
 * accumulators and work counter, and at most 1024 extra work units; about 98 KB) lives in a static
 * device array that every GPU loading the library holds until exit; jobs whose plan needs more extra
 * units are refused with WAR_EINVAL.  The first call on each device looks up that array's address
 * (cudaGetSymbolAddress) and should come before any stream capture.  It calls no cudaMalloc / cudaFree
 * and creates no stream or event.  All calls share the array: each clears it before use, and calls
 * whose work overlaps on the GPU race. */
int war_enumerate_noalloc(const war_job* job, const war_tune* tune, war_result* out);

/* Floyd cross-check (the second detector of gpu/war_gpu_floyd.py:95-105 and cpu/war_floyd.c:14-63): plays,
 * with Floyd's tortoise and hare, every position of the job whose seeded hash falls in the sample, and
 * fills the s_* fields of out (the rest is zero).  They must equal the s_* fields of war_enumerate /
 * war_enumerate_plain run with WAR_F_SAMPLE on the same job.  sample_ppm = 1000000 plays every position of
 * the job (the full-range check: s_count = positions, s_cyc = cycling, s_maxfin = longest ending game),
 * enumerated by its own lexicographic unrank and next-permutation. */
int war_floyd_sample(const war_job* job, war_result* out);

/* ---- serving: continuous batching of enumeration jobs (no reference counterpart) ----------- */

typedef struct war_server war_server;

typedef struct war_server_cfg {
    int32_t max_jobs;        /* resident job slots (accumulator sets kept on the device) */
    int32_t queue_cap;       /* pending jobs the submit queue holds before WAR_EBUSY */
    uint64_t mem_budget;     /* bytes of device memory the server may hold for job accumulators and cycle
                                memos; 0 = free memory / 2.  The accumulator slots come first (max_jobs of
                                them, or as many as fit); what is left, up to 16 GiB, is reserved at create
                                as the memo arena, from which each job class takes its table when its first
                                job is admitted (nothing is allocated after create) */
    uint64_t tick_ranks;     /* ranks issued per tick across all jobs (0 = default) */
    int32_t threads, blocks_per_sm;
    int32_t memo_bits;       /* cycle memo shared by all jobs of one n and rule, log2 of its 8-byte words
                                (grown with n up to this, shrunk to what the arena has left; 0 = 28, i.e.
                                2 GiB per class; < 0 = no memo).  A class whose table does not fit runs
                                without the memo, with the same results */
    int32_t reserved[3];
} war_server_cfg;

typedef struct war_job_status {
    int32_t state;           /* 0 queued, 1 running, 2 done, 3 failed */
    int32_t status;          /* war_status of a failed job */
    double submit_ms, admit_ms, finish_ms; /* host clock (ms since the server started) */
} war_job_status;

/* Deals of 2..17 cards with the held-out-card engine (gpu/war17.py:7-16, :36-71): card n-1 never loses,
 * so it is kept out of the packed piles and tracked by its depth in its holder's pile; that keeps 17
 * cards in 4-bit nibbles.  Same job and result as war_enumerate for deals (cycling count, longest ending
 * game, cycle-length and ending-length histograms, turns), both rules; only WAR_F_MEMO_KEEP applies.
 * tune: threads (0 = 512, 256 with the memo), blocks_per_sm, block_m (0 = 6), window (0 = 32), defer
 * (turns between services, 0 = 32, 16 with the memo); variant bits 0-1 pick the turn, all with the same
 * results: 0 = the two counts packed in one word with multiply-add card arithmetic (the default and the
 * fastest), 1 = multiply-adds on separate counts, 2 = packed counts in logic/shift form, 3 = the plain
 * branching turn of gpu/war17.py; bit 2 = the path memo with memo_bits (0 = 28), at most 512 threads then;
 * bit 3 = test Brent's checkpoint after every turn (by default it is saved at the services whenever the
 * window is a multiple of the service period).  NULL = defaults (no memo).  war_enumerate sends n = 17 deal
 * jobs here. */
int war_enumerate_held(const war_job* job, const war_tune* tune, war_result* out);

/* The 5-bit-pile engine (gpu/war24.py): deals of 2..20 cards (deal ranks are 64-bit), cards of 5 bits in
 * 128-bit piles.  det picks the cycle test: WAR_DET_BRENT (tortoise saved at turns W, 3W, 7W, ...; the only
 * one that measures cycle lengths for job.hbins), WAR_DET_FLOYD (gpu/war24.py:85-97) or WAR_DET_STREAK (odd n
 * and rule 0 only: the players alternate for lcm(n+1, W, L-1) turns from an anchor, gpu/war24.py:98-125).  A
 * game still undecided after `cap` turns counts in war_result.undetermined instead of cyc or the ending
 * counts (gpu/war24.py:57).  All zero fields take defaults. */
enum war_det { WAR_DET_BRENT = 0, WAR_DET_FLOYD = 1, WAR_DET_STREAK = 2 };
typedef struct war_wide_cfg {
    int32_t det;           /* war_det */
    uint32_t cap;          /* step cap in turns (1..2^30; 0 = 2^22, gpu/war24.py:57) */
    int32_t threads, blocks_per_sm, block_m, window, defer;   /* as in war_tune (defer: turns between services) */
    int32_t reserved;
} war_wide_cfg;

/* Deals [lo, hi) of job.n = 2..20 cards with the 5-bit-pile engine: cyc, done, maxfin, turns (turns played by
 * the detector), undetermined, endhist and (Brent) hist.  Only rule and hbins of the job apply (flags must be
 * 0 or WAR_F_MEMO_KEEP, which has no effect).  Replaces the launch loop of gpu/war24.py:186-201. */
int war_enumerate_wide(const war_job* job, const war_wide_cfg* cfg, war_result* out);

/* Coordinate descent over war_tune for the class of `job` (block_m, games, threads, blocks per SM, window,
 * defer, variant, memo_bits), timed by war_enumerate's kernel time on a slice of job's range from its
 * middle, sized to take about slice_ms (0 = 400 ms); starts from *start (NULL = the library defaults) and
 * makes at most `passes` passes (1..8).  Every configuration tried must return the first one's counts,
 * else WAR_EINVAL.  The memo variants only pay on long slices (a memo is cleared per job).  The search of
 * endless-games-of-war_b200/autotune.py, callable without Python; no counterpart in the reference. */
int war_autotune(const war_job* job, const war_tune* start, double slice_ms, int32_t passes, war_tune* best,
                 double* best_ms);

int war_server_create(const war_server_cfg* cfg, war_server** out);
/* Queue a job; *id receives its id.  Returns WAR_EBUSY when the queue is full, WAR_EINVAL for a bad job. */
int war_server_submit(war_server* s, const war_job* job, uint64_t* id);
/* WAR_PENDING while the job is queued or running; WAR_OK and *res filled once it is done (the job
 * is then forgotten); st (may be NULL) gets its timestamps. */
int war_server_poll(war_server* s, uint64_t id, war_result* res, war_job_status* st);
/* Waits (bounded by timeout_ms) until every submitted job is done. */
int war_server_drain(war_server* s, double timeout_ms);
int war_server_stats(war_server* s, uint64_t* ticks, uint64_t* jobs_done, uint64_t* peak_resident);
/* The memo arena reserved at create (bytes), the part of it the job classes took so far, and how many
 * classes have a table. */
int war_server_memo_info(war_server* s, uint64_t* arena_bytes, uint64_t* used_bytes, int32_t* classes);
int war_server_destroy(war_server* s);

/* ---- utilities --------------------------------------------------------------------------------- */

/* A work unit of war_enumerate: the orders r .. r + j! - 1 of the permuted cards (r a multiple of j!),
 * with the canonical split restricted to k0 <= k < k1 (deals: k0 = k1 = 0). */
typedef struct war_unit { uint64_t r; uint32_t j, k0, k1, pad; } war_unit;

/* The plan war_enumerate runs for a job (host only, no device needed): main units are the orders
 * [(main_base + u) * block_m!, + block_m!) for u < main_count; the extra units cover the rest of the
 * range.  Returns the number of extra units (written to extra up to cap) or < 0.  No reference
 * counterpart: the reference tiles ranks in spans of batch_threads * per (gpu/war_gpu.py:310-328). */
int war_plan(const war_job* job, int32_t block_m, uint64_t* main_base, uint64_t* main_count, war_unit* extra,
             int32_t cap);

typedef struct war_device_info {
    int32_t device, sm_count, cc_major, cc_minor, clock_mhz, max_threads_per_sm;
    uint64_t mem_free, mem_total;
    char name[128];
} war_device_info;

int war_device_info_get(war_device_info* info);
/* Launch subsequent work on this cudaStream_t (NULL = the library's own stream). */
int war_set_stream(void* cuda_stream);
/* Measures 32-bit integer instruction throughput (thread-instructions per second): issue = LOP3 and
 * IMAD alternating (ALU and FMA pipes, the issue-slot ceiling), alu = LOP3 only (the ALU pipe).  The
 * denominator of the roofline of the integer-bound enumeration kernels.  No reference counterpart. */
int war_measure_int_peak(double* issue_ops_per_s, double* alu_ops_per_s);
/* Measures random-gather throughput (lookups per second): independent loads of one 8-byte word
 * (bucket_bytes = 8) or one aligned 32-byte bucket (32) at uniformly random positions of a table of
 * 2^table_bits words (20..31; the cycle memo's table when it has that size, else one allocated for the
 * call), eight in flight per thread.  The ceiling of the cycle memo's lookups, which are such loads.  No
 * reference counterpart. */
int war_measure_gather_peak(int32_t table_bits, int32_t bucket_bytes, double* lookups_per_s);
/* Copies the last error message of the calling thread; returns its length. */
int war_last_error(char* buf, size_t len);
/* Kernels this library launched since load (its own kernels only). */
uint64_t war_launch_count(void);
/* Sample predicate shared by every kernel: 1 if the starting position is in the seeded sample.
 * w1s / w2s are the piles packed 4 bits per card, top card in the low nibble, with a 1 bit just
 * above the last card (w | 1 << 4*len).  x = seed ^ w1s*0x9E3779B97F4A7C15 ^ w2s*0xC2B2AE3D27D4EB4F,
 * then the splitmix64 finaliser; picked iff (x >> 32) < ppm * 2^32 / 10^6. */
int war_sample_pick(uint64_t seed, uint32_t ppm, uint64_t w1s, uint64_t w2s);

#ifdef __cplusplus
}
#endif
#endif
