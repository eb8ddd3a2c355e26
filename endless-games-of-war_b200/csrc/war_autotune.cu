// war_autotune.cu — the autotuner behind the C ABI (war_autotune in include/war.h): coordinate descent
// over the refill kernel's launch shape, record scheme, turn form and memo size for one job class,
// measured with war_enumerate's own CUDA-event kernel time on a slice of the job's range.  Host code
// only; the same search as autotune.py, for callers without Python.  No counterpart in the reference.
#include <algorithm>
#include <cstring>
#include <vector>
#include "war_host.h"

namespace war {
namespace {

struct Dim {
    const char* name;
    int32_t war_tune::*field;
    std::vector<int> values;
};

const std::vector<Dim>& dims() {
    static const std::vector<Dim> d = {
        {"block_m", &war_tune::block_m, {4, 5, 6, 7}},
        {"games", &war_tune::games, {1, 2, 4}},
        {"threads", &war_tune::threads, {128, 256, 512, 1024}},
        {"blocks_per_sm", &war_tune::blocks_per_sm, {0, 1, 2, 3, 4}},
        {"window", &war_tune::window, {8, 16, 32, 64, 128}},
        {"defer", &war_tune::defer, {1, 2, 4, 8, 12, 16, 24, 32}},
        {"variant", &war_tune::variant, {0, 1, 2, 3, 6, 7, 14, 15, 30, 31}},
        {"memo_bits", &war_tune::memo_bits, {24, 26, 28, 30, 31}},
        {"chunk", &war_tune::chunk, {1, 8, 64, 512, 1456}},
    };
    return d;
}

bool legal(const war_job& job, const war_tune& t) {
    const bool canon = job.mode == WAR_CANON;
    if (canon && (job.flags & WAR_F_DISTINCT) && t.window < 128) return false;   // the free on-cycle test
    if (t.games == 2 && t.threads > 512) return false;
    if (t.games == 4 && (t.threads > 256 || (t.variant != 3 && t.variant != 31))) return false;
    return t.block_m <= (canon ? job.n - 1 : job.n);
}

struct Key {
    u64 cyc, done, maxfin, oncycle, distinct_min;
    bool operator==(const Key& o) const {
        return cyc == o.cyc && done == o.done && maxfin == o.maxfin && oncycle == o.oncycle &&
               distinct_min == o.distinct_min;
    }
};

// Best of two runs (kernel ms), and the counts, of tune t on slice s.
int measure(const war_job& s, const war_tune& t, war_result* r, double* ms, Key* key) {
    double best = -1.0;
    for (int rep = 0; rep < 2; rep++) {
        int st = war_enumerate(&s, &t, r);
        if (st) return st;
        if (best < 0 || r->kernel_ms < best) best = r->kernel_ms;
    }
    *ms = best;
    *key = Key{r->cyc, r->done, r->maxfin, r->oncycle, r->distinct_min};
    return WAR_OK;
}

}  // namespace
}  // namespace war

using namespace war;

extern "C" int war_autotune(const war_job* job, const war_tune* start, double slice_ms, int32_t passes,
                            war_tune* best, double* best_ms) {
    int st = check_job(job);
    if (st) return st;
    if (!best) return fail(WAR_EINVAL, "best is NULL");
    if (passes < 1 || passes > 8) return fail(WAR_EINVAL, "passes=%d (1..8)", passes);
    if (job->lo == job->hi) return fail(WAR_EINVAL, "empty rank range");
    if (!(slice_ms > 0)) slice_ms = 400.0;
    std::vector<war_result> buf(1);   // ~140 KB: on the heap
    war_result* r = buf.data();
    war_tune cur;
    memset(&cur, 0, sizeof cur);
    if (start) {
        cur = *start;
    } else {
        cur.block_m = 5; cur.games = 1; cur.threads = 256; cur.window = job->mode == WAR_CANON ? 128 : 32;
        cur.defer = 8; cur.variant = 3; cur.memo_bits = 0;
    }
    // a slice from the middle of the range, grown until its kernel time is long enough to measure, then
    // sized to slice_ms
    war_job s = *job;
    s.flags &= ~(int32_t)WAR_F_MEMO_KEEP;
    const u64 span = job->hi - job->lo;
    u64 size = std::min<u64>(span, 1ull << 24);
    for (;;) {
        s.lo = job->lo + (span - size) / 2;
        s.hi = s.lo + size;
        if ((st = war_enumerate(&s, &cur, r))) return st;
        if (r->kernel_ms >= 50.0 || size >= span) break;
        size = std::min<u64>(span, size * 4);
    }
    const double rate = (double)size / std::max(r->kernel_ms, 1e-3);
    size = std::min<u64>(span, std::max<u64>(1, (u64)(rate * slice_ms)));
    s.lo = job->lo + (span - size) / 2;
    s.hi = s.lo + size;
    double cur_ms;
    Key ref;
    if ((st = measure(s, cur, r, &cur_ms, &ref))) return st;
    for (int p = 0; p < passes; p++) {
        bool improved = false;
        for (const Dim& d : dims()) {
            for (int v : d.values) {
                if (cur.*(d.field) == v) continue;
                war_tune t = cur;
                t.*(d.field) = v;
                if (!legal(*job, t)) continue;
                double ms;
                Key k;
                const int e = measure(s, t, r, &ms, &k);
                if (e == WAR_EINVAL) continue;   // a shape that does not fit this GPU
                if (e) return e;
                if (!(k == ref))
                    return fail(WAR_EINVAL, "tune %s=%d changed the counts of the slice: the engine is wrong", d.name, v);
                if (ms < cur_ms * 0.995) { cur = t; cur_ms = ms; improved = true; }
            }
        }
        if (!improved) break;
    }
    *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return WAR_OK;
}
