"""war_enumerate_noalloc, the entry point for callers that cannot allocate device memory (a host program
whose memory pool has reserved the GPU, or a latency-bound path that cannot take cudaMalloc's implicit
synchronisation).  Called through the C ABI, it must give exactly what war_enumerate gives and what the
oracle or the reference's recorded outputs say, on two calls in a row (the static scratch keeps the
previous call's contents and must be cleared).  Collected last, and safe alone in a fresh process: its
first call sets the scratch up on the device."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("cyc", "done", "maxfin", "turns", "shape_nonstd", "shape_unchecked", "oncycle", "distinct_min",
          "s_count", "s_cyc", "s_lamsum", "s_lensum", "s_maxfin", "units")
# what the oracle computes too (it has no work units, and counts turns with the reference's schedule)
ORACLE_FIELDS = ("cyc", "done", "maxfin", "shape_nonstd", "shape_unchecked", "oncycle", "distinct_min",
                 "s_count", "s_cyc", "s_lamsum", "s_lensum", "s_maxfin")


def call_noalloc(wl, job, tune=None):
    r = wl.Result()
    st = wl.lib().war_enumerate_noalloc(ctypes.byref(job), ctypes.byref(tune) if tune is not None else None,
                                        ctypes.byref(r))
    assert st == 0, wl.last_error()
    return r


def same(wl, a, b, fields=FIELDS):
    for k in fields:
        assert getattr(a, k) == getattr(b, k), k
    da, db = wl.to_dict(a), wl.to_dict(b)
    for h in ("hist", "dhist", "endhist"):
        assert da[h] == db[h], h


def same_as_oracle(wl, oracle, got, job):
    want = oracle.enumerate_job(oracle.make_job(job.n, job.mode, job.rule, job.flags, job.lo, job.hi, job.hbins,
                                                job.dbins, job.blk, job.sample_ppm, job.seed))
    g, w = wl.to_dict(got), oracle.to_dict(want)
    for k in ORACLE_FIELDS + ("hist", "dhist", "endhist"):
        assert g[k] == w[k], (k, g[k], w[k])


JOBS = [
    dict(n=11, hbins=64),
    dict(n=12, lo=123456789, hi=134567891, hbins=128, flags=8, sample_ppm=20000, seed=5),
    dict(n=10, mode=1, rule=1, flags=2 | 4, hbins=256, dbins=64),
    dict(n=13, lo=3000000000, hi=3005000000, hbins=256),
]


@pytest.mark.parametrize("spec", JOBS)
def test_noalloc_matches_enumerate_and_oracle_twice(wl, oracle, spec):
    job = wl.make_job(**spec)
    first = call_noalloc(wl, job)            # in a fresh process this call also sets the scratch up
    second = call_noalloc(wl, job)           # the scratch still holds the first call's results
    want = wl.enumerate_job(job)
    same(wl, first, want)
    same(wl, second, want)
    same_as_oracle(wl, oracle, first, job)


def test_noalloc_two_launches_all_13_deals(wl, golden):
    """All 13! deals are more games than one launch plays (fewer than 2^32), so the scratch is cleared and
    read back between launches; the memo bits of the tune are ignored (no table without allocation)."""
    job = wl.make_job(13, hbins=256)
    tune = wl.make_tune(variant=30, memo_bits=20, defer=8)
    g = golden["deals_rule0"][13]
    for _ in range(2):
        r = call_noalloc(wl, job, tune)
        d = wl.to_dict(r)
        assert (d["done"], d["cyc"], d["maxfin"], d["hist"]) == (g["deals"], g["cyc"], g["longest"], g["hist"])
        assert sum(d["endhist"].values()) == g["deals"] - g["cyc"] and max(d["endhist"]) == g["longest"]
        assert r.memo_lookups == 0 and r.memo_stores == 0
        assert r.units > 0


def test_noalloc_with_tune_and_refusals(wl, oracle):
    job = wl.make_job(11, hbins=32)
    t = wl.make_tune(games=2, threads=512, block_m=5, defer=8, variant=1)
    want = wl.enumerate_job(job, t)
    same(wl, call_noalloc(wl, job, t), want)
    same(wl, call_noalloc(wl, job, t), want)
    same_as_oracle(wl, oracle, call_noalloc(wl, job, t), job)
    r = wl.Result()
    bad = wl.make_job(11, hbins=5000)
    assert wl.lib().war_enumerate_noalloc(ctypes.byref(bad), None, ctypes.byref(r)) == -1
    # 17-card deals go to the held-out engine in war_enumerate; this entry point refuses them
    n17 = wl.make_job(17, lo=0, hi=1000)
    assert wl.lib().war_enumerate_noalloc(ctypes.byref(n17), None, ctypes.byref(r)) == -1
    assert "n=17" in wl.last_error()
