"""war_enumerate_noalloc, the entry point for callers that cannot allocate device memory (a host program
whose memory pool has reserved the GPU, or a latency-bound path that cannot take cudaMalloc's implicit
synchronisation).  Called through the C ABI, it must give exactly what war_enumerate gives, on two calls
in a row (the static scratch keeps the previous call's contents and must be cleared).  Collected last, and
safe alone in a fresh process: its first call sets the scratch up on the device."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("cyc", "done", "maxfin", "turns", "shape_nonstd", "shape_unchecked", "oncycle", "distinct_min",
          "s_count", "s_cyc", "s_lamsum", "s_lensum", "s_maxfin", "units")


def call_noalloc(wl, job, tune=None):
    r = wl.Result()
    st = wl.lib().war_enumerate_noalloc(ctypes.byref(job), ctypes.byref(tune) if tune is not None else None,
                                        ctypes.byref(r))
    assert st == 0, wl.last_error()
    return r


def same(wl, a, b):
    for k in FIELDS:
        assert getattr(a, k) == getattr(b, k), k
    da, db = wl.to_dict(a), wl.to_dict(b)
    for h in ("hist", "dhist", "endhist"):
        assert da[h] == db[h], h


JOBS = [
    dict(n=11, hbins=64),
    dict(n=12, lo=123456789, hi=234567891, hbins=128, flags=8, sample_ppm=20000, seed=5),
    dict(n=10, mode=1, rule=1, flags=2 | 4, hbins=256, dbins=64),
    dict(n=13, lo=3000000000, hi=3050000000, hbins=256),
]


@pytest.mark.parametrize("spec", JOBS)
def test_noalloc_matches_enumerate_twice(wl, spec):
    job = wl.make_job(**spec)
    first = call_noalloc(wl, job)            # in a fresh process this call also sets the scratch up
    second = call_noalloc(wl, job)           # the scratch still holds the first call's results
    want = wl.enumerate_job(job)
    same(wl, first, want)
    same(wl, second, want)


def test_noalloc_with_tune_and_refusal(wl):
    job = wl.make_job(11, hbins=32)
    t = wl.make_tune(games=2, threads=512, block_m=5, defer=8, variant=1)
    want = wl.enumerate_job(job, t)
    same(wl, call_noalloc(wl, job, t), want)
    same(wl, call_noalloc(wl, job, t), want)
    bad = wl.make_job(11, hbins=5000)
    r = wl.Result()
    assert wl.lib().war_enumerate_noalloc(ctypes.byref(bad), None, ctypes.byref(r)) == -1
