"""The 5-bit-pile engine (war_enumerate_wide, gpu/war24.py) against the oracle's restatement of gpu/war24.py,
the reference's recorded war24.py runs (data/checks.txt:73-79, data/long_runs.txt:62-75), the 4-bit engine and
the held-out-card engine.  Every count is exact, so every comparison is equality."""
import contextlib
import io
import re

import pytest

pytestmark = pytest.mark.gpu

KEYS = ("cyc", "done", "maxfin", "undetermined", "turns", "endhist")


def ojob(oracle, job):
    return oracle.make_job(job.n, 0, job.rule, 0, job.lo, job.hi, job.hbins)


def same(wl, oracle, got, want, keys=KEYS):
    g, w = wl.to_dict(got), oracle.to_dict(want)
    for k in keys:
        assert g[k] == w[k], (k, g[k], w[k])


@pytest.mark.parametrize("rule", [0, 1])
def test_all_small_n_against_the_oracle(wl, oracle, rule):
    """Every deal of n = 2..11 with each detector: counts, turns played and ending lengths equal the oracle's;
    Brent's cycle-length histogram too (first window W = 32, the oracle with the same window)."""
    for n in range(2, 12):
        job = wl.make_job(n, rule=rule, hbins=256)
        same(wl, oracle, wl.enumerate_wide(job, wl.DET_BRENT), oracle.war24(ojob(oracle, job), oracle.DET_BRENT, 32),
             KEYS + ("hist",))
        same(wl, oracle, wl.enumerate_wide(job, wl.DET_FLOYD), oracle.war24(ojob(oracle, job), oracle.DET_FLOYD))
        if n % 2 and not rule:
            same(wl, oracle, wl.enumerate_wide(job, wl.DET_STREAK),
                 oracle.war24(ojob(oracle, job), oracle.DET_STREAK))


@pytest.mark.parametrize("det", [0, 1, 2])
def test_step_cap_and_launch_shapes(wl, oracle, det):
    """A step cap below the games' lengths: the same games are undetermined as in the oracle; and the counts do
    not depend on the launch shape (threads, blocks, unit size, service period, window)."""
    job = wl.make_job(11, lo=1234567, hi=9876543, hbins=64)
    want = oracle.war24(ojob(oracle, job), det, 32, 24)
    got = wl.enumerate_wide(job, det, cap=24)
    assert got.undetermined > 0
    same(wl, oracle, got, want)
    base = wl.enumerate_wide(job, det)
    for kw in (dict(threads=128), dict(threads=1024, block_m=8), dict(block_m=1), dict(blocks_per_sm=1),
               dict(defer=4), dict(defer=64, block_m=3)):
        r = wl.enumerate_wide(job, det, **kw)
        assert (r.cyc, r.done, r.maxfin, r.turns, r.undetermined) == \
            (base.cyc, base.done, base.maxfin, base.turns, base.undetermined), kw
    if det == 0:
        same(wl, oracle, wl.enumerate_wide(job, det, window=1), oracle.war24(ojob(oracle, job), det, 1),
             KEYS + ("hist",))


def test_recorded_war24_runs(wl, golden):
    """The reference's war24.py runs that take seconds here: a(12) with Floyd, a(13) with the streak test, and
    the three 17-card slices (1e9 deals from 10^14 with both tests, the first 8,992,587,776 deals, the last
    785,219,584)."""
    seen = 0
    for e in golden["war24"]:
        if e["n"] < 12 or e["hi"] - e["lo"] > 10 ** 10:      # the CPU tests cover n < 12; no hours-long runs
            continue
        det = wl.DET_STREAK if e["det"] == "streak" else wl.DET_FLOYD
        r = wl.enumerate_wide(wl.make_job(e["n"], lo=e["lo"], hi=e["hi"]), det)
        assert (r.done, r.cyc, r.maxfin, r.undetermined) == (e["deals"], e["cyc"], e["longest"], e["undetermined"]), e
        seen += 1
    assert seen == 6


def test_agrees_with_the_4bit_and_held_out_engines(wl):
    """n = 14 and n = 16 slices against the 4-bit engine (histograms included), a 17-card slice against the
    held-out-card engine, with both rules."""
    for n, lo, hi, rule in ((14, 3 * 10 ** 10, 3 * 10 ** 10 + 2 * 10 ** 8, 0), (14, 5 * 10 ** 9, 5 * 10 ** 9 + 10 ** 8, 1),
                            (16, 10 ** 13, 10 ** 13 + 10 ** 8, 0)):
        job = wl.make_job(n, rule=rule, lo=lo, hi=hi, hbins=256)
        a, b = wl.to_dict(wl.enumerate_wide(job)), wl.to_dict(wl.enumerate_job(job))
        for k in ("cyc", "done", "maxfin", "hist", "endhist"):
            assert a[k] == b[k], (n, k)
    for rule in (0, 1):
        job = wl.make_job(17, rule=rule, lo=2 * 10 ** 14, hi=2 * 10 ** 14 + 2 * 10 ** 8, hbins=256)
        a, b = wl.to_dict(wl.enumerate_wide(job)), wl.to_dict(wl.enumerate_held(job))
        for k in ("cyc", "done", "maxfin", "hist", "endhist"):
            assert a[k] == b[k], (rule, k)


@pytest.mark.parametrize("n", [18, 19, 20])
def test_beyond_17_cards(wl, oracle, n):
    """Where no other engine reaches: slices of 18, 19 and 20 cards equal the oracle's restatement of gpu/war24.py
    under every detector (the streak test for odd n), and the detectors agree with one another on a larger slice."""
    from math import factorial
    lo = factorial(n) // 3
    small = wl.make_job(n, lo=lo, hi=lo + 200000, hbins=512)
    same(wl, oracle, wl.enumerate_wide(small, wl.DET_BRENT), oracle.war24(ojob(oracle, small), oracle.DET_BRENT, 32),
         KEYS + ("hist",))
    same(wl, oracle, wl.enumerate_wide(small, wl.DET_FLOYD), oracle.war24(ojob(oracle, small), oracle.DET_FLOYD))
    if n % 2:
        same(wl, oracle, wl.enumerate_wide(small, wl.DET_STREAK), oracle.war24(ojob(oracle, small), oracle.DET_STREAK))
    big = wl.make_job(n, lo=lo, hi=lo + 5 * 10 ** 7)
    rs = [wl.enumerate_wide(big, d) for d in ((0, 1, 2) if n % 2 else (0, 1))]
    assert len({(r.cyc, r.done, r.maxfin, r.undetermined) for r in rs}) == 1


def test_dropin_line(wl, golden, tmp_path):
    """`war24.py 13 --det streak` on the engine prints the recorded line (data/checks.txt:77) apart from the time."""
    import war24
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        war24.main(["13", "--dir", str(tmp_path)])
    tm = re.compile(r" time=[0-9.]+s")
    want = next(e for e in golden["war24"] if e["n"] == 13)
    assert tm.sub("", buf.getvalue().strip()) == tm.sub("", want["line"])
