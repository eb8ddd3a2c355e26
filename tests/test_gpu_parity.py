"""Parity of the sm_100a kernels with the oracle and with the reference's recorded outputs.  Every count
is exact, so every comparison is equality."""
import math
import random

import pytest

pytestmark = pytest.mark.gpu

CMP = ("cyc", "done", "maxfin", "shape_nonstd", "shape_unchecked", "oncycle", "distinct_min",
       "s_count", "s_cyc", "s_lamsum", "s_lensum", "s_maxfin")


def same(wl, oracle, got, want, turns=False):
    g, w = wl.to_dict(got), oracle.to_dict(want)
    for k in CMP + (("turns",) if turns else ()):
        assert g[k] == w[k], (k, g[k], w[k])
    for h in ("hist", "dhist", "endhist"):
        assert g[h] == w[h], h


def ojob(oracle, job):
    return oracle.make_job(job.n, job.mode, job.rule, job.flags, job.lo, job.hi, job.hbins, job.dbins, job.blk,
                           job.sample_ppm, job.seed)


@pytest.mark.parametrize("rule", [0, 1])
def test_deals_all_small_n(wl, oracle, rule):
    for n in range(1, 12):
        job = wl.make_job(n, rule=rule, hbins=256, flags=wl.F_SAMPLE, sample_ppm=20000, seed=7)
        want = oracle.enumerate_job(ojob(oracle, job))
        same(wl, oracle, wl.enumerate_plain(job), want, turns=True)
        same(wl, oracle, wl.enumerate_job(job), want)


@pytest.mark.parametrize("rule", [0, 1])
def test_canon_all_small_n(wl, oracle, rule):
    F = wl.F_DISTINCT | wl.F_SHAPE | wl.F_SAMPLE
    for n in range(2, 11):
        job = wl.make_job(n, wl.CANON, rule=rule, flags=F, hbins=512, dbins=4096, sample_ppm=30000, seed=3)
        want = oracle.enumerate_job(ojob(oracle, job))
        same(wl, oracle, wl.enumerate_plain(job), want, turns=True)
        same(wl, oracle, wl.enumerate_job(job), want)


def test_half_and_ref_launch_geometry(wl, oracle, golden):
    job = wl.make_job(10, flags=wl.F_HALF, hbins=128)
    want = oracle.enumerate_job(ojob(oracle, job))
    same(wl, oracle, wl.enumerate_job(job), want)
    same(wl, oracle, wl.enumerate_plain(job), want, turns=True)
    # war_count_launch with gpu/war_gpu.py's launch loop (per 256, 256 threads, 2^18 threads per launch)
    for n in (9, 10, 11):
        total, per, bt = math.factorial(n), 256, 1 << 18
        acc, hist = [0, 0, 0], [0] * 256
        start = 0
        while start < total:
            nth = min(bt, (total - start + per - 1) // per)
            wl.count_launch(n, start, total, per, 0, 256, nth, acc, hist)
            start += bt * per
        g = golden["deals_rule0"][n]
        assert acc == [g["cyc"], g["deals"], g["longest"]]
        assert {i: v for i, v in enumerate(hist) if v} == g["hist"]


@pytest.mark.parametrize("mode", [0, 1])
def test_random_ranges(wl, oracle, mode):
    rnd = random.Random(99 + mode)
    F = (wl.F_DISTINCT | wl.F_SHAPE) if mode else 0
    for n in (9, 10, 11):
        total = wl.space_size(n, mode)
        for _ in range(4):
            lo = rnd.randrange(0, total)
            hi = min(total, lo + rnd.choice([1, 7, 1000, 123457, 5000000]))
            job = wl.make_job(n, mode, rule=rnd.randint(0, 1), flags=F, lo=lo, hi=hi, hbins=128, dbins=256)
            want = oracle.enumerate_job(ojob(oracle, job))
            same(wl, oracle, wl.enumerate_job(job), want)
            same(wl, oracle, wl.enumerate_plain(job), want, turns=True)


@pytest.mark.parametrize("tune", [dict(games=2), dict(threads=128), dict(threads=1024), dict(block_m=1),
                                  dict(block_m=3), dict(block_m=8), dict(window=64), dict(window=256),
                                  dict(blocks_per_sm=1), dict(games=2, threads=512, block_m=7, window=32),
                                  dict(defer=4), dict(defer=32), dict(variant=1), dict(variant=1, games=2, defer=3),
                                  dict(variant=1, window=1, threads=128), dict(variant=2), dict(variant=3, games=2, defer=16),
                                  dict(variant=3, defer=4, threads=1024), dict(variant=2, window=1, defer=32, games=2),
                                  dict(variant=7, games=2, defer=8), dict(variant=6, threads=128, defer=4),
                                  dict(variant=7, window=1, memo_bits=12, defer=32), dict(variant=15, games=1, defer=16),
                                  dict(variant=14, games=2, threads=512, memo_bits=14), dict(variant=31, games=1, defer=16),
                                  dict(variant=30, games=2, memo_bits=13, defer=4),
                                  dict(variant=31, games=4, threads=256, defer=8), dict(variant=3, games=4, threads=128, defer=4),
                                  dict(variant=31, chunk=64, defer=8), dict(variant=31, chunk=7, games=2, memo_bits=16),
                                  dict(variant=3, chunk=1456, block_m=4), dict(chunk=3, block_m=8)])
def test_tunes_agree(wl, oracle, tune):
    for job in (wl.make_job(11, rule=0, hbins=64), wl.make_job(10, wl.CANON, rule=1, flags=wl.F_DISTINCT | wl.F_SHAPE,
                                                                 hbins=256, dbins=64)):
        want = oracle.enumerate_job(ojob(oracle, job))
        same(wl, oracle, wl.enumerate_job(job, wl.make_tune(**tune)), want)


@pytest.mark.parametrize("mode,n,ppm", [(0, 10, 10000), (0, 11, 10000), (1, 10, 10000), (0, 10, 1000000),
                                         (1, 10, 1000000), (0, 9, 1000000)])
def test_floyd_sample_cross_check(wl, oracle, mode, n, ppm):
    job = wl.make_job(n, mode, flags=wl.F_SAMPLE, sample_ppm=ppm, seed=2024)
    f = wl.floyd_sample(job)
    b = wl.enumerate_job(job)
    o = oracle.floyd_sample_job(ojob(oracle, job))
    key = lambda r: (r.s_count, r.s_cyc, r.s_lamsum, r.s_lensum, r.s_maxfin)
    assert key(f) == key(b) == key(o)
    assert f.s_count > 0


def test_n12_n13_deals_full(wl, golden):
    """a(12) and a(13) over every deal: the recorded values (data/deals.tsv, data/checks.txt:22-24)."""
    for n in (12, 13):
        r = wl.to_dict(wl.enumerate_job(wl.make_job(n, hbins=256)))
        g = golden["deals_rule0"][n]
        assert (r["done"], r["cyc"], r["maxfin"], r["hist"]) == (g["deals"], g["cyc"], g["longest"], g["hist"])
        assert sum(r["endhist"].values()) == g["deals"] - g["cyc"]
        assert max(r["endhist"]) == g["longest"]


def test_n13_rule1_full(wl, golden):
    r = wl.enumerate_job(wl.make_job(13, rule=1))
    g = golden["deals_rule1"][13]
    assert (r.done, r.cyc, r.maxfin) == (g["deals"], g["cyc"], g["longest"])


def test_n13_canon_distinct_full(wl, golden):
    F = wl.F_DISTINCT | wl.F_SHAPE
    r = wl.to_dict(wl.enumerate_job(wl.make_job(13, wl.CANON, flags=F, hbins=256, dbins=4096)))
    g = golden["canon_rule0"][13]
    assert (r["done"], r["cyc"], r["maxfin"], r["dhist"]) == (g["positions"], g["cycling"], g["longest"], g["dhist"])
    assert r["distinct_min"] == g["distinct"] == sum(v // k for k, v in r["dhist"].items())
    assert (r["shape_nonstd"], r["shape_unchecked"]) == (g["shape_nonstd"], g["shape_unchecked"])
    assert r["oncycle"] == golden["canon_table"][13]["oncycle"]


def test_n14_canon_full(wl, golden):
    """The 80,951,270,400 canonical positions of n = 14 (data/long_runs.txt:19-23), with a 1% Floyd sample."""
    F = wl.F_DISTINCT | wl.F_SAMPLE
    job = wl.make_job(14, wl.CANON, flags=F, hbins=256, dbins=4096, sample_ppm=10000, seed=14)
    r = wl.to_dict(wl.enumerate_job(job))
    g = golden["canon_rule0"][14]
    assert (r["done"], r["cyc"], r["maxfin"]) == (g["positions"], g["cycling"], g["longest"])
    assert r["hist"] == g["hist"]
    assert r["dhist"] == g["dhist"]
    assert r["distinct_min"] == g["distinct"] == 26640
    assert r["oncycle"] == golden["canon_table"][14]["oncycle"]
    f = wl.floyd_sample(job)
    assert (f.s_count, f.s_cyc, f.s_lamsum, f.s_lensum, f.s_maxfin) == \
        (r["s_count"], r["s_cyc"], r["s_lamsum"], r["s_lensum"], r["s_maxfin"])
    assert 0.009 * g["positions"] < r["s_count"] < 0.011 * g["positions"]


def floyd_key(r):
    return (r.s_count, r.s_cyc, r.s_lamsum, r.s_lensum, r.s_maxfin)


def test_floyd_full_range_a13(wl, golden):
    """Every one of the 13! deals played with Floyd (sample rate 100%: the full-range cross-check of
    gpu/war_gpu_floyd.py, recorded at data/long_runs.txt:35), by its own lexicographic enumeration: the recorded
    a(13) and longest game, and every aggregate equal to Brent's on the same job (refill kernel, path memo)."""
    job = wl.make_job(13, flags=wl.F_SAMPLE, sample_ppm=1000000, seed=1)
    f = wl.floyd_sample(job)
    g = golden["floyd_deals"][13]
    assert (f.s_count, f.s_cyc, f.s_maxfin) == (g["deals"], g["cyc"], g["longest"])
    assert floyd_key(f) == floyd_key(wl.enumerate_job(job))


def test_floyd_full_range_canon13(wl, golden):
    """The 5,748,019,200 canonical positions of n = 13 with Floyd (data/long_runs.txt:36) against Brent."""
    job = wl.make_job(13, wl.CANON, flags=wl.F_SAMPLE, sample_ppm=1000000, seed=1)
    f = wl.floyd_sample(job)
    g = golden["canon_rule0"][13]
    assert (f.s_count, f.s_cyc, f.s_maxfin) == (g["positions"], g["cycling"], g["longest"])
    assert floyd_key(f) == floyd_key(wl.enumerate_job(job))


def test_four_games_only_for_the_product_variants(wl):
    """Four games per lane are compiled for variants 3 and 31 only; other variants refuse them."""
    job = wl.make_job(10, hbins=32)
    with pytest.raises(wl.WarError):
        wl.enumerate_job(job, wl.make_tune(games=4, variant=7, threads=256, defer=8))
    with pytest.raises(wl.WarError):
        wl.enumerate_job(job, wl.make_tune(chunk=5000))


def test_native_autotune_keeps_counts(wl, oracle):
    """war_autotune searches on a slice and returns a tune whose full-job counts equal the oracle's."""
    job = wl.make_job(11, hbins=64)
    best, ms = wl.autotune_native(job, slice_ms=30.0, passes=1)
    assert ms > 0 and best.threads in (128, 256, 512, 1024)
    want = oracle.enumerate_job(ojob(oracle, job))
    same(wl, oracle, wl.enumerate_job(job, best), want)
