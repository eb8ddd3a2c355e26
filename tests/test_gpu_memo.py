"""The cycle memo (tune variant bit 2, landmarks; with bit 3, every cycle state; with bit 4, also states on
the paths of decided games with their outcome): deals decided as soon as they meet a memoised state give
the same counts as Brent alone — whole a(12) and a(13), both rules, slices of n = 14 and 15 (where the
cycle length field of a memo entry is narrowest), a table too small to hold the cycles, and the seeded
sample aggregates."""
import random

import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("cyc", "done", "maxfin", "shape_nonstd", "shape_unchecked", "oncycle", "distinct_min", "s_count", "s_cyc",
          "s_lamsum", "s_lensum", "s_maxfin")


def memo_tune(wl, **kw):
    t = dict(variant=7, games=2, threads=256, defer=8)
    t.update(kw)
    return wl.make_tune(**t)


def same(wl, a, b):
    da, db = wl.to_dict(a), wl.to_dict(b)
    for k in FIELDS + ("hist", "dhist", "endhist"):
        assert da[k] == db[k], (k, da[k], db[k])


@pytest.mark.parametrize("variant", [7, 15, 31])
def test_memo_full_a12_a13(wl, golden, variant):
    for n in (12, 13):
        r = wl.enumerate_job(wl.make_job(n, hbins=256), memo_tune(wl, variant=variant))
        d = wl.to_dict(r)
        g = golden["deals_rule0"][n]
        assert (d["done"], d["cyc"], d["maxfin"], d["hist"]) == (g["deals"], g["cyc"], g["longest"], g["hist"])
        assert max(d["endhist"]) == g["longest"]
        base = wl.enumerate_job(wl.make_job(n, hbins=256), wl.make_tune(variant=3, games=2, threads=256, defer=8))
        same(wl, r, base)
        if n == 13:
            assert r.turns < base.turns / 2   # the memo decides most cycling deals early


def test_memo_rule1_a13(wl, golden):
    r = wl.enumerate_job(wl.make_job(13, rule=1), memo_tune(wl, variant=6, games=1, threads=512))
    g = golden["deals_rule1"][13]
    assert (r.done, r.cyc, r.maxfin) == (g["deals"], g["cyc"], g["longest"])


@pytest.mark.parametrize("bits,variant", [(12, 7), (16, 7), (12, 15), (16, 14), (12, 31), (16, 30)])
def test_memo_small_table(wl, bits, variant):
    """A table far smaller than the cycles' states: most inserts are lost, lookups miss, counts stay exact."""
    job = wl.make_job(12, lo=10 ** 8, hi=2 * 10 ** 8, hbins=128)
    same(wl, wl.enumerate_job(job, memo_tune(wl, memo_bits=bits, variant=variant)), wl.enumerate_plain(job))


@pytest.mark.parametrize("n,lo,span", [(14, 7 * 10 ** 9, 3 * 10 ** 8), (15, 10 ** 12, 2 * 10 ** 8),
                                       (15, 3 * 10 ** 11 + 12345, 10 ** 7), (11, 0, 39916800),
                                       (16, 10 ** 13, 2 * 10 ** 8), (16, 2 * 10 ** 13 + 777, 3 * 10 ** 6)])
def test_memo_slices_vs_plain(wl, n, lo, span):
    for rule in (0, 1):
        job = wl.make_job(n, rule=rule, lo=lo, hi=lo + span, hbins=512)
        plain = wl.enumerate_plain(job)
        same(wl, wl.enumerate_job(job, memo_tune(wl)), plain)
        same(wl, wl.enumerate_job(job, memo_tune(wl, variant=15, games=1)), plain)   # all states (n <= 14)
        same(wl, wl.enumerate_job(job, memo_tune(wl, variant=31, games=1)), plain)   # and paths (n <= 16)


def test_memo_random_ranges_with_sample(wl, oracle):
    rnd = random.Random(4242)
    for n in (5, 7, 9, 10, 11):
        total = wl.space_size(n, wl.DEALS)
        for _ in range(3):
            lo = rnd.randrange(0, total)
            hi = min(total, lo + rnd.choice([1, 33, 5000, 400000]))
            job = wl.make_job(n, rule=rnd.randint(0, 1), flags=wl.F_SAMPLE, sample_ppm=50000, seed=11, lo=lo, hi=hi,
                              hbins=128)
            want = oracle.enumerate_job(oracle.make_job(n, 0, job.rule, job.flags, lo, hi, 128, 0, 0, 50000, 11))
            got = wl.to_dict(wl.enumerate_job(job, memo_tune(wl, games=rnd.choice([1, 2]),
                                                             variant=rnd.choice([6, 7, 14, 15, 30, 31]))))
            w = oracle.to_dict(want)
            for k in FIELDS + ("hist", "endhist"):
                assert got[k] == w[k], (n, lo, hi, k)


def test_memo_ignored_where_it_does_not_apply(wl, oracle):
    """Canonical scans, the immediate-record loop and n = 16 run without the memo, same counts."""
    job = wl.make_job(10, wl.CANON, flags=wl.F_DISTINCT, hbins=64, dbins=64)
    same(wl, wl.enumerate_job(job, memo_tune(wl)), wl.enumerate_job(job))
    job = wl.make_job(11, hbins=64)
    same(wl, wl.enumerate_job(job, wl.make_tune(variant=5)), wl.enumerate_job(job))
    job = wl.make_job(16, lo=10 ** 13, hi=10 ** 13 + 2 * 10 ** 6, hbins=128)
    same(wl, wl.enumerate_job(job, memo_tune(wl)), wl.enumerate_plain(job))


def test_memo_kept_across_jobs(wl):
    """WAR_F_MEMO_KEEP: a job that starts from the memo of the previous job of the same n and rule counts the
    same; a kept memo of another n or rule is not used (the job clears it)."""
    t = memo_tune(wl, variant=31)
    a = wl.make_job(13, lo=10 ** 9, hi=10 ** 9 + 3 * 10 ** 8, hbins=128)
    b = wl.make_job(13, flags=wl.F_MEMO_KEEP, lo=4 * 10 ** 9, hi=4 * 10 ** 9 + 3 * 10 ** 8, hbins=128)
    cold = wl.enumerate_job(b, wl.make_tune(variant=3, games=2, threads=256, defer=8))
    wl.enumerate_job(a, t)
    warm = wl.enumerate_job(b, t)
    same(wl, warm, cold)
    assert warm.turns < cold.turns
    wl.enumerate_job(wl.make_job(12, rule=1, lo=0, hi=10 ** 8), t)
    same(wl, wl.enumerate_job(b, t), cold)   # the rule-1 n = 12 memo is not kept for n = 13 rule 0
    c = wl.make_job(12, flags=wl.F_MEMO_KEEP, lo=2 * 10 ** 8, hi=4 * 10 ** 8, hbins=128)
    same(wl, wl.enumerate_job(c, t), wl.enumerate_plain(wl.make_job(12, lo=2 * 10 ** 8, hi=4 * 10 ** 8, hbins=128)))


@pytest.mark.parametrize("variant", [30, 31])
def test_memo_canon_small_vs_oracle(wl, oracle, variant):
    """Canonical scans with the path memo: cycling count, λ-histogram, ending lengths, the distinct-cycle
    outputs (on-cycle starts, min keys, weights) and the sample aggregates equal the oracle's."""
    for n in (5, 7, 9, 10, 11):
        for rule in (0, 1):
            job = wl.make_job(n, wl.CANON, rule=rule, flags=wl.F_DISTINCT | wl.F_SAMPLE, hbins=256, dbins=256,
                              sample_ppm=30000, seed=5)
            want = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, 1, rule, job.flags, 0, job.hi, 256, 256, 0,
                                                                       30000, 5)))
            got = wl.to_dict(wl.enumerate_job(job, memo_tune(wl, variant=variant, window=128, memo_bits=20)))
            for k in FIELDS + ("hist", "dhist", "endhist"):
                assert got[k] == want[k], (n, rule, k)


def test_memo_canon_random_ranges(wl, oracle):
    rnd = random.Random(77)
    for n in (9, 10, 11):
        total = wl.space_size(n, wl.CANON)
        for _ in range(3):
            lo = rnd.randrange(0, total)
            hi = min(total, lo + rnd.choice([1, 50, 7777, 300000]))
            job = wl.make_job(n, wl.CANON, rule=rnd.randint(0, 1), flags=wl.F_DISTINCT, lo=lo, hi=hi, hbins=128,
                              dbins=128)
            want = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, 1, job.rule, job.flags, lo, hi, 128, 128)))
            got = wl.to_dict(wl.enumerate_job(job, memo_tune(wl, variant=31, window=128)))
            for k in FIELDS + ("hist", "dhist", "endhist"):
                assert got[k] == want[k], (n, lo, hi, k)


def test_memo_canon_n13_n14_full(wl, golden):
    """The n = 13 and n = 14 canonical scans with --distinct and the path memo: the recorded cycling,
    on-cycle and distinct counts and the weights."""
    for n in (13, 14):
        job = wl.make_job(n, wl.CANON, flags=wl.F_DISTINCT, hbins=256, dbins=4096)
        r = wl.to_dict(wl.enumerate_job(job, memo_tune(wl, window=128, memo_bits=28)))
        g = golden["canon_table"][n]
        assert (r["cyc"], r["oncycle"], r["done"]) == (g["cycling"], g["oncycle"], g["positions"])
        assert sum(v // k for k, v in r["dhist"].items()) == g["distinct"]
        plain = wl.to_dict(wl.enumerate_job(job))   # the same scan without the memo
        for k in FIELDS + ("hist", "dhist", "endhist"):
            assert r[k] == plain[k], (n, k)


@pytest.mark.parametrize("variant", [30, 31])
def test_memo_canon_shape_small_vs_oracle(wl, oracle, variant):
    """The loop-shape test (--shape) with the path memo: the shape code travels with the cycle length."""
    for n in (5, 7, 8, 9, 10, 11):
        for rule in (0, 1):
            F = wl.F_DISTINCT | wl.F_SHAPE
            job = wl.make_job(n, wl.CANON, rule=rule, flags=F, hbins=256, dbins=256)
            want = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, 1, rule, F, 0, job.hi, 256, 256)))
            got = wl.to_dict(wl.enumerate_job(job, memo_tune(wl, variant=variant, window=128, memo_bits=20)))
            for k in FIELDS + ("hist", "dhist", "endhist"):
                assert got[k] == want[k], (n, rule, k)
    rnd = random.Random(5)
    for n in (10, 11):
        total = wl.space_size(n, wl.CANON)
        lo = rnd.randrange(0, total - 400000)
        job = wl.make_job(n, wl.CANON, flags=wl.F_SHAPE, lo=lo, hi=lo + 400000, hbins=128)
        want = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, 1, 0, wl.F_SHAPE, lo, lo + 400000, 128, 0)))
        got = wl.to_dict(wl.enumerate_job(job, memo_tune(wl, variant=variant, window=128, memo_bits=16)))
        for k in FIELDS + ("hist", "endhist"):
            assert got[k] == want[k], (n, lo, k)


def test_memo_canon_shape_n13_n14_full(wl, golden):
    """`war_gpu.py 13/14 --canon --distinct --shape` with the path memo against the recorded values (data/
    checks.txt:180-182, data/long_runs.txt:20-23), the shape counts included."""
    for n in (13, 14):
        job = wl.make_job(n, wl.CANON, flags=wl.F_DISTINCT | wl.F_SHAPE, hbins=256, dbins=4096)
        r = wl.to_dict(wl.enumerate_job(job, memo_tune(wl, variant=31, games=1, threads=512, block_m=5, window=128,
                                                       defer=16, memo_bits=28)))
        g = golden["canon_rule0"][n]
        assert (r["done"], r["cyc"], r["maxfin"], r["dhist"]) == (g["positions"], g["cycling"], g["longest"], g["dhist"])
        assert r["distinct_min"] == g["distinct"]
        assert (r["shape_nonstd"], r["shape_unchecked"]) == (g["shape_nonstd"], g["shape_unchecked"])
        if "hist" in g:
            assert r["hist"] == g["hist"]
