"""Host-side helpers that need no GPU: the serving workload generator and its statistics, and the
autotuner's defaults and legality rules."""
import math


def test_poisson_stream_is_seeded_and_in_range():
    import serve
    import warlib
    a = serve.poisson_stream(3000, rate=100.0, seed=11)
    b = serve.poisson_stream(3000, rate=100.0, seed=11)
    assert [(t, j.n, j.mode, j.lo, j.hi) for t, j in a] == [(t, j.n, j.mode, j.lo, j.hi) for t, j in b]
    times = [t for t, _ in a]
    assert times == sorted(times) and times[0] > 0
    assert abs(len(a) / times[-1] - 100.0) < 10.0                    # Poisson arrivals at the given rate
    deals = 0
    for _, j in a:
        assert j.n in (9, 10, 11, 13, 14, 15)
        total = warlib.space_size(j.n, j.mode)
        assert 0 <= j.lo < j.hi <= total
        assert j.hi - j.lo == min(total, j.hi - j.lo)
        assert j.hi - j.lo <= 10 ** 9 and (j.hi - j.lo >= 10 ** 4 or j.hi - j.lo == total)
        deals += j.mode == warlib.DEALS
    assert 0.65 < deals / len(a) < 0.75                                # 70% deals
    rule1 = sum(j.rule for _, j in a) / len(a)
    assert 0.15 < rule1 < 0.25                                         # 20% loser-first
    canon = [j for _, j in a if j.mode == warlib.CANON]
    dist = [j for j in canon if j.flags & warlib.F_DISTINCT]
    assert 0.4 < len(dist) / len(canon) < 0.6 and all(j.dbins == 256 for j in dist)   # half of them --distinct
    assert all(j.flags == 0 and j.dbins == 0 for _, j in a if j.mode == warlib.DEALS)


def test_percentile():
    import serve
    xs = list(range(1, 101))
    assert serve.percentile(xs, 50) == 50 and serve.percentile(xs, 99) == 99 and serve.percentile(xs, 100) == 100
    assert serve.percentile([], 50) is None


def test_default_tunes():
    import autotune
    import warlib
    c14 = autotune.default_tune(14, warlib.CANON, 0, warlib.F_DISTINCT | warlib.F_SHAPE)
    assert c14["variant"] == 31 and c14["window"] >= 128            # the free on-cycle test needs W >= lam
    assert autotune.default_tune(3, warlib.DEALS, 0, 0) is None
    t13, t17 = autotune.default_tune(13, warlib.DEALS, 0, 0), autotune.default_tune(17, warlib.DEALS, 0, 0)
    assert t13["variant"] == 31 and t17["variant"] == 3
    bits = [autotune.default_tune(n, warlib.DEALS, 0, 0)["memo_bits"] for n in range(4, 17)]
    assert bits == sorted(bits) and 12 <= bits[0] and bits[-1] <= 31
    assert all(autotune.default_tune(n, warlib.DEALS, 0, 0)["block_m"] <= n for n in range(4, 18))


def test_autotune_legality():
    import autotune
    import warlib
    base = dict(autotune.DEFAULT)
    assert autotune._legal(13, warlib.DEALS, 0, base)
    assert not autotune._legal(13, warlib.DEALS, 0, dict(base, games=2, threads=1024))
    assert not autotune._legal(4, warlib.DEALS, 0, dict(base, block_m=5))
    assert not autotune._legal(14, warlib.CANON, warlib.F_DISTINCT, dict(base, window=32))   # on-cycle test needs W >= lam
    assert autotune._legal(14, warlib.CANON, warlib.F_DISTINCT, dict(base, window=128))


def test_space_sizes():
    import warlib
    assert warlib.space_size(13) == math.factorial(13)
    assert warlib.space_size(14, warlib.CANON) == math.factorial(13) * 13
    assert warlib.space_size(1, warlib.CANON) == 0


def test_bench_counts_the_extra_units_the_library_plans():
    """bench.py's e2e line counts the bytes of the extra work units copied to the device per step; its count
    of units for a deal range equals the plan the library makes (war_plan, host only)."""
    import random
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import warlib
    rnd = random.Random(3)
    for _ in range(300):
        n = rnd.randint(6, 16)
        m = rnd.randint(1, min(8, n))
        total = warlib.space_size(n)
        lo = rnd.randrange(total)
        hi = min(total, lo + rnd.choice([1, 50, 5000, 10 ** 6, 10 ** 9, total]))
        assert bench.deal_extra_units(lo, hi, m) == len(warlib.plan(warlib.make_job(n, lo=lo, hi=hi), m)[2])


def test_bench_cpu_baseline_times_the_program_of_each_engine():
    """The cpu_baseline of the 17-card workloads samples the workload's own slice with the oracle's restatement of
    the program that engine replaces (gpu/war17.py for the held-out engine, gpu/war24.py for the 5-bit engine),
    and the main workloads the restatement of cpu/war.cpp; the line names which."""
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    for wl, prog in (("held17", "gpu/war17.py"), ("wide17", "gpu/war24.py"), ("deals11", "cpu/war.cpp")):
        line = bench.cpu_baseline(bench.WORKLOADS[wl], target_s=0.2)
        assert line["kind"] == "port" and line["value"] > 0 and line["unit"] == "deals/s"
        assert prog in line["sample"], (wl, line["sample"])


def test_tune_override():
    """war_gpu.py --tune and bench.py --tune: fields of the stored tune replaced, unknown fields refused."""
    import pytest
    import war_gpu
    import warlib
    base = warlib.make_tune(threads=256, block_m=6, window=32, defer=8, variant=31, memo_bits=31)
    t = war_gpu.override_tune(base, {"variant": 3, "threads": "512"})
    assert (t.variant, t.threads, t.block_m, t.window, t.defer, t.memo_bits) == (3, 512, 6, 32, 8, 31)
    assert base.variant == 31                       # a copy: the stored tune is left as it was
    assert war_gpu.override_tune(None, {"defer": 16}).defer == 16
    with pytest.raises(ValueError):
        war_gpu.override_tune(base, {"no_such_field": 1})
