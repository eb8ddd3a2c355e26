"""The continuous-batching server: every job's result is the same alone (war_enumerate, the plain kernel)
and in a mix of jobs of different n, mode, rule and range running together; admission respects the
memory budget; queued jobs wait for slots."""
import pytest

pytestmark = pytest.mark.gpu


def mix(wl):
    jobs = []
    for n in (9, 10, 11):
        jobs.append(wl.make_job(n, hbins=128))
        jobs.append(wl.make_job(n, rule=1, hbins=64))
    jobs.append(wl.make_job(10, wl.CANON, flags=wl.F_DISTINCT | wl.F_SHAPE, hbins=128, dbins=64))
    jobs.append(wl.make_job(11, wl.CANON, rule=1, hbins=64))
    jobs.append(wl.make_job(12, lo=1000, hi=3_000_000, hbins=128))
    jobs.append(wl.make_job(13, lo=3_000_000_000, hi=3_020_000_000, hbins=256))
    jobs.append(wl.make_job(13, lo=5, hi=17))
    jobs.append(wl.make_job(14, wl.CANON, lo=40_000_000_003, hi=40_010_000_000, hbins=256, flags=wl.F_DISTINCT,
                            dbins=64))
    jobs.append(wl.make_job(15, lo=10 ** 12, hi=10 ** 12 + 4_000_000, hbins=128))
    jobs.append(wl.make_job(14, flags=wl.F_HALF, lo=10 ** 9, hi=10 ** 9 + 5_000_000, hbins=128))
    jobs.append(wl.make_job(1))
    jobs.append(wl.make_job(12, lo=7, hi=7))
    jobs.append(wl.make_job(16, wl.CANON, lo=10 ** 13, hi=10 ** 13 + 300_000, hbins=64))
    return jobs


def same(wl, a, b, with_turns=False):
    da, db = wl.to_dict(a), wl.to_dict(b)
    for k in ("cyc", "done", "maxfin", "oncycle", "distinct_min", "shape_nonstd", "shape_unchecked", "hist", "dhist",
              "endhist"):
        assert da[k] == db[k], k


def test_each_job_same_alone_and_in_the_mix(wl, oracle):
    import serve
    jobs = mix(wl)
    alone = [wl.enumerate_job(j) for j in jobs]
    with serve.Server() as s:
        ids = [s.submit(j) for j in jobs]
        got = s.wait_all(ids)
        st = s.stats()
        mi = s.memo_info()
    for j, a, (r, info) in zip(jobs, alone, got):
        same(wl, r, a)
        assert info["finish_ms"] >= info["admit_ms"] >= info["submit_ms"]
    for j, a in zip(jobs, alone):
        if j.hi > j.lo and j.n > 1:
            same(wl, wl.enumerate_plain(j), a)
    # the small jobs of the mix against the oracle as well
    for j, (r, _) in zip(jobs, got):
        if j.n <= 11:
            want = oracle.to_dict(oracle.enumerate_job(oracle.make_job(j.n, j.mode, j.rule, j.flags, j.lo, j.hi,
                                                                       j.hbins, j.dbins, j.blk)))
            g = wl.to_dict(r)
            for k in ("cyc", "done", "maxfin", "oncycle", "distinct_min", "shape_nonstd", "hist", "dhist", "endhist"):
                assert g[k] == want[k], (j.n, j.mode, k)
    assert st["jobs_done"] == len(jobs)
    assert st["ticks"] >= 1
    # the memo tables came from the arena reserved at create, inside it
    assert mi["arena_bytes"] > 0 and 0 < mi["used_bytes"] <= mi["arena_bytes"] and mi["classes"] >= 2


def test_admission_by_memory_budget(wl):
    """A budget of three accumulator slots admits three jobs at a time and leaves nothing for a memo arena:
    the jobs run without the memo, with the same results (including an n = 13 slice, whose class would
    otherwise take a 2 GiB table)."""
    import serve
    jobs = [wl.make_job(11, lo=i * 1_000_000, hi=(i + 1) * 1_000_000, hbins=32) for i in range(12)]
    jobs.append(wl.make_job(13, lo=2_000_000_000, hi=2_030_000_000, hbins=128))
    alone = [wl.enumerate_job(j) for j in jobs]
    with serve.Server(mem_budget=3 * serve.SIZEOF_DEVACC + 100) as s:
        ids = [s.submit(j) for j in jobs]
        got = s.wait_all(ids)
        st = s.stats()
        mi = s.memo_info()
    assert st["peak_resident"] <= 3
    assert mi == {"arena_bytes": 0, "used_bytes": 0, "classes": 0}
    for j, a, (r, _) in zip(jobs, alone, got):
        same(wl, r, a)
        same(wl, wl.enumerate_plain(j), r)


def test_memo_arena_inside_the_budget(wl):
    """A budget with room for the slots and a small arena: the first class takes what fits, a later class
    whose table no longer fits runs without one; every result is the same."""
    import serve
    jobs = [wl.make_job(13, lo=10 ** 9, hi=10 ** 9 + 2 * 10 ** 7, hbins=128),
            wl.make_job(14, lo=5 * 10 ** 9, hi=5 * 10 ** 9 + 10 ** 7, hbins=128),
            wl.make_job(13, lo=4 * 10 ** 9, hi=4 * 10 ** 9 + 10 ** 7, rule=1, hbins=64)]
    alone = [wl.enumerate_job(j) for j in jobs]
    budget = 8 * serve.SIZEOF_DEVACC + (8 << 20)          # 8 slots and an 8 MiB arena
    with serve.Server(max_jobs=8, mem_budget=budget) as s:
        got = s.wait_all([s.submit(j) for j in jobs])
        mi = s.memo_info()
    assert mi["arena_bytes"] == 8 << 20 and mi["used_bytes"] == 8 << 20 and mi["classes"] == 1
    for a, (r, _) in zip(alone, got):
        same(wl, r, a)


def test_poisson_stream_small(wl):
    import serve
    stream = serve.poisson_stream(120, rate=400.0, seed=7, lmax=3e7)
    with serve.Server() as s:
        results, lat, wall = serve.serve_stream(stream, s)
    assert all(r is not None for r in results)
    assert serve.verify(stream[:60], results[:60]) == 0
    assert any(j.rule for _, j in stream[:60]) and any(j.flags & wl.F_DISTINCT for _, j in stream[:60])
    assert serve.percentile(lat, 50) <= serve.percentile(lat, 99)


def test_shared_memo_same_as_without(wl):
    """Jobs of one n and rule share the server's cycle memo; the results equal a server without it, and a
    memo far too small for the class changes nothing either."""
    import serve
    jobs = mix(wl) + [wl.make_job(13, lo=10 ** 9, hi=10 ** 9 + 2 * 10 ** 7, hbins=128),
                      wl.make_job(13, lo=10 ** 9 + 5, hi=10 ** 9 + 10 ** 7, hbins=128)]
    got = {}
    for bits in (0, -1, 12):
        with serve.Server(memo_bits=bits) as s:
            ids = [s.submit(j) for j in jobs]
            got[bits] = [r for r, _ in s.wait_all(ids)]
    for a, b, c in zip(got[0], got[-1], got[12]):
        same(wl, a, b)
        same(wl, c, b)
