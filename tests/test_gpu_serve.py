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


def test_each_job_same_alone_and_in_the_mix(wl):
    import serve
    jobs = mix(wl)
    alone = [wl.enumerate_job(j) for j in jobs]
    with serve.Server() as s:
        ids = [s.submit(j) for j in jobs]
        got = s.wait_all(ids)
        st = s.stats()
    for j, a, (r, info) in zip(jobs, alone, got):
        same(wl, r, a)
        assert info["finish_ms"] >= info["admit_ms"] >= info["submit_ms"]
    for j, a in zip(jobs, alone):
        if j.hi > j.lo and j.n > 1:
            same(wl, wl.enumerate_plain(j), a)
    assert st["jobs_done"] == len(jobs)
    assert st["ticks"] >= 1


def test_admission_by_memory_budget(wl):
    import serve
    jobs = [wl.make_job(11, lo=i * 1_000_000, hi=(i + 1) * 1_000_000, hbins=32) for i in range(12)]
    alone = [wl.enumerate_job(j) for j in jobs]
    with serve.Server(mem_budget=3 * serve.SIZEOF_DEVACC + 100) as s:
        ids = [s.submit(j) for j in jobs]
        got = s.wait_all(ids)
        st = s.stats()
    assert st["peak_resident"] <= 3
    for a, (r, _) in zip(alone, got):
        same(wl, r, a)


def test_poisson_stream_small(wl):
    import serve
    stream = serve.poisson_stream(120, rate=400.0, seed=7, lmax=3e7)
    with serve.Server() as s:
        results, lat, wall = serve.serve_stream(stream, s)
    assert all(r is not None for r in results)
    assert serve.verify(stream[:40], results[:40]) == 0
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
