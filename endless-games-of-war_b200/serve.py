"""Python face of the continuous-batching job server (war_server_* in include/war.h).

    with Server() as s:
        ids = [s.submit(job) for job in jobs]
        results = s.wait_all(ids)

`poisson_stream()` draws the seeded job mix of the serving workload: n uniform over {9, 10, 11, 13, 14, 15},
mode deals (p = 0.7) or canonical positions (p = 0.3), a rank range of log-uniform length in [1e4, 1e9]
clipped to the space, at a uniform offset, arriving as a Poisson process; a job plays the loser-first rule
(--rule 1) with probability p_rule1 and a canonical job counts distinct cycles (--distinct) with
probability p_distinct.  `serve_stream()` replays such a
stream against a server in real time and reports throughput and job latencies (p50 / p99).

    python serve.py --jobs 2000 --rate 200 --verify
"""
import argparse
import ctypes
import json
import math
import os
import random
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import warlib  # noqa: E402

SIZEOF_DEVACC = 20 * 8 + (warlib.WAR_HBINS_MAX + warlib.WAR_DBINS_MAX + warlib.WAR_EBINS) * 8


class Server:
    def __init__(self, max_jobs=256, queue_cap=1 << 16, mem_budget=0, tick_ranks=0, memo_bits=0):
        self.h = ctypes.c_void_p()
        cfg = warlib.ServerCfg(max_jobs, queue_cap, mem_budget, tick_ranks, 0, 0, memo_bits)
        warlib.check(warlib.lib().war_server_create(ctypes.byref(cfg), ctypes.byref(self.h)), "war_server_create")

    def submit(self, job):
        i = ctypes.c_uint64()
        warlib.check(warlib.lib().war_server_submit(self.h, ctypes.byref(job), ctypes.byref(i)), "war_server_submit")
        return i.value

    def poll(self, jid):
        """(done, result or None, status dict).  A finished job is forgotten by the server after this."""
        r, st = warlib.Result(), warlib.JobStatus()
        code = warlib.lib().war_server_poll(self.h, jid, ctypes.byref(r), ctypes.byref(st))
        info = {"state": st.state, "submit_ms": st.submit_ms, "admit_ms": st.admit_ms, "finish_ms": st.finish_ms}
        if code == warlib.PENDING:
            return False, None, info
        warlib.check(code, "war_server_poll")
        return True, r, info

    def drain(self, timeout_ms=600000.0):
        warlib.check(warlib.lib().war_server_drain(self.h, timeout_ms), "war_server_drain")

    def stats(self):
        t, d, p = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        warlib.check(warlib.lib().war_server_stats(self.h, ctypes.byref(t), ctypes.byref(d), ctypes.byref(p)),
                     "war_server_stats")
        return {"ticks": t.value, "jobs_done": d.value, "peak_resident": p.value}

    def memo_info(self):
        """The memo arena reserved at create, the bytes the job classes took from it, and their count."""
        a, u, k = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int32()
        warlib.check(warlib.lib().war_server_memo_info(self.h, ctypes.byref(a), ctypes.byref(u), ctypes.byref(k)),
                     "war_server_memo_info")
        return {"arena_bytes": a.value, "used_bytes": u.value, "classes": k.value}

    def wait_all(self, ids, timeout_s=600.0):
        """Results of the jobs, in order, waiting for each."""
        out = {}
        t_end = time.time() + timeout_s
        left = list(ids)
        while left:
            rest = []
            for jid in left:
                done, r, info = self.poll(jid)
                if done:
                    out[jid] = (r, info)
                else:
                    rest.append(jid)
            left = rest
            if left:
                if time.time() > t_end:
                    raise TimeoutError("%d jobs still running" % len(left))
                time.sleep(0.0005)
        return [out[j] for j in ids]

    def close(self):
        if self.h:
            warlib.lib().war_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def poisson_stream(count, rate, seed=2026, ns=(9, 10, 11, 13, 14, 15), p_deals=0.7, lmin=1e4, lmax=1e9,
                   hbins=256, p_rule1=0.2, p_distinct=0.5, dbins=256):
    """[(arrival_s, job)] of the serving workload, seeded."""
    rnd = random.Random(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += rnd.expovariate(rate)
        n = rnd.choice(ns)
        mode = warlib.DEALS if rnd.random() < p_deals else warlib.CANON
        total = warlib.space_size(n, mode)
        length = int(math.exp(rnd.uniform(math.log(lmin), math.log(lmax))))
        length = max(1, min(length, total))
        lo = rnd.randrange(0, total - length + 1)
        rule = 1 if rnd.random() < p_rule1 else 0
        distinct = mode == warlib.CANON and rnd.random() < p_distinct
        out.append((t, warlib.make_job(n, mode, rule, warlib.F_DISTINCT if distinct else 0, lo, lo + length,
                                       hbins=hbins, dbins=dbins if distinct else 0)))
    return out


def serve_stream(stream, server, poll_sleep=0.0002):
    """Submits each job at its arrival time, collects every result; returns (results, latencies_ms, wall_s)."""
    t0 = time.perf_counter()
    ids, submit_at = [], []
    pending = {}
    results = [None] * len(stream)
    lat = [None] * len(stream)
    i = 0
    while i < len(stream) or pending:
        now = time.perf_counter() - t0
        while i < len(stream) and stream[i][0] <= now:
            pending[server.submit(stream[i][1])] = i
            i += 1
        for jid in list(pending):
            done, r, info = server.poll(jid)
            if done:
                k = pending.pop(jid)
                results[k] = r
                lat[k] = info["finish_ms"] - info["submit_ms"]
        if i < len(stream) and not pending:
            time.sleep(max(0.0, min(stream[i][0] - (time.perf_counter() - t0), 0.01)))
        elif pending:
            time.sleep(poll_sleep)
    return results, lat, time.perf_counter() - t0


def percentile(xs, p):
    s = sorted(xs)
    if not s:
        return None
    k = min(len(s) - 1, max(0, int(math.ceil(p / 100.0 * len(s))) - 1))
    return s[k]


def same_result(p, r, job):
    """Bit-exact equality of two results of one job (every count and histogram the job asks for)."""
    return ((p.cyc, p.done, p.maxfin, p.oncycle, p.distinct_min, p.shape_nonstd, p.shape_unchecked) ==
            (r.cyc, r.done, r.maxfin, r.oncycle, r.distinct_min, r.shape_nonstd, r.shape_unchecked) and
            list(p.hist[:job.hbins]) == list(r.hist[:job.hbins]) and
            list(p.dhist[:job.dbins]) == list(r.dhist[:job.dbins]) and list(p.endhist) == list(r.endhist))


def verify(stream, results):
    """Every job's result against the plain kernel on the same range (bit-exact); returns mismatches."""
    bad = 0
    for (_, job), r in zip(stream, results):
        if not same_result(warlib.enumerate_plain(job), r, job):
            bad += 1
    return bad


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=10000)
    ap.add_argument("--rate", type=float, default=100.0, help="mean arrivals per second")
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--verify", action="store_true", help="check every job against the plain kernel")
    a = ap.parse_args()
    stream = poisson_stream(a.jobs, a.rate, a.seed)
    with Server() as s:
        results, lat, wall = serve_stream(stream, s)
        st = s.stats()
    ranks = sum(j.hi - j.lo for _, j in stream)
    line = {"workload": "serving: %d seeded Poisson jobs, rate %.0f/s" % (a.jobs, a.rate), "jobs": a.jobs,
            "ranks": ranks, "wall_s": wall, "ranks_per_s": ranks / wall, "jobs_per_s": a.jobs / wall,
            "latency_ms": {"p50": percentile(lat, 50), "p99": percentile(lat, 99), "max": max(lat)},
            "server": st}
    if a.verify:
        line["mismatches_vs_plain"] = verify(stream, results)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
