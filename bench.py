"""Benchmark of the exhaustive War enumerator on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload deals13|canon14|deals11] [--impl ours|reference]

One step = one complete enumeration of the workload's rank space by the persistent refill kernel
(war_enumerate), results checked bit-exactly against the reference's recorded values after the timed
region.  Workloads (the rank spaces are the inputs; nothing is random):
  deals13  all 13! = 6,227,020,800 deals, cycle-length and ending-length histograms   (default)
  canon14  all 13!*13 = 80,951,270,400 canonical positions of n = 14, distinct cycles, cycle-length
           histogram and the seeded 1% Floyd cross-check
  deals11  all 11! deals (plain GPU drop-in size)
With N ranks (torchrun, one GPU each) the rank space is cut into N contiguous shards and the per-rank
results are summed with one all-reduce of the accumulators (strong scaling).  Rank 0 prints one JSON
line.  --impl reference times the reference's own CPU program (cpu/war.cpp, built unmodified into
oracle/_ref/) or, when a full run would not fit the time budget, the oracle's restatement of it on a
bounded strided sample, on all host cores.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "endless-games-of-war_b200")
sys.path.insert(0, PKG)

# Algorithmic integer operations per turn: the turn step (pop both tops, compare, build the pair, place it
# under the winner: 22), Brent's test and bookkeeping (6), the end test (2).  Fixed from the source of
# war_turn / batched_kernel, not from compiled code.
K_OPS_PER_TURN = 30
# DRAM bytes (read + write) per deal of the path-memo refill kernel, from an ncu capture of the second span
# of `war_gpu.py 13 --hist 256` (1.94e9 deals, 214.6 GB): the random memo reads cost ~108 B each.
MEMO_DRAM_BYTES_PER_DEAL = 110.8

WORKLOADS = {
    "deals13": dict(n=13, mode=0, hbins=256, flags=0, label="n=13 all deals (war_gpu.py 13 --hist 256)"),
    "canon14": dict(n=14, mode=1, hbins=256, dbins=4096, flags=2 | 8, sample_ppm=10000, seed=14,
                    label="n=14 canonical positions, --distinct, --hist 256, 1% Floyd sample"),
    "deals11": dict(n=11, mode=0, hbins=256, flags=0, label="n=11 all deals"),
    # a 2e8-deal slice from the middle of the n = 13 space (profiling size)
    "deals13slice": dict(n=13, mode=0, hbins=256, flags=0, lo=3013510400, hi=3213510400,
                         label="n=13 deals, ranks [3013510400, 3213510400)"),
}


def measured_hbm_peak():
    """(GB/s, source): the pool's measured copy bandwidth, else the stated fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def space(n, mode):
    return math.factorial(n - 1) * (n - 1) if mode else math.factorial(n)


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons every 200 ms while running."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [float(r[0]) for r in self.rows if len(r) >= 8 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 8:
                for name, v in zip(names, r[4:8]):
                    if v.lower() == "active":
                        reasons.add(name)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws == 1:
        return 0, 1, 0
    import datetime
    import torch
    import torch.distributed as dist
    rank, local = int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, ws, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reference_arm(args, rank, ws):
    """The reference's CPU implementation on the host cores (rank 0 only)."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    w = WORKLOADS[args.workload]
    n, mode = w["n"], w["mode"]
    cores = os.cpu_count() or 1
    total = space(n, mode)
    line = {"impl": "reference", "metric": "positions/s" if mode else "deals/s", "unit": "positions/s" if mode else "deals/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "exhaustive (deterministic rank space)",
            "config": {"workload": w["label"], "n": n, "mode": "canon" if mode else "deals"}}
    use_ref = (mode == 0 and oracle.ref_available("war"))
    est = None
    if use_ref:
        t0 = time.time()
        oracle.ref_war(11, 0)
        t11 = time.time() - t0
        # n = 13 plays 156x the deals of n = 11 at 3.6x the turns per deal (Brent turn totals)
        est = t11 * (math.factorial(n) * (686746920144 / 6227020800)) / (39916800 * 30.46)
        use_ref = est * args.steps <= 240
    times = []
    if use_ref:
        for _ in range(args.steps):
            t0 = time.time()
            deals, cyc, longest = oracle.ref_war(n, 0)
            times.append(time.time() - t0)
        assert deals == total
        sample, kind, units = "full run of cpu/war.cpp %d 0 (%d deals)" % (n, total), "reference", total
    else:
        # bounded strided samples of the same rank space, ~150 s in all
        per_step = 150.0 / max(1, args.steps + 1)
        _oracle_sample_rate(w, min(per_step, 10.0), cores)           # warm-up
        done_units = 0
        for s in range(args.steps):
            v, slice_len = _oracle_sample_rate(w, per_step, cores, seed=s + 1)
            times.append(slice_len * 64 / v)
            done_units += slice_len * 64
        units = done_units / len(times)
        sample, kind = ("64 strided slices of %d ranks of the %s space per step (oracle restatement of the "
                        "reference algorithm; a full cpu/war.cpp run is estimated at %s s here)" % (
                            slice_len, "canonical-position" if mode else "deal",
                            "%.0f" % est if est else "n/a"), "port")
    t = sum(times) / len(times)
    v = units / t
    line.update({"value": v, "ms_per_step": t * 1e3,
                 "cpu_baseline": {"value": v, "unit": line["unit"], "cores": cores, "kind": kind, "sample": sample,
                                  "estimate_full_s": est},
                 "e2e": {"value": v, "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)


def _oracle_sample_rate(w, target_s, cores, seed=0):
    """Times the oracle's restatement of the reference algorithm on a strided sample of the workload's
    rank space (64 slices spread evenly), sized by a short probe to take about target_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    n, mode = w["n"], w["mode"]
    total = space(n, mode)

    def run(slice_len):
        t0 = time.time()
        for i in range(64):
            lo = (total // 64) * i + (seed * 7919) % max(1, total // 64 - slice_len)
            job = oracle.make_job(n, mode, 0, w["flags"] & ~8, lo, min(total, lo + slice_len), hbins=w["hbins"],
                                  dbins=w.get("dbins", 0))
            oracle.enumerate_job(job, cores)
        return time.time() - t0

    probe = 4096
    dt = run(probe)
    slice_len = max(probe, int(probe * target_s / max(dt, 1e-3)))
    dt = run(slice_len)
    return slice_len * 64 / dt, slice_len


def cpu_baseline(w, target_s=12.0):
    """The oracle's restatement of the reference algorithm on a bounded strided sample (all host threads)."""
    cores = os.cpu_count() or 1
    v, slice_len = _oracle_sample_rate(w, target_s, cores)
    mode = w["mode"]
    return {"value": v, "unit": "positions/s" if mode else "deals/s", "cores": cores, "kind": "port",
            "sample": "64 strided slices of %d ranks of the %s space, oracle/war_oracle.c (restatement of "
                      "cpu/war.cpp's algorithm, OpenMP on all host threads), ~%.0f s" % (
                          slice_len, "canonical-position" if mode else "deal", target_s)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="deals13", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-kernel comparison run")
    args = ap.parse_args()

    rank, ws, local = dist_init()
    if args.impl == "reference":
        reference_arm(args, rank, ws)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    import warlib
    import war_gpu
    w = WORKLOADS[args.workload]
    n, mode = w["n"], w["mode"]
    import shard
    lo0, hi0 = w.get("lo", 0), w.get("hi", space(n, mode))
    total = hi0 - lo0
    lo, hi = shard.shard_range(lo0, hi0, rank, ws)
    job = warlib.make_job(n, mode, 0, w["flags"], lo, hi, hbins=w["hbins"], dbins=w.get("dbins", 0),
                          sample_ppm=w.get("sample_ppm", 0), seed=w.get("seed", 0))
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    warlib.set_stream(stream.cuda_stream)
    tune = war_gpu._tune_for(n, mode == 1, 0, w["flags"])

    floyd_ms = []

    def step():
        r = warlib.enumerate_job(job, tune)
        if w["flags"] & 8:
            f = warlib.floyd_sample(job)
            assert (f.s_count, f.s_cyc, f.s_lamsum, f.s_lensum, f.s_maxfin) == \
                (r.s_count, r.s_cyc, r.s_lamsum, r.s_lensum, r.s_maxfin), "Floyd sample disagrees with Brent"
            floyd_ms.append(f.kernel_ms)
        return r

    for _ in range(args.warmup):
        step()
    launches0 = warlib.launch_count()
    results = []
    with Clocks(local) as clk:
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            results.append(step())
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
    launches = warlib.launch_count() - launches0
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, ws)
    kernel_ms = sum(r.kernel_ms for r in results) / len(results)
    turns = results[-1].turns
    # exactness of every step
    for r in results:
        assert r.done == results[0].done and r.cyc == results[0].cyc and r.maxfin == results[0].maxfin
    res = results[-1]
    acc = [res.cyc, res.done, res.maxfin, res.turns, res.distinct_min, res.oncycle]
    if ws > 1:   # the one exchange of the sharded path: combine the per-rank results
        import shard
        d = shard.allreduce_result(shard.result_to_dict(res), device="cuda")
        acc = [d["cyc"], d["done"], d["maxfin"], d["turns"], d["distinct_min"], d["oncycle"]]
    check = verify(w, acc, res if ws == 1 else None) if "lo" not in w else "slice (no recorded total)"

    # e2e through the public drop-in API (war_gpu.run), host buffers, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        kw = dict(hbins=w["hbins"], canon=mode == 1, dbins=w.get("dbins", 0), quiet=True)
        warlib.set_stream(0)

        def e2e_step():
            if ws == 1 and "lo" not in w:
                war_gpu.run(n, **kw)
            else:
                warlib.enumerate_job(job, tune)
        e2e_step()                      # untimed: first-call set-up of the Python side
        reps = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(reps):
            e2e_step()
        torch.cuda.synchronize()
        barrier(ws)
        e2e_s = max_over_ranks((time.perf_counter() - t0) / reps, ws)
        h2d = 64 + 24 * 64 + 512       # job/tune structs, extra units, kernel parameter block per launch
        d2h = 73880                      # the accumulator block read back per launch
        e2e = {"value": total / e2e_s, "unit": "positions/s" if mode else "deals/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "api": "war_gpu.run" if ws == 1 else "warlib.enumerate_job"}

    # the plain kernel (the reference's per-thread rank blocks, restated for sm_100a) on the same job,
    # once, outside the timed region: the batched-versus-plain ratio
    plain = None
    if not args.no_plain and ws == 1:
        warlib.set_stream(stream.cuda_stream)
        rp = warlib.enumerate_plain(job)
        assert (rp.cyc, rp.done, rp.maxfin) == (res.cyc, res.done, res.maxfin), "plain and refill kernels disagree"
        plain = {"value": (hi - lo) / (rp.kernel_ms * 1e-3), "kernel_ms": rp.kernel_ms, "turns": rp.turns,
                 "batched_over_plain": rp.kernel_ms / kernel_ms}

    if rank == 0:
        issue_peak, alu_peak = warlib.measure_int_peak()
        achieved = turns * K_OPS_PER_TURN / (kernel_ms * 1e-3)    # algorithmic int ops/s of the refill kernel
        memo = None
        if tune is not None and (tune.variant & 4) and res.memo_lookups:
            # the cycle memo's own traffic: one 8-byte word read per lookup, one written per store
            hbm_peak, hbm_src = measured_hbm_peak()
            mbytes = 8.0 * (res.memo_lookups + res.memo_stores)
            memo = {"variant": tune.variant, "table_bytes": 8 << (tune.memo_bits or 24),
                    "lookups_per_game": res.memo_lookups / res.done, "hit_rate": res.memo_hits / res.memo_lookups,
                    "stores_per_game": res.memo_stores / res.done, "turns_per_game": res.turns / res.done,
                    "algorithmic_GBps": mbytes / (kernel_ms * 1e-3) / 1e9, "hbm_peak_GBps": hbm_peak,
                    "frac_of_hbm": mbytes / (kernel_ms * 1e-3) / 1e9 / hbm_peak, "hbm_peak_source": hbm_src}
        unit = "positions/s" if mode else "deals/s"
        value = total * args.steps / (ms_max * 1e-3)
        cs = clk.summary()
        line = {
            "metric": unit, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "u64 (4-bit packed cards, integer only)", "data": "exhaustive rank space (deterministic, no sampling)",
            "config": {"workload": w["label"], "n": n, "mode": "canon" if mode else "deals", "ranks": total,
                       "parallelism": "shard%d" % ws, "l2": "working set in registers; no per-step input (L2 flush n/a)"},
            "turns_per_s": turns * ws / (ms_max * 1e-3 / args.steps),
            "turns_per_step": turns * ws,
            "kernel_ms": kernel_ms,
            "floyd_check_ms": (sum(floyd_ms[-args.steps:]) / args.steps) if floyd_ms else None,
            "gpu_launches": launches,
            "roofline": {"bound": "int_issue", "achieved": achieved / 1e12, "peak": issue_peak / 1e12,
                         "unit": "Tops/s (INT32 thread-ops)", "frac": achieved / issue_peak,
                         "alu_pipe_peak": alu_peak / 1e12, "frac_of_alu_pipe": achieved / alu_peak,
                         "ops_per_turn": K_OPS_PER_TURN,
                         "traffic": (MEMO_DRAM_BYTES_PER_DEAL * total / max(1, launches // args.steps)
                                     if memo and mode == 0 and n == 13 else None),
                         "traffic_unit": "DRAM bytes per launch (ncu capture scaled by deals per launch)",
                         "peak_source": "war_measure_int_peak on this GPU (LOP3+IMAD issue ceiling)"},
            "clocks": cs,
            "check": check,
            "tune": {k: getattr(tune, k) for k, _ in tune._fields_} if tune is not None else None,
        }
        if memo:
            line["memo"] = memo
        if e2e:
            line["e2e"] = e2e
        if plain:
            line["plain_kernel"] = plain
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(w)
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def verify(w, acc, res):
    """Bit-exact check against the reference's recorded values (data/checks.txt, data/long_runs.txt)."""
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        g = json.load(f)
    cyc, done, maxfin, turns, dmin, oncyc = acc
    n = w["n"]
    if w["mode"] == 0:
        e = g["deals_rule0"][str(n)]
        ok = (cyc, done, maxfin) == (e["cyc"], e["deals"], e["longest"])
        if res is not None and "hist" in e:
            ok = ok and {str(i): v for i, v in enumerate(res.hist[:w["hbins"]]) if v} == {k: v for k, v in e["hist"].items()}
    else:
        e = g["canon_rule0"][str(n)]
        ok = (cyc, done, maxfin) == (e["cycling"], e["positions"], e["longest"]) and dmin == e["distinct"]
    if not ok:
        raise SystemExit("RESULT MISMATCH: %r" % (acc,))
    return "bit-exact vs recorded reference output"


if __name__ == "__main__":
    main()
