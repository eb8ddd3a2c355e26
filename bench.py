"""Benchmark of the exhaustive War enumerator on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload deals13|canon14|deals11|deals13slice]
                    [--impl ours|reference] [--peaks]

One step = one complete enumeration of the workload's rank space by the persistent refill kernel
(war_enumerate), every step checked bit-exactly against the reference's recorded values.  Workloads (the
rank spaces are the inputs; nothing is random):
  deals13  all 13! = 6,227,020,800 deals, cycle-length and ending-length histograms   (default)
  canon14  all 13!*13 = 80,951,270,400 canonical positions of n = 14, distinct cycles, cycle-length
           histogram and the seeded 1% Floyd cross-check
  deals11  all 11! deals (plain GPU drop-in size)
The default line also carries the rest of the headline metric, measured after the timed region: the
batched-versus-plain ratio (the plain kernel on the same job), `canon14` (the reference's long run
`war_gpu.py 14 --canon --distinct --shape --hist 256` with the 1% Floyd sample, bit-exact against
data/long_runs.txt:20-23) and `serving` (a seeded Poisson stream of jobs below the server's capacity:
throughput, p50 / p99 job latency, every job checked against the plain kernel).
With N ranks (torchrun, one GPU each) the rank space is cut into N contiguous shards and the per-rank
results are summed with one all-reduce of the accumulators (strong scaling).  Rank 0 prints one JSON
line.  --impl reference times the reference's own CPU program (cpu/war.cpp, built unmodified into
oracle/_ref/) over the whole workload once, and the oracle's restatement of it on bounded strided
samples, on all host cores.  --peaks prints the measured ceilings (integer issue, random gathers) alone.
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
# DRAM bytes (read + write) per deal of the path-memo refill kernel at this line's configuration (all 13!
# deals, 16 GiB table): one-pass ncu capture of both launches of a timed step, 699.5 GB read and 11.4 GB
# written for 6,227,020,800 deals (112.3 + 1.8 B per deal); each random 8-byte lookup costs a DRAM line.
MEMO_DRAM_BYTES_PER_DEAL = 114.2
# Turns of the reference's own schedule (Brent with the tortoise saved at powers of two from the first turn)
# over all 13! deals, as counted by an instrumented copy of cpu/war.cpp; the plain kernel reproduces it
# exactly (its `turns`).
REF_SCHEDULE_TURNS = {13: 686746920144}

WORKLOADS = {
    "deals13": dict(n=13, mode=0, hbins=256, flags=0, label="n=13 all deals (war_gpu.py 13 --hist 256)"),
    "canon14": dict(n=14, mode=1, hbins=256, dbins=4096, flags=2 | 8, sample_ppm=10000, seed=14,
                    label="n=14 canonical positions, --distinct, --hist 256, 1% Floyd sample"),
    "deals11": dict(n=11, mode=0, hbins=256, flags=0, label="n=11 all deals"),
    # a 2e8-deal slice from the middle of the n = 13 space (profiling size)
    "deals13slice": dict(n=13, mode=0, hbins=256, flags=0, lo=3013510400, hi=3213510400,
                         label="n=13 deals, ranks [3013510400, 3213510400)"),
    # the reference's recorded 17-card slice (data/long_runs.txt:61-64: war24.py 17 --start 10^14 --count 10^9)
    # on the 5-bit engine with each cycle test, and on the held-out-card engine
    "wide17": dict(n=17, mode=0, hbins=0, flags=0, lo=10 ** 14, hi=10 ** 14 + 10 ** 9, engine="wide", det=2,
                   label="n=17 deals [1e14, 1e14+1e9), war24.py 17 --det streak (5-bit engine)"),
    "wide17floyd": dict(n=17, mode=0, hbins=0, flags=0, lo=10 ** 14, hi=10 ** 14 + 10 ** 9, engine="wide", det=1,
                        label="n=17 deals [1e14, 1e14+1e9), war24.py 17 --det floyd (5-bit engine)"),
    "wide17brent": dict(n=17, mode=0, hbins=0, flags=0, lo=10 ** 14, hi=10 ** 14 + 10 ** 9, engine="wide", det=0,
                        label="n=17 deals [1e14, 1e14+1e9), Brent (5-bit engine)"),
    "held17": dict(n=17, mode=0, hbins=0, flags=0, lo=10 ** 14, hi=10 ** 14 + 10 ** 9, engine="held",
                   label="n=17 deals [1e14, 1e14+1e9), war17.py engine (card n-1 held out)"),
}
# Algorithmic integer operations per turn of the other engines, counted from their source like K_OPS_PER_TURN:
# the 5-bit turn on 128-bit piles (two 128-bit pops 8, cards and compare 3, pair 3, position 2, the clamped
# 128-bit shift of the pair 12, the masked XOR into four words 9, length 2: 39) plus Brent's four-word test and
# bookkeeping (13) and the end test (2); the held-out turn is counted like the 4-bit turn.
K_OPS_PER_TURN_ENGINE = {"refill": K_OPS_PER_TURN, "wide": 54, "held": K_OPS_PER_TURN}


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
    """The reference's CPU implementation on the host cores (rank 0 only).

    Deals: the reference's own cpu/war.cpp (built unmodified into oracle/_ref/) over the whole workload once,
    `war 13 0` (about 70 s on 16 threads); its rate is the line's value.  Beside it, the oracle's restatement
    of the same algorithm is timed on bounded strided samples for the requested steps (each a few seconds),
    and its calibration against the full run is reported.  Canonical positions: the reference has no CPU
    program that fits the time (cpu/distinct_cycles.c takes tens of minutes at n = 14), so the samples of the
    restatement are the value."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    w = WORKLOADS[args.workload]
    n, mode = w["n"], w["mode"]
    cores = os.cpu_count() or 1
    total = space(n, mode)
    unit = "positions/s" if mode else "deals/s"
    line = {"impl": "reference", "metric": unit, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "u64", "data": "exhaustive (deterministic rank space)",
            "config": {"workload": w["label"], "n": n, "mode": "canon" if mode else "deals"}}
    full = None
    if mode == 0 and "lo" not in w and oracle.ref_available("war"):
        oracle.ref_war(min(n, 11), 0)                                  # warm-up: page cache, thread pool
        t0 = time.time()
        deals, cyc, longest = oracle.ref_war(n, 0)
        t_full = time.time() - t0
        assert deals == total, (deals, total)
        full = {"value": total / t_full, "seconds": t_full, "cores": cores, "cycling": cyc, "longest": longest,
                "sample": "full run of the unmodified cpu/war.cpp: war %d 0 (%d deals)" % (n, total)}
    # bounded strided samples of the same rank space with the restatement, ~60 s in all
    per_step = 60.0 / max(1, args.steps + 1)
    _oracle_sample_rate(w, min(per_step, 5.0), cores)                   # warm-up
    times, done_units = [], 0
    for s in range(args.steps):
        v, slice_len, _ = _oracle_sample_rate(w, per_step, cores, seed=s + 1)
        times.append(slice_len * 64 / v)
        done_units += slice_len * 64
    port = done_units / sum(times)
    port_line = {"value": port, "steps": args.steps, "ms_per_step": sum(times) / len(times) * 1e3,
                 "sample": "64 strided slices of %d ranks of the %s space per step, oracle/war_oracle.c "
                           "(restatement of the reference algorithm, OpenMP on all host threads)" % (
                               slice_len, "canonical-position" if mode else "deal")}
    if full:
        v, t = full["value"], full["seconds"]
        port_line["calibration_vs_reference"] = port / v
        line.update({"steps": 1, "steps_requested": args.steps, "warmup": 1, "value": v, "ms_per_step": t * 1e3,
                     "cpu_baseline": {"value": v, "unit": unit, "cores": cores, "kind": "reference",
                                      "sample": full["sample"]},
                     "reference_full": full, "port_samples": port_line})
    else:
        line.update({"value": port, "ms_per_step": port_line["ms_per_step"],
                     "cpu_baseline": {"value": port, "unit": unit, "cores": cores, "kind": "port",
                                      "sample": port_line["sample"]}})
    line["e2e"] = {"value": line["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)


def _oracle_sample_rate(w, target_s, cores, seed=0):
    """Times the oracle's restatement of the reference algorithm on a strided sample of the workload's
    rank space (64 slices spread evenly), sized by a short probe to take about target_s seconds.  Returns
    (ranks per second, ranks per slice, seconds the sample took)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    n, mode = w["n"], w["mode"]
    total = space(n, mode)

    engine = w.get("engine", "refill")
    # the space the workload samples: its own slice for the 17-card workloads, else the whole rank space
    base, total = (w["lo"], w["hi"] - w["lo"]) if engine != "refill" else (0, total)

    def run(slice_len):
        t0 = time.time()
        for i in range(64):
            lo = base + (total // 64) * i + (seed * 7919) % max(1, total // 64 - slice_len)
            job = oracle.make_job(n, mode, 0, w["flags"] & ~8, lo, min(base + total, lo + slice_len), hbins=w["hbins"],
                                  dbins=w.get("dbins", 0))
            if engine == "held":      # the restatement of gpu/war17.py
                oracle.enumerate_held(job, cores)
            elif engine == "wide":    # the restatement of gpu/war24.py with the workload's cycle test
                oracle.war24(job, det=w["det"], window=32 if w["det"] == 0 else 1, threads=cores)
            else:                     # the restatement of cpu/war.cpp / gpu/war_gpu.py
                oracle.enumerate_job(job, cores)
        return time.time() - t0

    # grow the probe until it runs long enough for the per-call overhead not to dominate its rate
    probe, cap = 4096, max(4096, total // 64)
    dt = run(probe)
    while dt < min(1.0, target_s / 4) and probe < cap:
        probe = min(cap, probe * 4)
        dt = run(probe)
    slice_len = min(cap, max(probe, int(probe * target_s / max(dt, 1e-3))))
    dt = run(slice_len)
    return slice_len * 64 / dt, slice_len, dt


def cpu_baseline(w, target_s=12.0):
    """The oracle's restatement of the reference algorithm on a bounded strided sample (all host threads)."""
    cores = os.cpu_count() or 1
    v, slice_len, dt = _oracle_sample_rate(w, target_s, cores)
    mode = w["mode"]
    what = {"held": "gpu/war17.py's", "wide": "gpu/war24.py's"}.get(w.get("engine"), "cpu/war.cpp's")
    return {"value": v, "unit": "positions/s" if mode else "deals/s", "cores": cores, "kind": "port",
            "sample": "64 strided slices of %d ranks of the %s, oracle/war_oracle.c (restatement of "
                      "%s algorithm, OpenMP on all host threads), %.1f s" % (
                          slice_len, "workload's slice" if "engine" in w else
                          ("canonical-position space" if mode else "deal space"), what, dt)}


def deal_extra_units(lo, hi, m):
    """How many extra work units the engines copy to the device for deals [lo, hi): the aligned blocks of j!
    ranks (j <= m) that cover the ragged ends around the main units of m! ranks (war_plan)."""
    f = math.factorial

    def blocks(x, y):
        k = 0
        while x < y:
            j = m
            while j > 0 and (x % f(j) or x + f(j) > y):
                j -= 1
            x += f(j)
            k += 1
        return k
    a2, b2 = -(-lo // f(m)) * f(m), hi // f(m) * f(m)
    return blocks(lo, a2) + blocks(b2, hi) if a2 < b2 else blocks(lo, hi)


def peaks(warlib, table_bits, clk_mhz=None):
    """The measured ceilings on this GPU: integer issue (LOP3+IMAD), the ALU pipe alone, random 8-byte and
    32-byte gathers from a table of 2^table_bits words, and the nominal issue rate (SMs x 4 schedulers x 32
    lanes x SM clock)."""
    issue, alu = warlib.measure_int_peak()
    info = warlib.device_info()
    clk = clk_mhz or info.clock_mhz
    return {"int_issue_ops_per_s": issue, "alu_ops_per_s": alu,
            "nominal_issue_ops_per_s": info.sm_count * 4 * 32 * clk * 1e6, "sm_count": info.sm_count,
            "clock_mhz": clk, "gather_table_bytes": 8 << table_bits,
            "gather8_lookups_per_s": warlib.measure_gather_peak(table_bits, 8),
            "gather32_lookups_per_s": warlib.measure_gather_peak(table_bits, 32)}


def canon14_leg(warlib, war_gpu, golden, stream):
    """The reference's long run `war_gpu.py 14 --canon --distinct --shape --hist 256` (data/long_runs.txt:20-23)
    with the seeded 1% sample of the north-star's canonical configuration: every canonical position of n = 14
    once per rep through war_enumerate (device time, CUDA events on the launching stream), checked
    bit-exactly, then the sample replayed with Floyd and compared with Brent's aggregates."""
    import torch
    F = warlib.F_DISTINCT | warlib.F_SHAPE | warlib.F_SAMPLE
    tune = war_gpu._tune_for(14, True, 0, F)
    job = warlib.make_job(14, warlib.CANON, 0, F, hbins=256, dbins=4096, sample_ppm=10000, seed=14)
    warlib.enumerate_job(warlib.make_job(14, warlib.CANON, 0, F, 0, 10 ** 8, hbins=256, dbins=4096,
                                         sample_ppm=10000, seed=14), tune)        # untimed: first launch
    g = golden["canon_rule0"]["14"]
    dh = {int(k): v for k, v in g["dhist"].items()}
    hh = {int(k): v for k, v in g["hist"].items()}
    ms = []
    for _ in range(2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = warlib.enumerate_job(job, tune)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        d = warlib.to_dict(r)
        ok = ((d["cyc"], d["done"], d["maxfin"], d["distinct_min"], d["dhist"], d["hist"], d["shape_nonstd"],
               d["shape_unchecked"]) == (g["cycling"], g["positions"], g["longest"], g["distinct"], dh, hh,
                                         g["shape_nonstd"], g["shape_unchecked"]))
        if not ok:
            raise SystemExit("canon14 RESULT MISMATCH: %r" % ({k: d[k] for k in ("cyc", "done", "maxfin")},))
    f = warlib.floyd_sample(job)
    key = lambda x: (x.s_count, x.s_cyc, x.s_lamsum, x.s_lensum, x.s_maxfin)
    if key(f) != key(r):
        raise SystemExit("canon14 Floyd sample disagrees with Brent")
    t = min(ms)
    return {"workload": "n=14 canonical positions, war_gpu.py 14 --canon --distinct --shape --hist 256, "
                        "1% seeded Floyd sample", "positions": g["positions"], "value": g["positions"] / (t * 1e-3),
            "unit": "positions/s", "ms": t, "ms_reps": ms, "floyd_sample_ms": f.kernel_ms,
            "floyd_sample_positions": f.s_count, "turns": r.turns, "memo_hit_rate": r.memo_hits / max(1, r.memo_lookups),
            "check": "bit-exact vs data/long_runs.txt:20-23 (cycling, longest, distinct, weights, shape, lengths); "
                     "Floyd sample = Brent sample",
            "reference_published_s": 596.6, "tune": {k: getattr(tune, k) for k, _ in tune._fields_}}


def serving_leg(warlib, jobs, rate, seed=2026):
    """A seeded Poisson stream of the serving workload below the server's capacity: throughput over the
    stream, job latency (submit to result) percentiles, and every job against the plain kernel."""
    import serve
    stream = serve.poisson_stream(jobs, rate, seed)
    with serve.Server() as s:
        results, lat, wall = serve.serve_stream(stream, s)
        st = s.stats()
        mi = s.memo_info()
    ranks = sum(j.hi - j.lo for _, j in stream)
    t0 = time.time()
    bad = serve.verify(stream, results)
    return {"workload": "serving: %d seeded Poisson jobs at %.0f/s (n uniform over 9,10,11,13,14,15; 70%% deals; "
                        "20%% loser-first; half of the canonical jobs --distinct; log-uniform 1e4..1e9 ranks)"
                        % (jobs, rate),
            "jobs": jobs, "ranks": ranks, "wall_s": wall, "offered_ranks_per_s": ranks / stream[-1][0],
            "ranks_per_s": ranks / wall, "latency_ms": {"p50": serve.percentile(lat, 50),
                                                        "p99": serve.percentile(lat, 99), "max": max(lat)},
            "server": st, "memo_arena": mi, "mismatches_vs_plain": bad, "verify_s": time.time() - t0}


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
    ap.add_argument("--no-canon14", action="store_true", help="skip the n = 14 canonical leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--serving-jobs", type=int, default=600)
    ap.add_argument("--serving-rate", type=float, default=20.0)
    ap.add_argument("--tune", default=None,
                    help='JSON object overriding fields of the stored tune of the refill engine, e.g. '
                         '\'{"variant": 3}\' (the line reports the tune it ran)')
    ap.add_argument("--peaks", action="store_true", help="print the measured ceilings only")
    ap.add_argument("--table-bits", type=int, default=30, help="--peaks: gather table of 2^bits words")
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
    if args.peaks:
        print(json.dumps(peaks(warlib, args.table_bits)), flush=True)
        return
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        golden = json.load(f)
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
    engine = w.get("engine", "refill")
    # the 17-card engines run with their own defaults (war_enumerate_held / war_enumerate_wide, tune NULL)
    tune = war_gpu._tune_for(n, mode == 1, 0, w["flags"]) if engine == "refill" else None
    if args.tune and engine == "refill":
        tune = war_gpu.override_tune(tune, json.loads(args.tune))

    floyd_ms = []

    def step():
        if engine == "wide":
            return warlib.enumerate_wide(job, w["det"])
        if engine == "held":
            return warlib.enumerate_held(job)
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
    res = results[-1]
    check = "slice (no recorded total)"
    for r in results:                  # every timed step, bit-exact
        acc = [r.cyc, r.done, r.maxfin, r.turns, r.distinct_min, r.oncycle]
        hist = {i: int(v) for i, v in enumerate(r.hist[:w["hbins"]]) if v}
        if ws > 1:   # the one exchange of the sharded path: combine the per-rank results
            d = shard.allreduce_result(shard.result_to_dict(r), device="cuda")
            acc = [d["cyc"], d["done"], d["maxfin"], d["turns"], d["distinct_min"], d["oncycle"]]
            hist = {int(k): v for k, v in d["hist"].items() if int(k) < w["hbins"]}
        if "lo" not in w:
            check = verify(w, acc, hist, golden)
        elif engine in ("wide", "held") and ws == 1:
            rec = [e for e in golden["war24"] if (e["n"], e["lo"], e["hi"]) == (n, lo0, hi0)]
            if not rec or (r.cyc, r.done, r.maxfin, r.undetermined) != (rec[0]["cyc"], rec[0]["deals"],
                                                                        rec[0]["longest"], rec[0]["undetermined"]):
                raise SystemExit("RESULT MISMATCH: %r" % ((r.cyc, r.done, r.maxfin, r.undetermined),))
            check = "bit-exact vs the recorded war24.py run (data/long_runs.txt:63-64)"

    # e2e through the public drop-in API (war_gpu.run), host structs in, host results out, every copy inside
    # the timed region; its result is checked against the recorded one
    e2e = None
    if not args.no_e2e:
        kw = dict(hbins=w["hbins"], canon=mode == 1, dbins=w.get("dbins", 0), quiet=True)
        warlib.set_stream(0)

        def e2e_step():
            if engine != "refill":
                step()
            elif ws == 1 and "lo" not in w:
                out = war_gpu.run(n, **kw)
                dmin = sum(v // k for k, v in out[6].items()) if out[6] else None
                verify(w, [out[0], out[1], out[2], None, dmin, None], out[4] if mode == 0 else None, golden)
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
        # per step: the extra work units copied in for each engine call, and the accumulator block read back
        spans = []
        if ws == 1 and "lo" not in w:
            mult = (n - 1) if mode else 1
            orders = hi0 // mult
            span = max(war_gpu.SPAN_RANKS // mult, 1)
            spans = [(a * mult, min(orders, a + span) * mult) for a in range(0, orders, span)]
        else:
            spans = [(lo, hi)]
        h2d = 0
        for a, b in spans:
            if mode == 0:
                h2d += 24 * deal_extra_units(a, b, min(n, tune.block_m if tune else 6))
            else:
                h2d += 24 * len(warlib.plan(warlib.make_job(n, mode, 0, w["flags"], a, b), tune.block_m)[2])
        import serve
        d2h = serve.SIZEOF_DEVACC * len(spans)
        e2e = {"value": total / e2e_s, "unit": "positions/s" if mode else "deals/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "api": "war_gpu.run" if ws == 1 else "warlib.enumerate_job",
               "check": "result tuple equal to the recorded one" if ws == 1 and "lo" not in w else None}

    # the plain kernel (the reference's per-thread rank blocks, restated for sm_100a) on the same job,
    # once, outside the timed region: the batched-versus-plain ratio
    plain = None
    warlib.set_stream(stream.cuda_stream)
    if not args.no_plain and ws == 1 and engine == "refill":
        rp = warlib.enumerate_plain(job)
        assert (rp.cyc, rp.done, rp.maxfin) == (res.cyc, res.done, res.maxfin), "plain and refill kernels disagree"
        plain = {"value": (hi - lo) / (rp.kernel_ms * 1e-3), "kernel_ms": rp.kernel_ms, "turns": rp.turns,
                 "batched_over_plain": rp.kernel_ms / kernel_ms}

    c14 = None
    if rank == 0 and ws == 1 and args.workload == "deals13" and not args.no_canon14:
        c14 = canon14_leg(warlib, war_gpu, golden, stream)
    serving = None
    if rank == 0 and ws == 1 and args.workload == "deals13" and not args.no_serving:
        serving = serving_leg(warlib, args.serving_jobs, args.serving_rate)

    if rank == 0:
        cs = clk.summary()
        pk = peaks(warlib, (tune.memo_bits or 24) if tune is not None and (tune.variant & 4) else 30,
                   clk_mhz=cs["sm_mhz"])
        issue_peak, alu_peak, nominal = pk["int_issue_ops_per_s"], pk["alu_ops_per_s"], pk["nominal_issue_ops_per_s"]
        kops = K_OPS_PER_TURN_ENGINE[engine]
        achieved = turns * kops / (kernel_ms * 1e-3)    # algorithmic int ops/s of the enumeration kernel
        memo = None
        if tune is not None and (tune.variant & 4) and res.memo_lookups:
            # the cycle memo's own traffic: one 8-byte word read per lookup, one written per store
            hbm_peak, hbm_src = measured_hbm_peak()
            mbytes = 8.0 * (res.memo_lookups + res.memo_stores)
            lps = res.memo_lookups / (kernel_ms * 1e-3)
            memo = {"variant": tune.variant, "table_bytes": 8 << (tune.memo_bits or 24),
                    "lookups_per_game": res.memo_lookups / res.done, "hit_rate": res.memo_hits / res.memo_lookups,
                    "stores_per_game": res.memo_stores / res.done, "turns_per_game": res.turns / res.done,
                    "lookups_per_s": lps, "gather_peak_lookups_per_s": pk["gather8_lookups_per_s"],
                    "frac_of_gather_peak": lps / pk["gather8_lookups_per_s"],
                    "algorithmic_bytes_per_lookup": 8,
                    "dram_bytes_per_deal": MEMO_DRAM_BYTES_PER_DEAL if mode == 0 and n == 13 else None,
                    "algorithmic_GBps": mbytes / (kernel_ms * 1e-3) / 1e9, "hbm_peak_GBps": hbm_peak,
                    "frac_of_hbm": mbytes / (kernel_ms * 1e-3) / 1e9 / hbm_peak, "hbm_peak_source": hbm_src}
        # The integer-issue roofline of the turns (north-star's report: turns x ops per turn against the measured
        # LOP3+IMAD ceiling and the nominal issue rate) and, for the memo kernel, the roofline that binds it:
        # random 8-byte table reads against the measured random-gather ceiling of this GPU.
        int_issue = {"achieved": achieved / 1e12, "peak": issue_peak / 1e12, "unit": "Tops/s (INT32 thread-ops)",
                     "frac": achieved / issue_peak, "peak_nominal": nominal / 1e12, "frac_of_nominal": achieved / nominal,
                     "alu_pipe_peak": alu_peak / 1e12, "frac_of_alu_pipe": achieved / alu_peak, "ops_per_turn": kops,
                     "turns_per_launch": turns / max(1, launches // args.steps),
                     "peak_source": "war_measure_int_peak on this GPU (LOP3+IMAD issue ceiling, measured); "
                                    "nominal = SMs x 4 x 32 x median SM clock"}
        per_launch = total / max(1, launches // args.steps)
        if memo:
            roofline = {"bound": "hbm_random_access", "achieved": memo["lookups_per_s"] / 1e9,
                        "peak": memo["gather_peak_lookups_per_s"] / 1e9, "unit": "G lookups/s (random 8-byte reads)",
                        "frac": memo["frac_of_gather_peak"],
                        "traffic": (MEMO_DRAM_BYTES_PER_DEAL * per_launch if mode == 0 and n == 13 else None),
                        "traffic_unit": "DRAM bytes per launch (ncu capture scaled by deals per launch)",
                        "algorithmic_bytes_per_launch": 8.0 * (res.memo_lookups + res.memo_stores) / max(
                            1, launches // args.steps),
                        "peak_source": "war_measure_gather_peak on this GPU (random ld.global.cg of 8 bytes from a "
                                       "table of the memo's size, measured)",
                        "int_issue": int_issue}
            if mode == 0 and n == 13:
                # the same kernel against the copy bandwidth: its algorithmic bytes (8 per lookup or store) and
                # the DRAM bytes it actually moves (ncu, per deal), per second of kernel time
                hbm_peak, hbm_src = measured_hbm_peak()
                dram_gbs = MEMO_DRAM_BYTES_PER_DEAL * total / (kernel_ms * 1e-3) / 1e9
                roofline["hbm"] = {"achieved_algorithmic_GBps": memo["algorithmic_GBps"],
                                   "achieved_dram_GBps": dram_gbs, "peak_GBps": hbm_peak,
                                   "frac_algorithmic": memo["algorithmic_GBps"] / hbm_peak,
                                   "frac_dram": dram_gbs / hbm_peak, "peak_source": hbm_src}
        else:
            roofline = dict(int_issue, bound="int_issue", traffic=None,
                            traffic_unit="DRAM bytes per launch: accumulators only (no table)")
        unit = "positions/s" if mode else "deals/s"
        value = total * args.steps / (ms_max * 1e-3)
        step_s = ms_max * 1e-3 / args.steps
        line = {
            "metric": unit, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "u64 (4-bit packed cards, integer only)", "data": "exhaustive rank space (deterministic, no sampling)",
            "config": {"workload": w["label"], "n": n, "mode": "canon" if mode else "deals", "ranks": total,
                       "parallelism": "shard%d" % ws, "l2": "working set in registers; no per-step input (L2 flush n/a)"},
            "turns_per_s": turns * ws / step_s,
            "turns_per_step": turns * ws,
            "turns_ref_schedule_per_s": (REF_SCHEDULE_TURNS[n] / step_s if mode == 0 and n in REF_SCHEDULE_TURNS
                                         and "lo" not in w else None),
            "kernel_ms": kernel_ms,
            "floyd_check_ms": (sum(floyd_ms[-args.steps:]) / args.steps) if floyd_ms else None,
            "gpu_launches": launches,
            "roofline": roofline,
            "peaks": pk,
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
        if c14:
            line["canon14"] = c14
        if serving:
            line["serving"] = serving
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(w)
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def verify(w, acc, hist, g):
    """Bit-exact check against the reference's recorded values (data/checks.txt, data/long_runs.txt); hist is
    the cycle-length histogram as {bin: count} (all ranks combined), or None."""
    cyc, done, maxfin, turns, dmin, oncyc = acc
    n = w["n"]
    if w["mode"] == 0:
        e = g["deals_rule0"][str(n)]
        ok = (cyc, done, maxfin) == (e["cyc"], e["deals"], e["longest"])
        if hist is not None and "hist" in e:
            ok = ok and {str(k): v for k, v in hist.items()} == {k: v for k, v in e["hist"].items()}
    else:
        e = g["canon_rule0"][str(n)]
        ok = (cyc, done, maxfin) == (e["cycling"], e["positions"], e["longest"]) and dmin == e["distinct"]
    if not ok:
        raise SystemExit("RESULT MISMATCH: %r" % (acc,))
    return "bit-exact vs recorded reference output"


if __name__ == "__main__":
    main()
