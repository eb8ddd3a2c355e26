"""Autotuner for the persistent refill kernel (war_enumerate).

For one (n, mode, rule, flag class) it times the kernel on a representative contiguous slice of the rank
space (about `slice_s` seconds of work, taken from the middle of the space) and searches, one coordinate
at a time, over
    block_m        work-unit size: m! consecutive orders per unit        (4..8)
    games          games in flight per thread                            (1, 2, 4)
    chunk          units a lane takes from the work counter at a time: chunks of chunk x m! consecutive ranks
                   (1 .. 1456: with m = 6 from 720 to 2^20 ranks)
    threads        block size                                            (128..1024)
    blocks_per_sm  resident blocks (0 = as many as fit)
    window         Brent's first tortoise window                         (8..128)
    defer          immediate records: lanes that wait before the warp refills; latched records: turns
                   between services                                      (1..32)
    variant        bit 0: multiply-add turn form; bit 1: latched records serviced every `defer` iterations;
                   bit 2: cycle memo (deals); bit 3: the memo holds every cycle state; bit 4: and paths
    memo_bits      log2 of the memo table's 8-byte words                 (26..31)
Every configuration must return exactly the same counts as the first one; a mismatch raises.  The best
configuration is stored in tune_cache.json next to this file, keyed by GPU name, n, mode, rule and flags.

The cycle memo is cleared per job and pays only once it has warmed up, so a short slice favours the
variants without it: tune memo configurations on the whole space (--full) or on a long slice.

    python autotune.py 13                         deals, n = 13 (its whole space takes well under a second)
    python autotune.py 14 --canon --distinct --full
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import warlib  # noqa: E402

CACHE = os.path.join(HERE, "tune_cache.json")
SPACE = {
    "block_m": [4, 5, 6, 7, 8],
    "games": [1, 2, 4],
    "chunk": [1, 8, 64, 512, 1456],
    "threads": [128, 256, 512, 1024],
    "blocks_per_sm": [0, 1, 2, 3, 4],
    "window": [8, 16, 32, 64, 128],
    "defer": [1, 2, 4, 6, 8, 12, 16, 24, 32],
    "variant": [0, 1, 2, 3, 6, 7, 14, 15, 30, 31],
    "memo_bits": [26, 28, 29, 30, 31],
}
DEFAULT = {"block_m": 5, "games": 2, "threads": 512, "blocks_per_sm": 0, "window": 32, "defer": 8, "variant": 1,
           "memo_bits": 24, "chunk": 1}


_device_name = None
_cache = {"mtime": None, "data": {}}


def key(n, mode, rule, flags, device=None):
    global _device_name
    if device is None:
        if _device_name is None:      # the device's properties once per process (the query takes milliseconds)
            _device_name = warlib.device_info().name.decode()
        device = _device_name
    return "%s|n=%d|mode=%d|rule=%d|flags=%d" % (device, n, mode, rule, flags & ~(warlib.F_SAMPLE | warlib.F_MEMO_KEEP))


def load_cache():
    """The stored tunes, re-read only when the file changed."""
    if not os.path.exists(CACHE):
        return {}
    m = os.path.getmtime(CACHE)
    if _cache["mtime"] != m:
        with open(CACHE) as f:
            _cache["data"] = json.load(f)
        _cache["mtime"] = m
    return _cache["data"]


def default_tune(n, mode, rule, flags):
    """The tune for a job class with no stored entry: the path memo with a table that grows with n (the
    n = 13 deal and n = 14 canonical measurements: 6! (deals) or 5! x splits (canonical) work units,
    services every 8 (deals) or 16 (canonical) turns, one game per lane); none below 4 cards."""
    if n < 4:
        return None
    # from 13 cards a 2^31-word table (16 GiB): all 13! deals 166.0 ms against 170.7 ms at 2^30
    bits = {4: 12, 5: 12, 6: 14, 7: 16, 8: 18, 9: 20, 10: 22, 11: 24, 12: 27}.get(n, 31)
    variant = 31 if n <= 16 else 3   # the path memo up to 16 cards (it loses on 17-card slices)
    if mode == warlib.CANON:
        return {"block_m": min(5, n - 1), "blocks_per_sm": 0, "defer": 16, "games": 1, "threads": 512,
                "window": 128, "variant": variant, "memo_bits": bits}
    return {"block_m": min(6, n), "blocks_per_sm": 0, "defer": 8, "games": 1, "threads": 256, "window": 32,
            "variant": variant, "memo_bits": bits}


def cached_tune(n, mode, rule, flags):
    """The stored best war_tune for this job class on this GPU, else default_tune(), or None."""
    c = load_cache().get(key(n, mode, rule, flags))
    t = c["tune"] if c else default_tune(n, mode, rule, flags)
    if not t:
        return None
    return warlib.make_tune(t["threads"], t["blocks_per_sm"], t["games"], t["block_m"], t["window"], t["defer"],
                            t.get("variant", 0), t.get("memo_bits", 0), t.get("chunk", 0))


def _legal(n, mode, flags, cfg):
    if mode == warlib.CANON and (flags & warlib.F_DISTINCT) and cfg["window"] < 128:
        return False          # the free on-cycle test needs a first window at least as long as the cycles
    if cfg["games"] == 2 and cfg["threads"] > 512:
        return False
    if cfg["games"] == 4 and (cfg["threads"] > 256 or cfg["variant"] not in (3, 31)):
        return False
    return cfg["block_m"] <= (n - 1 if mode else n)


def _slice(n, mode, rule, flags, slice_s, cfg):
    """A contiguous slice from the middle of the space taking about slice_s seconds.  The probe that
    sizes it grows until it runs long enough (>= 50 ms) for the launch tail not to dominate."""
    total = warlib.space_size(n, mode)
    if total <= 5e7:
        return 0, total
    size = 1 << 26
    while True:
        lo = max(0, total // 2 - size // 2)
        probe = warlib.make_job(n, mode, rule, flags, lo, min(total, lo + size))
        r = warlib.enumerate_job(probe, warlib.make_tune(**cfg))
        if r.kernel_ms >= 50 or size >= total:
            break
        size = min(total, size * 4)
    rate = (probe.hi - probe.lo) / max(r.kernel_ms * 1e-3, 1e-6)
    size = min(total, int(rate * slice_s))
    lo = max(0, total // 2 - size // 2)
    return lo, min(total, lo + size)


def measure(job, cfg, reps=2):
    t = warlib.make_tune(**cfg)
    best = None
    res = None
    for _ in range(reps):
        r = warlib.enumerate_job(job, t)
        ms = r.kernel_ms
        best = ms if best is None else min(best, ms)
        res = (r.cyc, r.done, r.maxfin, r.distinct_min, r.oncycle)
    return best, res


def autotune(n, mode=warlib.DEALS, rule=0, flags=0, slice_s=0.4, passes=2, verbose=True, dims=None):
    cur = dict(DEFAULT)
    if mode == warlib.CANON:
        cur.update(block_m=5, window=128 if flags & warlib.F_DISTINCT else 64)
    stored = load_cache().get(key(n, mode, rule, flags))
    if stored:   # start from the stored best
        cur.update(stored["tune"])
    elif default_tune(n, mode, rule, flags):
        cur.update(default_tune(n, mode, rule, flags))
    lo, hi = _slice(n, mode, rule, flags, slice_s, cur)
    job = warlib.make_job(n, mode, rule, flags, lo, hi, hbins=256, dbins=4096 if flags & warlib.F_DISTINCT else 0)
    best_ms, ref = measure(job, cur)
    log = [(dict(cur), best_ms)]
    for _ in range(passes):
        improved = False
        for name, values in SPACE.items():
            if dims and name not in dims:
                continue
            for v in values:
                if v == cur[name]:
                    continue
                cfg = dict(cur, **{name: v})
                if not _legal(n, mode, flags, cfg):
                    continue
                try:
                    ms, res = measure(job, cfg)
                except warlib.WarError as e:
                    if verbose:
                        print("skip", cfg, e)
                    continue
                if res != ref:
                    raise AssertionError("configuration %r changed the counts: %r != %r" % (cfg, res, ref))
                log.append((cfg, ms))
                if verbose:
                    print("%-90s %8.2f ms" % (cfg, ms), flush=True)
                if ms < best_ms * 0.995:
                    best_ms, cur, improved = ms, cfg, True
        if not improved:
            break
    rate = (hi - lo) / (best_ms * 1e-3)
    entry = {"tune": cur, "ms": best_ms, "ranks": hi - lo, "rate": rate, "slice": [lo, hi],
             "when": time.strftime("%Y-%m-%d %H:%M:%S"), "tried": len(log)}
    cache = load_cache()
    cache[key(n, mode, rule, flags)] = entry
    with open(CACHE, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    return entry


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("n", type=int)
    ap.add_argument("--canon", action="store_true")
    ap.add_argument("--rule", type=int, default=0)
    ap.add_argument("--distinct", action="store_true")
    ap.add_argument("--shape", action="store_true")
    ap.add_argument("--slice-s", type=float, default=0.4)
    ap.add_argument("--full", action="store_true", help="time every configuration on the whole space")
    ap.add_argument("--passes", type=int, default=2)
    ap.add_argument("--dims", default=None, help="comma-separated dimensions to search (default: all)")
    a = ap.parse_args()
    flags = (warlib.F_DISTINCT if a.distinct else 0) | (warlib.F_SHAPE if a.shape else 0)
    e = autotune(a.n, warlib.CANON if a.canon else warlib.DEALS, a.rule, flags, 1e9 if a.full else a.slice_s,
                 a.passes, dims=a.dims.split(",") if a.dims else None)
    print(json.dumps(e))


if __name__ == "__main__":
    main()
