"""Sharding a job's rank space across processes (one per GPU) and combining their results.

Ranks are independent, so rank r of N takes the contiguous slice [lo + len*r/N, lo + len*(r+1)/N) and
plays it alone; the only exchange is one all-reduce of the result counters at the end (sums for the
counts and histograms, maximum for the longest games).  Works with any torch.distributed backend: NCCL
between GPUs, gloo on the CPU (tests).
"""

SUM_FIELDS = ("cyc", "done", "turns", "oncycle", "distinct_min", "shape_nonstd", "shape_unchecked",
              "s_count", "s_cyc", "s_lamsum", "s_lensum")
MAX_FIELDS = ("maxfin", "s_maxfin")
HISTS = (("hist", 4096), ("dhist", 4096), ("endhist", 1024))


def shard_range(lo, hi, rank, world):
    """The contiguous slice of [lo, hi) that rank `rank` of `world` plays."""
    if not (0 <= rank < world) or lo > hi:
        raise ValueError("bad shard request")
    span = hi - lo
    return lo + span * rank // world, lo + span * (rank + 1) // world


def result_to_dict(r):
    """A war_result-like object (ctypes struct) as {field: int, hist: {bin: count}, ...}."""
    d = {k: int(getattr(r, k)) for k in SUM_FIELDS + MAX_FIELDS}
    for name, bins in HISTS:
        arr = getattr(r, name)
        d[name] = {i: int(v) for i, v in enumerate(arr[:bins]) if v}
    return d


def allreduce_result(d, device="cpu"):
    """Sums the counters and histograms and takes the maxima of d across the default process group."""
    import torch
    import torch.distributed as dist
    vec = [d[k] for k in SUM_FIELDS]
    for name, bins in HISTS:
        h = [0] * bins
        for k, v in d[name].items():
            h[int(k)] = v
        vec += h
    t = torch.tensor(vec, dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    m = torch.tensor([d[k] for k in MAX_FIELDS], dtype=torch.int64, device=device)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    t, m = t.tolist(), m.tolist()
    out = dict(zip(SUM_FIELDS, t[:len(SUM_FIELDS)]))
    out.update(zip(MAX_FIELDS, m))
    pos = len(SUM_FIELDS)
    for name, bins in HISTS:
        out[name] = {i: v for i, v in enumerate(t[pos:pos + bins]) if v}
        pos += bins
    return out
