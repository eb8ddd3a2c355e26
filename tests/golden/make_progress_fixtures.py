"""Writes the progress-file fixtures tests/golden/progress_*.json: interrupted runs of gpu/war_gpu.py, in the
exact schema its run() writes (gpu/war_gpu.py:331-338, same keys in the same order), with the accumulators of
the ranks before next_start computed by the oracle (the CPU restatement of the reference's kernels).  The
drop-in's --resume must take such a file, written by the reference, and finish the run to the recorded
totals.  next_start is where the reference itself would have stopped: a whole number of its launch spans
(batch_threads * per orders, gpu/war_gpu.py:274-278, :313).

    python tests/golden/make_progress_fixtures.py          (about a minute on 8 cores)
"""
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402


def ref_span(n, canon, per=256, threads=256, batch_threads=1 << 18):
    """The reference's launch span in orders (deals, or orders of the n-1 other cards)."""
    if canon:
        batch_threads = max(1 << 12, batch_threads // max(1, n - 1))
    batch_threads = max(threads, (batch_threads // threads) * threads)
    return batch_threads * per


def fixture(n, canon, spans, hbins, shape, dbins, elapsed_s, slowest_s, updated):
    per = 256
    total = math.factorial(n - 1) if canon else math.factorial(n)
    next_start = spans * ref_span(n, canon)
    mult = (n - 1) if canon else 1
    blk = (n & -n) if (canon and shape) else 0
    flags = (oracle.F_DISTINCT if dbins else 0) | (oracle.F_SHAPE if blk else 0)
    r = oracle.enumerate_job(oracle.make_job(n, oracle.CANON if canon else oracle.DEALS, 0, flags, 0,
                                             next_start * mult, hbins, dbins, blk))
    d = oracle.to_dict(r)
    # the keys and their order of gpu/war_gpu.py:331-338
    return {"n": n, "half": False, "canon": canon, "per": per, "next_start": next_start, "total": total,
            "cyc": d["cyc"], "done": d["done"], "maxfin": d["maxfin"],
            "hist": {str(i): v for i, v in sorted(d["hist"].items())} if hbins else {},
            "shape": [d["shape_nonstd"], d["shape_unchecked"]] if blk else None,
            "rule": 0,
            "dhist": {str(i): v for i, v in sorted(d["dhist"].items())} if dbins else {},
            "elapsed_s": elapsed_s, "slowest_launch_s": slowest_s, "updated": updated}


def main():
    out = {
        # python war_gpu.py 13 --hist 256 --out n13, stopped after 4 launches
        "progress_deals13_ref.json": fixture(13, False, 4, 256, False, 0, 40.2, 0.215, "2025-11-02 10:14:07"),
        # python war_gpu.py 13 --canon --distinct --shape --out c13, stopped after 2 launches
        "progress_canon13_ref.json": fixture(13, True, 2, 0, True, 4096, 20.5, 0.377, "2025-11-02 11:02:51"),
    }
    for name, st in out.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(st, f)
        print("wrote", name, st["next_start"], st["cyc"], st["done"])


if __name__ == "__main__":
    main()
