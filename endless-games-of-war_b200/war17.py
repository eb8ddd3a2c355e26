"""Count the deals of single-suit War that never end, on a B200, for n <= 17 (drop-in for gpu/war17.py).

Card n-1 never loses, so it is kept out of the packed piles and tracked by its depth in its holder's pile
(gpu/war17.py:7-16); the engine is war_enumerate_held in libwar.so (csrc/war_held.cu).  Same command line,
output line and progress file as gpu/war17.py:160-178 / :131-157:

    python war17.py 15 --nmin 5            # reproduces the known terms
    python war17.py 17 --out n17 [--resume] [--per 32]

--per and --batch keep their meaning for the progress file (the reference's launch tiling); the engine
itself takes whole spans of about 4e9 deals per call.  --rule 1 (loser's card first) is an addition.
"""
import argparse
import json
import math
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import warlib  # noqa: E402

# Deals per engine call: just under 2^32, one launch of the engine, a second or so at n = 17.
SPAN_RANKS = (1 << 32) - (1 << 25)


def run(n, per=64, threads=256, batch_threads=1 << 16, out=None, resume=False, quiet=True, rule=0, hbins=0,
        tune=None):
    """gpu/war17.py:116-157.  Returns (cyc, done, maxfin, elapsed_s, slowest_call_s); with hbins > 0 the
    cycle-length histogram is in run.last_hist afterwards."""
    assert 1 <= n <= 17
    batch_threads = max(threads, (batch_threads // threads) * threads)   # no overlap between launches
    total = math.factorial(n)
    cyc = done = mx = 0
    hist = [0] * max(hbins, 1)
    start = 0
    prog = (out + ".progress") if out else None
    if resume and prog and os.path.exists(prog):
        with open(prog) as f:
            st = json.load(f)
        assert st["n"] == n and st["per"] == per and st["batch_threads"] == batch_threads
        start = st["next_start"]
        cyc, done, mx = st["cyc"], st["done"], st["maxfin"]
    span = max(batch_threads * per, SPAN_RANKS)
    t0 = time.time()
    last = 0.0
    slowest = 0.0
    while start < total:
        tl = time.time()
        end = min(total, start + span)
        if n == 1:   # the single 1-card deal: player 2 has no card (gpu/war17.py:61)
            d = warlib.enumerate_job(warlib.make_job(1, lo=start, hi=end, hbins=hbins))
        else:
            d = warlib.enumerate_held(warlib.make_job(n, rule=rule, lo=start, hi=end, hbins=hbins), tune)
        cyc += d.cyc
        done += d.done
        mx = max(mx, d.maxfin)
        for i in range(hbins):
            hist[i] += d.hist[i]
        slowest = max(slowest, time.time() - tl)
        start = end
        if prog and (time.time() - last >= 10 or start >= total):
            last = time.time()
            st = {"n": n, "per": per, "batch_threads": batch_threads, "next_start": min(start, total),
                  "total": total, "cyc": cyc, "done": done, "maxfin": mx,
                  "elapsed_s": round(time.time() - t0, 1), "slowest_launch_s": round(slowest, 3),
                  "updated": time.strftime("%Y-%m-%d %H:%M:%S")}
            with open(prog + ".tmp", "w") as f:
                json.dump(st, f)
            os.replace(prog + ".tmp", prog)
            if not quiet:
                print("%.4f%%  cyc=%d  %.0fs  slowest %.3fs" % (100 * min(start, total) / total, cyc,
                                                              time.time() - t0, slowest), flush=True)
    run.last_hist = {i: v for i, v in enumerate(hist) if v} if hbins else {}
    return cyc, done, mx, time.time() - t0, slowest


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("nmax", type=int)
    ap.add_argument("--nmin", type=int)
    ap.add_argument("--per", type=int, default=64)
    ap.add_argument("--batch", type=int, default=1 << 16)
    ap.add_argument("--out")
    ap.add_argument("--resume", action="store_true")
    ap.add_argument("--rule", type=int, default=0, choices=[0, 1],
                    help="put-back order: 0 = winner's card first (Spivey), 1 = loser's card first")
    a = ap.parse_args(argv)
    for n in range(a.nmin or a.nmax, a.nmax + 1):
        c, d, mx, el, sl = run(n, per=a.per, batch_threads=a.batch, out=a.out, resume=a.resume, quiet=a.out is None,
                               rule=a.rule)
        assert d == math.factorial(n), (d, math.factorial(n))
        print("n=%d  a(n)=%d  of %d deals  longest finite=%d  %.1fs  slowest launch %.3fs" % (n, c, d, mx, el, sl),
              flush=True)


if __name__ == "__main__":
    main()
