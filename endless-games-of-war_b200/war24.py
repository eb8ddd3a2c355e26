"""Count the deals of single-suit War that never end, for up to 20 cards, on a B200.

Drop-in for the reference's gpu/war24.py: the same command line, the same checkpoint and progress files, the
same result line (gpu/war24.py:158-210).  The work runs in libwar.so's 5-bit-pile engine
(war_enumerate_wide: 5-bit cards in 128-bit piles, a persistent refill kernel) through ctypes.

Rule (Spivey 2010): the higher top card wins; the winning card, then the losing card, go under the winner's
pile.  Deals: all n! orders of the cards 0..n-1, player 1 gets the cards at even positions (first dealt on
top).  Deal ranks are 64-bit, so n <= 20.

Cycle detection:
  --det streak  (default; odd n only) the players alternate for lcm(n+1, W, L-1) turns after an anchor where
                the next winner holds an even number of cards, and the state is compared with the anchor
                (Spivey Thm 6) — gpu/war24.py:98-125.
  --det floyd   tortoise and hare (any n) — gpu/war24.py:85-97.
  --det brent   Brent's cycle test (any n; this engine's fastest, not in the reference).
Games still undecided after 2^22 turns are counted as undetermined.

  python war24.py 17 --det streak --start 100000000000000 --count 1000000000
  python war24.py 19 --resume                      continue from the checkpoint of the same range

--chunk and --threads set the reference's launch geometry; they are accepted (and checked the same way) but
the persistent kernel sizes its own grid.  --dir puts the checkpoint and progress files elsewhere than next to
this file.
"""
import argparse
import json
import math
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import warlib  # noqa: E402

DETS = {"brent": warlib.DET_BRENT, "floyd": warlib.DET_FLOYD, "streak": warlib.DET_STREAK}
# Deals per engine call: a few seconds of work at 17 cards.  The checkpoint is written after a call when
# CKPT_EVERY_S seconds have passed since the last one (and at the end), as the reference does.
SPAN = (1 << 32) - (1 << 25)
CKPT_EVERY_S = 10.0


def run(n, det="streak", lo=0, hi=None, resume=False, tag="", directory=None):
    """Deals [lo, hi) of n cards (gpu/war24.py:186-201).  Returns (cycling, longest_finite, deals, undetermined,
    elapsed_s).  Writes war24_<n>_<det>_<lo>_<hi><tag>.ckpt (JSON: pos, cyc, max, deals, und) and appends to
    the matching .progress log, as the reference does; resume=True continues from the checkpoint."""
    total_all = math.factorial(n)
    hi = total_all if hi is None else min(total_all, hi)
    here = directory or os.path.dirname(os.path.abspath(__file__))
    name = f"n{n}_{det}_{lo}_{hi}{tag}"
    prog = os.path.join(here, f"war24_{name}.progress")
    ckpt = os.path.join(here, f"war24_{name}.ckpt")
    st = {"pos": lo, "cyc": 0, "max": 0, "deals": 0, "und": 0}
    if resume and os.path.exists(ckpt):
        with open(ckpt) as f:
            st = json.load(f)
    pos = st["pos"]
    t0 = time.time()
    last = t0
    pos0 = pos
    with open(prog, "a") as pf:
        while pos < hi:
            end = min(hi, pos + SPAN)
            r = warlib.enumerate_wide(warlib.make_job(n, warlib.DEALS, 0, 0, pos, end), det=DETS[det])
            st["cyc"] += r.cyc
            st["max"] = max(st["max"], r.maxfin)
            st["deals"] += r.done
            st["und"] += r.undetermined
            pos = end
            st["pos"] = pos
            now = time.time()
            if now - last > CKPT_EVERY_S or pos >= hi:
                with open(ckpt + ".tmp", "w") as f:
                    json.dump(st, f)
                os.replace(ckpt + ".tmp", ckpt)
                rate = (pos - pos0) / max(now - t0, 1e-9)
                pf.write(f"{time.strftime('%H:%M:%S')} n={n} det={det} pos={pos}/{hi} "
                         f"({100 * (pos - lo) / max(1, hi - lo):.4f}%) cyc={st['cyc']} max={st['max']} "
                         f"und={st['und']} rate={rate:.3e}/s\n")
                pf.flush()
                last = now
    return st["cyc"], st["max"], st["deals"], st["und"], time.time() - t0


def result_line(n, det, lo, hi, cyc, mx, deals, und, el):
    """The result line of gpu/war24.py:204-205."""
    return (f"n={n} det={det} range=[{lo},{hi}) deals_simulated={deals} (expected {hi - lo}) "
            f"cycling={cyc} longest_finite={mx} undetermined={und} time={el:.1f}s")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("n", type=int)
    ap.add_argument("--det", choices=["floyd", "streak", "brent"], default="streak")
    ap.add_argument("--start", type=int, default=0)
    ap.add_argument("--count", type=int, default=0, help="number of deals from --start (0 = to the end)")
    ap.add_argument("--chunk", type=int, default=32)
    ap.add_argument("--threads", type=int, default=1 << 17)
    ap.add_argument("--resume", action="store_true")
    ap.add_argument("--tag", default="", help="suffix for the progress and checkpoint file names")
    ap.add_argument("--dir", default=None, help="directory of the progress and checkpoint files (default: here)")
    a = ap.parse_args(argv)
    n = a.n
    assert 2 <= n <= 20, "deal ranks are 64-bit: n <= 20"
    if a.det == "streak" and n % 2 == 0:
        sys.exit("streak detection is only valid for odd n (Spivey Thm 6)")
    assert a.threads % 256 == 0, "--threads must be a multiple of 256"
    total_all = math.factorial(n)
    lo = a.start
    hi = total_all if a.count == 0 else min(total_all, lo + a.count)
    cyc, mx, deals, und, el = run(n, a.det, lo, hi, resume=a.resume, tag=a.tag, directory=a.dir)
    msg = result_line(n, a.det, lo, hi, cyc, mx, deals, und, el)
    print(msg, flush=True)
    here = a.dir or os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, f"war24_n{n}_{a.det}_{lo}_{hi}{a.tag}.progress"), "a") as pf:
        pf.write(msg + "\n")
    if deals != hi - lo:
        print("ERROR: deal count mismatch", flush=True)
        sys.exit(1)


if __name__ == "__main__":
    main()
