"""Count the deals of single-suit War that never end, on a B200 (n <= 16; deals of 17 cards go to the
held-out-card engine, see war17.py).

Drop-in for the reference's gpu/war_gpu.py: the same command line, the same run() signature and return
tuple, the same output lines and the same <out>.progress file (gpu/war_gpu.py:272-398).  The work runs
in libwar.so (hand-written sm_100a kernels, C ABI in include/war.h) through ctypes; there is no other
path.

Cards are 0..n-1 (0 lowest).  Deck positions 0, 2, 4, ... go to player 1 and 1, 3, 5, ... to player 2,
top card first.  Each turn the higher top card wins, and the winner puts the winning card and then the
losing card under their own pile (--rule 1 reverses the order).  --half (even n) plays only the deals
that give the highest card to player 1 and doubles the counts.  --canon scans the (n-1)! (n-1) positions
in which player 1's top card is the highest card.

  python war_gpu.py 12                        a(12)
  python war_gpu.py 15 --hist 128             a(15) and the cycle lengths
  python war_gpu.py 16 --canon --out n16c     every 16-card canonical position, resumable
  python war_gpu.py 13 --plain                the plain kernel (one thread per 256 consecutive deals)
"""
import argparse
import json
import math
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import warlib  # noqa: E402

# Ranks enumerated per call of the engine: a few seconds of work, so progress is written about as
# often as the reference writes it (every 10 s) and an interrupted run loses little.  Just under 2^32,
# so that a span of deals is one launch of the engine (a launch plays fewer than 2^32 - 2^24 games).
SPAN_RANKS = (1 << 32) - (1 << 25)


def _tune_for(n, canon, rule, flags):
    try:
        import autotune
        return autotune.cached_tune(n, warlib.CANON if canon else warlib.DEALS, rule, flags)
    except Exception:
        return None


def override_tune(tune, fields):
    """A copy of tune (a warlib.Tune or None) with the given fields replaced."""
    t = warlib.make_tune()
    if tune is not None:
        for k, _ in warlib.Tune._fields_:
            setattr(t, k, getattr(tune, k))
    for k, v in fields.items():
        if k not in dict(warlib.Tune._fields_):
            raise ValueError("unknown tune field %r" % k)
        setattr(t, k, int(v))
    return t


def run(n, half=False, per=256, threads=256, batch_threads=1 << 18, out=None, resume=False, quiet=False, hbins=0,
        canon=False, shape=False, rule=0, dbins=0, plain=False, tune=None):
    """gpu/war_gpu.py:272-352.  Returns (cyc, done, maxfin, elapsed_s, hist, shape, dhist): cyc, done and hist
    doubled with half; shape = (not_T3, unchecked, blk) or None; dhist = {weight: positions} or None.

    per / threads / batch_threads keep their meaning for the progress file and for plain=True (the plain
    kernel launches exactly the reference's geometry); the default path is the persistent refill kernel."""
    total = math.factorial(n - 1) if canon else math.factorial(n)     # orders (canon) or deals
    if canon:
        batch_threads = max(1 << 12, batch_threads // max(1, n - 1))
    batch_threads = max(threads, (batch_threads // threads) * threads)
    if not canon:
        dbins = 0
    blk = (n & -n) if (canon and shape) else 0
    if blk and os.environ.get("WAR_BLK_OVERRIDE"):      # negative control only: force a wrong block length
        blk = int(os.environ["WAR_BLK_OVERRIDE"])
    acc = {"cyc": 0, "done": 0, "maxfin": 0}
    hist = [0] * max(hbins, 1)
    shp = [0, 0]
    dh = [0] * max(dbins, 1)
    start = 0
    prog = (out + ".progress") if out else None
    if resume and prog and os.path.exists(prog):
        with open(prog) as f:
            st = json.load(f)
        assert st["n"] == n and st["half"] == half and st["per"] == per and st.get("canon", False) == canon
        start = st["next_start"]
        acc["cyc"], acc["done"], acc["maxfin"] = st["cyc"], st["done"], st["maxfin"]
        for k, v in st.get("hist", {}).items():
            hist[int(k)] = v
        if "shape" in st and st["shape"]:
            shp = [st["shape"][0], st["shape"][1]]
        for kk, vv in (st.get("dhist") or {}).items():
            dh[int(kk)] = vv
        assert st.get("rule", 0) == rule
        if not quiet:
            print("resuming at %d / %d" % (start, total), flush=True)
    flags = (warlib.F_HALF if half else 0) | (warlib.F_DISTINCT if dbins else 0) | (warlib.F_SHAPE if blk else 0)
    mode = warlib.CANON if canon else warlib.DEALS
    mult_pos = (n - 1) if canon else 1                    # engine ranks per order
    if tune is None and not plain:
        tune = _tune_for(n, canon, rule, flags)
    span = max(batch_threads * per, SPAN_RANKS // mult_pos if mult_pos else SPAN_RANKS)
    t0 = time.time()
    last_write = 0.0
    slowest = 0.0
    first = start
    while start < total:
        tl = time.time()
        end = min(total, start + span)
        # spans after the first keep the cycle memo of the one before (same n and rule)
        keep = warlib.F_MEMO_KEEP if start > first else 0
        job = warlib.make_job(n, mode, rule, flags | keep, start * mult_pos, end * mult_pos, hbins=hbins, dbins=dbins,
                              blk=blk)
        r = warlib.enumerate_plain(job) if plain else warlib.enumerate_job(job, tune)
        acc["cyc"] += r.cyc
        acc["done"] += r.done
        acc["maxfin"] = max(acc["maxfin"], r.maxfin)
        for i in range(hbins):
            hist[i] += r.hist[i]
        for i in range(dbins):
            dh[i] += r.dhist[i]
        shp[0] += r.shape_nonstd
        shp[1] += r.shape_unchecked
        slowest = max(slowest, time.time() - tl)
        start = end
        if prog and (time.time() - last_write >= 10 or start >= total):
            last_write = time.time()
            st = {"n": n, "half": half, "canon": canon, "per": per, "next_start": min(start, total), "total": total,
                  "cyc": acc["cyc"], "done": acc["done"], "maxfin": acc["maxfin"],
                  "hist": {str(i): v for i, v in enumerate(hist) if v} if hbins else {},
                  "shape": [shp[0], shp[1]] if blk else None,
                  "rule": rule,
                  "dhist": {str(i): v for i, v in enumerate(dh) if v} if dbins else {},
                  "elapsed_s": round(time.time() - t0, 1), "slowest_launch_s": round(slowest, 3),
                  "updated": time.strftime("%Y-%m-%d %H:%M:%S")}
            tmp = prog + ".tmp"
            with open(tmp, "w") as f:
                json.dump(st, f)
            os.replace(tmp, prog)
            if not quiet:
                frac = min(start, total) / total
                el = time.time() - t0
                print("%.4f%%  cyc=%d  elapsed %.0fs  slowest launch %.3fs" % (100 * frac, acc["cyc"], el, slowest),
                      flush=True)
    mult = 2 if half else 1
    c = acc["cyc"] * mult
    d = acc["done"] * mult
    h = {i: v * mult for i, v in enumerate(hist) if v} if hbins else {}
    sh = (shp[0], shp[1], blk) if blk else None
    dd = {i: v for i, v in enumerate(dh) if v} if dbins else None
    return c, d, acc["maxfin"], time.time() - t0, h, sh, dd


def format_lines(n, c, d, mx, el, h, sh, dd, canon, half, hist_bins):
    """The result lines of gpu/war_gpu.py:384-398, byte for byte apart from the time."""
    lines = []
    what = "canonical positions cycling" if canon else "a(n)"
    lines.append("n=%d  %s=%d  of %d  longest finite=%d rounds  %.1fs%s"
                 % (n, what, c, d, mx, el, "  (half)" if half else ""))
    if dd is not None:
        lines.append("   distinct cycles (up to swapping players): %d   [on-cycle canonical positions by weight: %s]"
                     % (sum(v // k for k, v in dd.items()), dict(sorted(dd.items()))))
    if sh:
        lines.append("   loop shape: %d cycling positions checked for runs of exactly %d; "
                     "not that shape: %d; too long to check: %d" % (c, sh[2], sh[0], sh[1]))
    if h:
        lines.append("   loop lengths (rounds: %s): " % ("positions" if canon else "deals") + ", ".join(
            ("%s%d: %d" % (">=" if k == hist_bins - 1 else "", k, v)) for k, v in sorted(h.items())))
    return lines


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("nmax", type=int)
    ap.add_argument("--nmin", type=int, default=None)
    ap.add_argument("--half", action="store_true", help="even n: use player-swap symmetry")
    ap.add_argument("--per", type=int, default=256,
                    help="deck orders per thread per launch (with --canon: orders of the other n-1 cards, n-1 positions each)")
    ap.add_argument("--out", help="progress file prefix (enables resumable progress)")
    ap.add_argument("--resume", action="store_true")
    ap.add_argument("--hist", type=int, default=0, help="loop-length histogram bins (last bin = overflow)")
    ap.add_argument("--canon", action="store_true",
                    help="scan canonical positions (player 1's top card is n) instead of deals")
    ap.add_argument("--rule", type=int, default=0, choices=[0, 1],
                    help="put-back order: 0 = winner's card first (Spivey), 1 = loser's card first")
    ap.add_argument("--distinct", action="store_true",
                    help="canon only: count distinct cycles up to swapping the players")
    ap.add_argument("--shape", action="store_true",
                    help="canon only: check every loop alternates in runs of exactly 2^v (Spivey Thm 3 type)")
    ap.add_argument("--plain", action="store_true",
                    help="use the plain kernel (the reference's per-thread blocks) instead of the refill kernel")
    ap.add_argument("--tune", default=None,
                    help='JSON object overriding fields of the stored tune, e.g. \'{"memo_bits": 28}\'')
    a = ap.parse_args(argv)
    if a.hist > warlib.WAR_HBINS_MAX:
        ap.error("--hist is at most %d" % warlib.WAR_HBINS_MAX)
    lo = a.nmin if a.nmin is not None else a.nmax
    for n in range(lo, a.nmax + 1):
        half = a.half and n % 2 == 0 and not a.canon
        tune = None
        if a.tune and not a.plain:
            flags = (warlib.F_HALF if half else 0) | (warlib.F_DISTINCT if a.distinct else 0) | \
                (warlib.F_SHAPE if a.shape and a.canon else 0)
            tune = override_tune(_tune_for(n, a.canon, a.rule, flags), json.loads(a.tune))
        c, d, mx, el, h, sh, dd = run(n, half=half, per=a.per, out=a.out, resume=a.resume,
                                      quiet=a.out is None, hbins=a.hist, canon=a.canon, shape=a.shape,
                                      rule=a.rule, dbins=4096 if a.distinct else 0, plain=a.plain, tune=tune)
        expect = math.factorial(n - 1) * (n - 1) if a.canon else math.factorial(n)
        assert d == expect, (d, expect)
        if h:
            assert sum(h.values()) == c, ("histogram does not add up", sum(h.values()), c)
        lines = format_lines(n, c, d, mx, el, h, sh, dd, a.canon, half, a.hist)
        print(lines[0], flush=True)
        if dd is not None:
            bad = {k: v for k, v in dd.items() if v % k}
            assert not bad, ("distinct-cycle weights not divisible", bad)
            assert 4095 not in dd, "a cycle had more than 4094 canonical states: raise dbins"
        for line in lines[1:]:
            print(line, flush=True)


if __name__ == "__main__":
    main()
