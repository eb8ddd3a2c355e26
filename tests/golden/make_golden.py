"""Writes tests/golden/golden.json from the reference's recorded outputs.

Run it where the reference is mounted (read-only):  python tests/golden/make_golden.py [REF_ROOT]
(REF_ROOT defaults to $WAR_REF, else the reference's mount point in the build container).
The JSON is committed; nothing reads the reference at test time.  Sources (paths in the reference):
  data/deals.tsv                 a(n), longest ending game, cycle-length split, n = 1..17
  data/canonical_positions.tsv   canonical positions: entering a cycle, on a cycle, cycles
  data/loser_first.tsv           the loser-first rule, n = 1..15
  data/checks.txt                small-n outputs of gpu/war_gpu.py and cpu/distinct_cycles.c,
                                 the Floyd program's negative controls, loser-first canonical scans
  data/long_runs.txt             the n = 14..16 runs
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WAR_REF", "/root/reference")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def parse_hist(s):
    return {int(a): int(b) for a, b in re.findall(r"(\d+):\s*(\d+)", s)}


def tsv(rel):
    rows = []
    for line in read(rel).splitlines():
        if not line.strip() or line.startswith("#"):
            continue
        rows.append(line.split("\t"))
    return rows


def main():
    g = {"source": "OrygnsCode/endless-games-of-war data/ (recorded program outputs)"}

    # deals, rule 0: data/deals.tsv
    deals = {}
    for r in tsv("data/deals.tsv"):
        n = int(r[0])
        e = {"deals": int(r[1]), "cyc": int(r[2])}
        if len(r) > 3 and r[3]:
            e["longest"] = int(r[3])
        if len(r) > 4 and r[4]:
            e["hist"] = parse_hist(r[4])
        elif e["cyc"] == 0 and "longest" in e:
            e["hist"] = {}
        deals[n] = e
    g["deals_rule0"] = deals

    # canonical positions: data/canonical_positions.tsv
    canon_tab = {}
    for r in tsv("data/canonical_positions.tsv"):
        n = int(r[0])
        e = {"positions": int(r[1])}
        if r[2]:
            e["cycling"] = int(r[2])
        if r[3]:
            e["oncycle"] = int(r[3])
        if r[4]:
            e["distinct"] = int(r[4])
        canon_tab[n] = e
    g["canon_table"] = canon_tab

    # loser first deals: data/loser_first.tsv
    g["deals_rule1"] = {int(r[0]): {"deals": int(r[1]), "cyc": int(r[2]), "longest": int(r[3])}
                        for r in tsv("data/loser_first.tsv")}

    checks = read("data/checks.txt")
    long_runs = read("data/long_runs.txt")

    # gpu/war_gpu.py --canon --distinct --shape output blocks (checks.txt, long_runs.txt)
    canon = {}
    pat = re.compile(
        r"n=(\d+)  canonical positions cycling=(\d+)  of (\d+)  longest finite=(\d+) rounds[^\n]*\n"
        r"   distinct cycles \(up to swapping players\): (\d+)   \[on-cycle canonical positions by weight: \{([^}]*)\}\]\n"
        r"   loop shape: (\d+) cycling positions checked for runs of exactly (\d+); not that shape: (\d+); too long to check: (\d+)"
        r"(?:\n   loop lengths \(rounds: positions\): ([^\n]*))?")
    for text in (checks, long_runs):
        for m in pat.finditer(text):
            n = int(m.group(1))
            e = {"cycling": int(m.group(2)), "positions": int(m.group(3)), "longest": int(m.group(4)),
                 "distinct": int(m.group(5)), "dhist": parse_hist(m.group(6)), "blk": int(m.group(8)),
                 "shape_nonstd": int(m.group(9)), "shape_unchecked": int(m.group(10))}
            if m.group(11):
                e["hist"] = parse_hist(m.group(11))
            canon[n] = e
    g["canon_rule0"] = canon

    # n=16 canonical scans (rule 0 and rule 1), long_runs.txt
    c16 = re.search(r"n=16  canonical positions cycling=(\d+)  of (\d+)  longest finite=(\d+) rounds  13551", long_runs)
    c16r1 = re.search(r"n=16  canonical positions cycling=(\d+)  of (\d+)  longest finite=(\d+) rounds  45196", long_runs)
    g["canon16"] = {"rule0": [int(x) for x in c16.groups()], "rule1": [int(x) for x in c16r1.groups()]}

    # loser-first canonical scan n = 2..12 (gpu/war_gpu.py 12 --nmin 2 --canon --rule 1)
    blk = checks.split("== Losing card first, canonical positions, both GPU programs")[1].split("==")[0]
    g["canon_rule1"] = {int(a): {"cycling": int(b), "positions": int(c), "longest": int(d)}
                        for a, b, c, d in re.findall(
                            r"n=(\d+)  canonical positions cycling=(\d+)  of (\d+)  longest finite=(\d+) rounds", blk)}

    # deal cycle-length histograms printed by gpu/war_gpu.py 13 --nmin 1 --hist 256 (checks.txt:5-24)
    blk = checks.split("== Deals, n = 1..13")[1].split("==")[0]
    hists = {}
    for m in re.finditer(r"n=(\d+)  a\(n\)=(\d+)  of (\d+)  longest finite=(\d+) rounds[^\n]*\n"
                         r"(   loop lengths \(rounds: deals\): ([^\n]*))?", blk):
        hists[int(m.group(1))] = {"cyc": int(m.group(2)), "deals": int(m.group(3)), "longest": int(m.group(4)),
                                 "hist": parse_hist(m.group(6)) if m.group(6) else {}}
    g["war_gpu_deals_hist"] = hists

    # the printed lines themselves (the drop-in CLI must print them byte for byte apart from the time):
    # deals n = 1..13 with --hist 256, canonical n = 1..13 with --distinct --shape (checks.txt:5-24, 143-182)
    def out_lines(text):
        return [ln for ln in text.split("\n") if ln.startswith("n=") or ln.startswith("   ")]
    g["war_gpu_lines"] = {
        "deals_hist256": out_lines(checks.split("== Deals, n = 1..13")[1].split("==")[0]),
        "canon_distinct_shape": out_lines(
            checks.split("== Canonical positions, distinct cycles and the Theorem-3 test, n = 1..13")[1].split("==")[0]),
        # gpu/war17.py 13 --nmin 5 (checks.txt:81-91)
        "war17_5_13": out_lines(checks.split("== Deals, 17-card GPU program")[1].split("==")[0]),
        # war_gpu.py 14 --half --hist 256 (long_runs.txt:14-15)
        "long14_half": out_lines(long_runs.split("python war_gpu.py 14 --half --hist 256;")[1].split("n=15")[0]),
        # war_gpu.py 14 --canon --distinct --shape --hist 256 (long_runs.txt:20-23)
        "long14_canon": out_lines(long_runs.split("python war_gpu.py 14 --canon --distinct --shape --hist 256")[1]
                                  .split("$")[0]),
    }

    # gpu/war24.py result lines (checks.txt:73-79, long_runs.txt:62-75)
    w24 = []
    for m in re.finditer(r"n=(\d+) det=(\w+) range=\[(\d+),(\d+)\) deals_simulated=(\d+) \(expected (\d+)\) "
                         r"cycling=(\d+) longest_finite=(\d+) undetermined=(\d+)", checks + long_runs):
        w24.append({"n": int(m.group(1)), "det": m.group(2), "lo": int(m.group(3)), "hi": int(m.group(4)),
                    "deals": int(m.group(5)), "cyc": int(m.group(7)), "longest": int(m.group(8)),
                    "undetermined": int(m.group(9)), "line": m.group(0)})
    g["war24"] = w24

    # gpu/war_gpu_floyd.py full-range deal runs without --half (long_runs.txt:35, :39)
    fd = {}
    for m in re.finditer(r"n=(\d+) half=False deals_simulated=(\d+) \(expected \d+\) cycling_found=(\d+) a\(n\)=(\d+) "
                         r"longest_finite=(\d+)", long_runs):
        fd[int(m.group(1))] = {"deals": int(m.group(2)), "cyc": int(m.group(3)), "longest": int(m.group(5))}
    g["floyd_deals"] = fd

    # n = 14, 15 long deal runs with histograms (long_runs.txt:13-17)
    lr = {}
    for m in re.finditer(r"n=(\d+)  a\(n\)=(\d+)  of (\d+)  longest finite=(\d+) rounds  [\d.]+s(  \(half\))?\n"
                         r"   loop lengths \(rounds: deals\): ([^\n]*)", long_runs):
        lr[int(m.group(1))] = {"cyc": int(m.group(2)), "deals": int(m.group(3)), "longest": int(m.group(4)),
                               "half": bool(m.group(5)), "hist": parse_hist(m.group(6))}
    g["long_deals_rule0"] = lr

    # cpu/distinct_cycles.c outputs (checks.txt:200-221)
    dc = {}
    for m in re.finditer(r"n=(\d+): canonical positions that never end (\d+); on a cycle (\d+); DISTINCT cycles up to swap (\d+)\n"
                         r"   cycle lengths \(distinct cycles\):([^\n]*)", checks):
        dc[int(m.group(1))] = {"cycling": int(m.group(2)), "oncycle": int(m.group(3)), "distinct": int(m.group(4)),
                               "lengths": parse_hist(m.group(5))}
    g["distinct_cycles_c"] = dc

    # Floyd program: half-mode and Theorem-3 negative controls (checks.txt:184-198, long_runs.txt:37-38)
    fl = []
    for m in re.finditer(r"n=(\d+) CANON positions_simulated=(\d+) \(expected \d+\) cycling_canonical_positions=(\d+) "
                         r"cycle_exists=\w+ q1_nonTheorem3_loops=(\d+) \(block=(\d+)\)", checks + long_runs):
        fl.append({"n": int(m.group(1)), "positions": int(m.group(2)), "cycling": int(m.group(3)),
                   "nonstd": int(m.group(4)), "blk": int(m.group(5))})
    g["floyd_canon_q1"] = fl
    half = []
    for m in re.finditer(r"n=(\d+) half=True deals_simulated=(\d+) \(expected \d+\) cycling_found=(\d+) a\(n\)=(\d+) "
                         r"longest_finite=(\d+)", checks + long_runs):
        half.append({"n": int(m.group(1)), "played": int(m.group(2)), "cyc_half": int(m.group(3)),
                     "a": int(m.group(4)), "longest": int(m.group(5))})
    g["floyd_half"] = half

    with open(OUT, "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
