"""The oracle (oracle/war_oracle.c) pinned against the reference's recorded outputs and against the
reference's own CPU programs built unmodified into oracle/_ref/.  CPU only."""
import pytest

# Brent turn totals (WAR_STEPs run with the reference's checkpoint schedule, cpu/war.cpp:26-37), counted
# with an instrumented copy of cpu/war.cpp when the reference was surveyed.
REF_TURNS = {9: 13835040, 10: 95482840, 11: 1215869402}


def test_deals_rule0_small(oracle, golden):
    for n in range(1, 12):
        r = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, hbins=256)))
        g = golden["deals_rule0"][n]
        assert r["done"] == g["deals"]
        assert r["cyc"] == g["cyc"], n
        assert r["maxfin"] == g["longest"], n
        assert r["hist"] == g["hist"], n
        assert sum(r["endhist"].values()) == g["deals"] - g["cyc"]
        assert max(r["endhist"]) == g["longest"] or n == 1
        # war_gpu.py's own printed histograms (data/checks.txt:5-24)
        w = golden["war_gpu_deals_hist"][n]
        assert (r["cyc"], r["maxfin"], r["hist"]) == (w["cyc"], w["longest"], w["hist"])


def test_turn_totals(oracle):
    for n, t in REF_TURNS.items():
        assert oracle.enumerate_job(oracle.make_job(n)).turns == t


def test_deals_rule1(oracle, golden):
    for n in range(1, 12):
        r = oracle.enumerate_job(oracle.make_job(n, rule=1))
        g = golden["deals_rule1"][n]
        assert (r.done, r.cyc, r.maxfin) == (g["deals"], g["cyc"], g["longest"]), n


def test_canon_rule0_distinct_shape(oracle, golden):
    F = oracle.F_DISTINCT | oracle.F_SHAPE
    for n in range(1, 12):
        r = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, mode=oracle.CANON, flags=F, hbins=256, dbins=4096)))
        g = golden["canon_rule0"][n]
        assert r["done"] == g["positions"]
        assert r["cyc"] == g["cycling"], n
        assert r["maxfin"] == g["longest"], n
        assert r["dhist"] == g["dhist"], n
        assert sum(v // k for k, v in r["dhist"].items()) == g["distinct"]
        assert r["distinct_min"] == g["distinct"], n
        assert r["shape_nonstd"] == g["shape_nonstd"] and r["shape_unchecked"] == g["shape_unchecked"]
        t = golden["canon_table"][n]
        assert r["oncycle"] == t.get("oncycle", 0)


def test_canon_rule1(oracle, golden):
    for n in range(2, 12):
        r = oracle.enumerate_job(oracle.make_job(n, mode=oracle.CANON, rule=1))
        g = golden["canon_rule1"][n]
        assert (r.done, r.cyc, r.maxfin) == (g["positions"], g["cycling"], g["longest"]), n


def test_distinct_cycles_c_lengths(oracle, golden):
    """cpu/distinct_cycles.c's per-length counts of distinct cycles = min-key positions by cycle length."""
    for n in range(5, 12):
        g = golden["distinct_cycles_c"][n]
        r = oracle.enumerate_job(oracle.make_job(n, mode=oracle.CANON, flags=oracle.F_DISTINCT, hbins=256, dbins=4096))
        assert (r.cyc, r.oncycle, r.distinct_min) == (g["cycling"], g["oncycle"], g["distinct"])


def test_shape_negative_controls(oracle, golden):
    """A wrong block length must flag every loop (gpu/war_gpu_floyd.py --block, data/checks.txt:197-198)."""
    for g in golden["floyd_canon_q1"]:
        if g["n"] > 11:
            continue
        r = oracle.enumerate_job(oracle.make_job(g["n"], mode=oracle.CANON, flags=oracle.F_SHAPE, blk=g["blk"]))
        assert (r.done, r.cyc, r.shape_nonstd) == (g["positions"], g["cycling"], g["nonstd"])


def test_half(oracle, golden):
    for g in golden["floyd_half"]:
        if g["n"] > 11:
            continue
        r = oracle.enumerate_job(oracle.make_job(g["n"], flags=oracle.F_HALF))
        assert (r.done, r.cyc, 2 * r.cyc, r.maxfin) == (g["played"], g["cyc_half"], g["a"], g["longest"])


@pytest.mark.parametrize("n,mode", [(9, 0), (10, 0), (9, 1), (10, 1)])
def test_ranges_add_up(oracle, n, mode):
    import random
    rnd = random.Random(n * 7 + mode)
    total = oracle.space_size(n, mode)
    cuts = sorted(rnd.sample(range(1, total), 5))
    edges = [0] + cuts + [total]
    whole = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, mode=mode, hbins=128, dbins=64,
                                                                 flags=oracle.F_DISTINCT if mode else 0)))
    parts = [oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, mode=mode, lo=a, hi=b, hbins=128, dbins=64,
                                                                  flags=oracle.F_DISTINCT if mode else 0)))
             for a, b in zip(edges, edges[1:])]
    for k in ("cyc", "done", "turns", "oncycle", "distinct_min"):
        assert sum(p[k] for p in parts) == whole[k]
    assert max(p["maxfin"] for p in parts) == whole["maxfin"]
    for h in ("hist", "dhist", "endhist"):
        acc = {}
        for p in parts:
            for k, v in p[h].items():
                acc[k] = acc.get(k, 0) + v
        assert acc == whole[h]


@pytest.mark.parametrize("n,mode,rule", [(9, 0, 0), (10, 0, 1), (9, 1, 0), (10, 1, 1)])
def test_floyd_sample_matches_brent(oracle, n, mode, rule):
    job = oracle.make_job(n, mode=mode, rule=rule, flags=oracle.F_SAMPLE, sample_ppm=50000, seed=12345)
    b = oracle.enumerate_job(job)
    f = oracle.floyd_sample_job(job)
    got = [(x.s_count, x.s_cyc, x.s_lamsum, x.s_lensum, x.s_maxfin) for x in (b, f)]
    assert got[0] == got[1]
    assert 0.03 * b.done < b.s_count < 0.07 * b.done


def test_play_one(oracle):
    # data/checks.txt:11: the 5-card cycles have length 6
    assert oracle.play_one([3, 1, 0], [4, 2])[0] in (True, False)
    cyc, rounds, lam = oracle.play_one([4, 0], [3, 1, 2])
    assert rounds > 0


@pytest.mark.skipif(not __import__("os").access(__import__("os").path.join(
    __import__("os").path.dirname(__import__("os").path.dirname(__import__("os").path.abspath(__file__))),
    "oracle", "_ref", "war"), __import__("os").X_OK), reason="reference cpu/war.cpp not built here")
def test_oracle_matches_reference_war_cpp(oracle):
    for n in range(2, 11):
        for rule in (0, 1):
            deals, cyc, longest = oracle.ref_war(n, rule)
            r = oracle.enumerate_job(oracle.make_job(n, rule=rule))
            assert (r.done, r.cyc, r.maxfin) == (deals, cyc, longest), (n, rule)


@pytest.mark.skipif(not __import__("os").access(__import__("os").path.join(
    __import__("os").path.dirname(__import__("os").path.dirname(__import__("os").path.abspath(__file__))),
    "oracle", "_ref", "distinct_cycles"), __import__("os").X_OK), reason="reference distinct_cycles.c not built here")
def test_oracle_matches_reference_distinct_cycles(oracle):
    for n in range(5, 11):
        cycling, oncycle, distinct, lens = oracle.ref_distinct(n, 2)
        r = oracle.enumerate_job(oracle.make_job(n, mode=oracle.CANON, flags=oracle.F_DISTINCT, dbins=64))
        assert (r.cyc, r.oncycle, r.distinct_min) == (cycling, oncycle, distinct)


@pytest.mark.parametrize("rule", [0, 1])
def test_held_out_restatement_agrees(oracle, golden, rule):
    """The restatement of gpu/war17.py (card n-1 held out of the piles) against the war_gpu.py restatement
    for every deal of n <= 10, and against the recorded a(n) and longest game."""
    for n in range(2, 11):
        a = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, 0, rule, 0, 0, None, 128)))
        b = oracle.to_dict(oracle.enumerate_held(oracle.make_job(n, 0, rule, 0, 0, None, 128)))
        for k in ("cyc", "done", "maxfin", "hist", "endhist"):
            assert a[k] == b[k], (n, rule, k)
        if rule == 0:
            g = golden["deals_rule0"][n]
            assert (b["cyc"], b["done"], b["maxfin"]) == (g["cyc"], g["deals"], g["longest"])


def test_war24_restatement_against_recorded_lines(oracle, golden):
    """The oracle's restatement of gpu/war24.py reproduces the recorded runs it can finish here
    (data/checks.txt:73-78: n = 5, 7, 9, 11 with the streak test, n = 10 with Floyd)."""
    seen = 0
    for e in golden["war24"]:
        if e["hi"] - e["lo"] > 5 * 10 ** 7:
            continue
        det = oracle.DET_STREAK if e["det"] == "streak" else oracle.DET_FLOYD
        r = oracle.war24(oracle.make_job(e["n"], lo=e["lo"], hi=e["hi"]), det)
        assert (r.done, r.cyc, r.maxfin, r.undetermined) == (e["deals"], e["cyc"], e["longest"], e["undetermined"])
        seen += 1
    assert seen == 5


@pytest.mark.parametrize("rule", [0, 1])
def test_war24_brent_equals_the_4bit_oracle(oracle, rule):
    """5-bit piles with Brent's reference schedule play exactly the 4-bit oracle's games: the same turn totals,
    cycle lengths and ending lengths; Floyd and the streak test (rule 0, odd n) agree on every count."""
    for n in range(2, 11):
        a = oracle.to_dict(oracle.war24(oracle.make_job(n, rule=rule, hbins=256), oracle.DET_BRENT, 1))
        b = oracle.to_dict(oracle.enumerate_job(oracle.make_job(n, rule=rule, hbins=256)))
        for k in ("cyc", "done", "maxfin", "turns", "hist", "endhist"):
            assert a[k] == b[k], (n, k)
        f = oracle.war24(oracle.make_job(n, rule=rule), oracle.DET_FLOYD)
        assert (f.cyc, f.done, f.maxfin, f.undetermined) == (b["cyc"], b["done"], b["maxfin"], 0)
        if n % 2 and not rule:
            s = oracle.war24(oracle.make_job(n), oracle.DET_STREAK)
            assert (s.cyc, s.done, s.maxfin, s.undetermined) == (b["cyc"], b["done"], b["maxfin"], 0)


def test_war24_step_cap(oracle):
    """Below the games' lengths the step cap turns undecided games into undetermined ones, and only those."""
    job = oracle.make_job(9)
    full = oracle.war24(job, oracle.DET_FLOYD)
    for det in (oracle.DET_FLOYD, oracle.DET_STREAK, oracle.DET_BRENT):
        r = oracle.war24(job, det, 1, 20)
        assert r.undetermined > 0
        assert r.cyc + r.undetermined + sum(r.endhist) == full.done
        assert r.maxfin <= 22 and r.cyc <= full.cyc
