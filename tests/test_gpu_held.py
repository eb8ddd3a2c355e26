"""The held-out-card engine (war_enumerate_held, the n <= 17 program gpu/war17.py): bit-exact against the
oracle's restatement of gpu/war17.py and against the main engine where both apply, and against the
recorded a(12), a(13) and histogram."""
import random

import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("cyc", "done", "maxfin", "hist", "endhist")


def held(wl, n, rule=0, lo=0, hi=None, hbins=128, tune=None):
    return wl.to_dict(wl.enumerate_held(wl.make_job(n, rule=rule, lo=lo, hi=hi, hbins=hbins), tune))


def oracle_held(oracle, n, rule=0, lo=0, hi=None, hbins=128):
    import math
    hi = math.factorial(n) if hi is None else hi
    return oracle.to_dict(oracle.enumerate_held(oracle.make_job(n, 0, rule, 0, lo, hi, hbins)))


# tune.variant of the held-out engine, bits 0-1 the turn: 0 counts packed in one word with multiply-add card
# arithmetic (the default), 1 multiply-adds on separate counts, 2 packed counts in logic/shift form, 3 the plain
# branching turn of gpu/war17.py; bit 2 the path memo; bit 3 the tortoise checkpoint tested after every turn
# (else saved at the services where the window is a multiple of the service period)
@pytest.mark.parametrize("rule,variant", [(r, v) for r in (0, 1) for v in (0, 1, 2, 3, 8, 9, 10, 11)])
def test_small_n_full_against_oracle_and_main_engine(wl, oracle, rule, variant):
    """Every deal of n <= 11, every turn form of the held-out engine, with the checkpoint saved at the services
    and (variants 8..11) after every turn."""
    for n in range(2, 12):
        got = held(wl, n, rule, tune=wl.make_tune(variant=variant))
        want = oracle_held(oracle, n, rule)
        main = wl.to_dict(wl.enumerate_job(wl.make_job(n, rule=rule, hbins=128)))
        for k in FIELDS:
            assert got[k] == want[k] == main[k], (n, rule, k)


def test_a12_a13_recorded(wl, golden):
    for n in (12, 13):
        r = held(wl, n, hbins=256)
        g = golden["deals_rule0"][n]
        assert (r["done"], r["cyc"], r["maxfin"], r["hist"]) == (g["deals"], g["cyc"], g["longest"], g["hist"])


def test_recorded_17_card_slices(wl, golden):
    """The reference's recorded 17-card runs that take seconds here (gpu/war24.py, data/long_runs.txt:61-75): 1e9
    deals from 10^14, the first 8,992,587,776 deals and the last 785,219,584, through the held-out engine's
    default turn and through the plain branching turn (variant 3) on the middle slice."""
    seen = set()
    for e in golden["war24"]:
        if e["n"] != 17 or e["hi"] - e["lo"] > 10 ** 10 or (e["lo"], e["hi"]) in seen:
            continue
        seen.add((e["lo"], e["hi"]))
        r = wl.enumerate_held(wl.make_job(17, lo=e["lo"], hi=e["hi"]))
        assert (r.done, r.cyc, r.maxfin, r.undetermined) == (e["deals"], e["cyc"], e["longest"], 0), e
        if e["lo"] == 10 ** 14:
            r3 = wl.enumerate_held(wl.make_job(17, lo=e["lo"], hi=e["hi"]), wl.make_tune(variant=3))
            assert (r3.done, r3.cyc, r3.maxfin, r3.turns) == (r.done, r.cyc, r.maxfin, r.turns)
    assert len(seen) == 3


@pytest.mark.parametrize("n", [14, 15, 16, 17])
def test_slices_against_oracle(wl, oracle, n):
    import math
    rnd = random.Random(n)
    total = math.factorial(n)
    for _ in range(4):
        lo = rnd.randrange(0, total)
        hi = min(total, lo + rnd.choice([1, 5, 999, 40320, 300001]))
        rule = rnd.randint(0, 1)
        got, want = held(wl, n, rule, lo, hi, 256), oracle_held(oracle, n, rule, lo, hi, 256)
        for k in FIELDS:
            assert got[k] == want[k], (n, lo, hi, rule, k)
    for lo in (0, total - 720 * 33 - 17):   # the first and the last deals of the space
        got, want = held(wl, n, 0, lo, lo + 720 * 33 + 17, 256), oracle_held(oracle, n, 0, lo, lo + 720 * 33 + 17, 256)
        for k in FIELDS:
            assert got[k] == want[k], (n, lo, k)


def test_n16_slice_against_main_engine(wl):
    job = dict(lo=10 ** 13, hi=10 ** 13 + 5 * 10 ** 7, hbins=256)
    got = held(wl, 16, **job)
    main = wl.to_dict(wl.enumerate_plain(wl.make_job(16, **job)))
    for k in FIELDS:
        assert got[k] == main[k], k


def test_n17_through_war_enumerate_and_tunes(wl, oracle):
    lo, hi = 2 * 10 ** 14 + 12345, 2 * 10 ** 14 + 12345 + 250000
    want = oracle_held(oracle, 17, 0, lo, hi, 256)
    got = wl.to_dict(wl.enumerate_job(wl.make_job(17, lo=lo, hi=hi, hbins=256)))   # routed to the held engine
    for k in FIELDS:
        assert got[k] == want[k], k
    for t in (dict(threads=128), dict(threads=1024, defer=4), dict(block_m=3, defer=16), dict(block_m=8, window=1),
              dict(blocks_per_sm=1, window=128), dict(variant=1), dict(variant=1, threads=1024, rule=0),
              dict(variant=5, memo_bits=20), dict(variant=2), dict(variant=2, defer=12), dict(variant=10),
              dict(variant=2, window=1, block_m=5), dict(variant=6, memo_bits=20), dict(variant=4, memo_bits=20),
              dict(variant=3), dict(variant=3, defer=32), dict(variant=3, defer=20), dict(variant=11),
              dict(variant=3, window=8, defer=12), dict(variant=7, memo_bits=20), dict(variant=15, memo_bits=20)):
        t.pop("rule", None)
        got = held(wl, 17, 0, lo, hi, 256, wl.make_tune(**t))
        for k in FIELDS:
            assert got[k] == want[k], (t, k)


def test_refusals(wl):
    import warlib
    for bad in (dict(n=1), dict(n=18), dict(n=9, mode=1), dict(n=9, flags=warlib.F_SAMPLE)):
        job = wl.make_job(**bad)
        with pytest.raises(warlib.WarError):
            wl.enumerate_held(job)


def memo_held(wl, bits=24, **kw):
    t = dict(variant=4, threads=256, memo_bits=bits)   # the default turn with the path memo
    t.update(kw)
    return wl.make_tune(**t)


@pytest.mark.parametrize("bits,variant", [(12, 4), (24, 4), (24, 5), (24, 6), (24, 7), (12, 7)])
def test_memo_small_n_and_slices(wl, oracle, bits, variant):
    """The held-out engine with the path memo (its own 63/64-bit state keys) against the oracle: every deal
    of n <= 11, slices of n = 14..17, and a table far too small (2^12 words)."""
    for n in range(4, 12):
        got, want = held(wl, n, n & 1, tune=memo_held(wl, bits, variant=variant)), oracle_held(oracle, n, n & 1)
        for k in FIELDS:
            assert got[k] == want[k], (n, k)
    rnd = random.Random(bits)
    import math
    for n in (14, 15, 16, 17):
        lo = rnd.randrange(0, math.factorial(n) - 10 ** 6)
        hi = lo + rnd.choice([777, 300001, 10 ** 6])
        rule = rnd.randint(0, 1)
        got, want = held(wl, n, rule, lo, hi, 256, memo_held(wl, bits, variant=variant)), oracle_held(oracle, n, rule, lo, hi, 256)
        for k in FIELDS:
            assert got[k] == want[k], (n, lo, hi, k)


def test_memo_a13_and_long_n17_slice(wl, golden):
    r = held(wl, 13, hbins=256, tune=memo_held(wl, 28))
    g = golden["deals_rule0"][13]
    assert (r["done"], r["cyc"], r["maxfin"], r["hist"]) == (g["deals"], g["cyc"], g["longest"], g["hist"])
    lo, hi = 10 ** 14, 10 ** 14 + 2 * 10 ** 8
    a = held(wl, 17, 0, lo, hi, 256, memo_held(wl, 26))
    b = held(wl, 17, 0, lo, hi, 256)
    for k in FIELDS:
        assert a[k] == b[k], k


def test_memo_kept_only_for_the_same_key_format(wl):
    """A table left by the main engine (n = 16 keys) is not reused by the held-out engine, whose keys mean
    other states, even with WAR_F_MEMO_KEEP."""
    import warlib
    lo, hi = 10 ** 13, 10 ** 13 + 10 ** 7
    t_main = wl.make_tune(variant=31, games=1, threads=256, defer=8, block_m=6, memo_bits=22)
    wl.enumerate_job(wl.make_job(16, lo=lo, hi=hi, hbins=128), t_main)
    job = wl.make_job(16, flags=warlib.F_MEMO_KEEP, lo=lo, hi=hi, hbins=128)
    a = wl.to_dict(wl.enumerate_held(job, memo_held(wl, 22)))
    b = held(wl, 16, 0, lo, hi, 128)
    for k in FIELDS:
        assert a[k] == b[k], k
