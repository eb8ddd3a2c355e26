"""libwar.so on a machine without a GPU: it loads, exports every function include/war.h declares, its
host-only entry points work (plan, sample predicate, errors), and every compute entry point refuses to
run without a device (there is no CPU fallback)."""
import ctypes
import math
import os
import random
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:int|uint64_t|void)\s+\**\s*(war_\w+)\s*\(", src, flags=re.M)
    return names


def test_library_exports_every_declared_symbol():
    import warlib
    L = warlib.lib()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
    assert set(names) <= set(warlib.SYMBOLS), set(names) - set(warlib.SYMBOLS)


def test_sample_pick_matches_oracle(oracle):
    import warlib
    rnd = random.Random(5)
    for _ in range(2000):
        w1, w2 = rnd.getrandbits(60), rnd.getrandbits(60)
        seed, ppm = rnd.getrandbits(64), rnd.choice([0, 1, 10000, 500000, 1000000])
        assert warlib.sample_pick(seed, ppm, w1, w2) == oracle.sample_pick(seed, ppm, w1, w2)


def test_compute_entry_points_fail_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import warlib
    with pytest.raises(warlib.WarError) as e:
        warlib.enumerate_job(warlib.make_job(9))
    assert e.value.status in (-8, -2)
    with pytest.raises(warlib.WarError):
        warlib.enumerate_plain(warlib.make_job(9))
    with pytest.raises(warlib.WarError):
        warlib.floyd_sample(warlib.make_job(9, flags=warlib.F_SAMPLE, sample_ppm=1000))
    with pytest.raises(warlib.WarError):
        warlib.autotune_native(warlib.make_job(9))


def test_argument_errors():
    import warlib
    for bad in (dict(n=0), dict(n=17), dict(n=9, mode=2), dict(n=9, rule=2), dict(n=9, hbins=5000),
                dict(n=9, flags=warlib.F_HALF), dict(n=10, mode=warlib.CANON, flags=warlib.F_HALF),
                dict(n=9, lo=5, hi=4), dict(n=9, hi=math.factorial(9) + 1)):
        job = warlib.make_job(**bad) if "hi" in bad or bad.get("n", 9) in (0, 17) else warlib.make_job(**bad)
        with pytest.raises(warlib.WarError) as e:
            warlib.plan(job, 6)
        assert e.value.status == -1
        assert warlib.last_error()


def fact(k):
    return math.factorial(k)


def expand(n, mode, main_base, main_count, m, extra):
    """Every rank the plan covers, as a sorted list (small spaces only)."""
    s = n - 1 if mode else 1
    ranks = []
    units = [((main_base + u) * fact(m), m, 0, s if mode else 0) for u in range(main_count)] + extra
    for r, j, k0, k1 in units:
        assert r % fact(j) == 0
        for o in range(r, r + fact(j)):
            if mode:
                ranks += [o * s + k for k in range(k0, k1)]
            else:
                ranks.append(o)
    return sorted(ranks)


@pytest.mark.parametrize("mode", [0, 1])
def test_plan_covers_range_exactly(mode):
    import warlib
    rnd = random.Random(11 + mode)
    for n in (5, 6, 7, 8):
        total = warlib.space_size(n, mode)
        for _ in range(25):
            lo = rnd.randrange(0, total)
            hi = rnd.randrange(lo, total + 1)
            m = rnd.randint(1, 8)
            job = warlib.make_job(n, mode, lo=lo, hi=hi)
            mb, mc, extra = warlib.plan(job, m)
            mm = min(m, n - 1 if mode else n)
            got = expand(n, mode, mb, mc, mm, extra)
            assert got == list(range(lo, hi)), (n, mode, lo, hi, m)


def test_plan_full_space_is_main_units():
    import warlib
    mb, mc, extra = warlib.plan(warlib.make_job(13), 6)
    assert (mb, mc, extra) == (0, fact(13) // fact(6), [])
    mb, mc, extra = warlib.plan(warlib.make_job(14, warlib.CANON), 5)
    assert (mb, mc, extra) == (0, fact(13) // fact(5), [])


C_CALLER = r"""
#include "war.h"
#include <stdio.h>
#include <stdlib.h>
int main(void) {
    war_job job = { .n = 11, .mode = WAR_DEALS, .hbins = 64, .lo = 0, .hi = 39916800ull };
    war_tune t = { .threads = 256, .games = 1, .block_m = 6, .window = 32, .defer = 8, .variant = 31, .memo_bits = 20 };
    war_result* r = (war_result*)malloc(sizeof *r);
    int st = war_enumerate(&job, &t, r);
    if (st != WAR_OK) { char e[256]; war_last_error(e, sizeof e); printf("status %d: %s\n", st, e); return 0; }
    printf("a(11)=%llu longest=%llu\n", (unsigned long long)r->cyc, (unsigned long long)r->maxfin);
    return 0;
}
"""


def test_header_is_plain_c_and_links(tmp_path):
    """include/war.h compiles as strict C99 and a C program links against libwar.so and runs: on a machine
    without a GPU it gets WAR_ENODEV and a message, with one it prints a(11)."""
    import os
    import subprocess
    import warlib
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(warlib.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(root, "include"),
                    str(src), "-L", libdir, "-lwar", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120).stdout
    assert out.startswith("status -8:") or out.startswith("a(11)=28223770 longest=41"), out


def test_held_engine_argument_errors():
    """war_enumerate_held validates before touching the device: bad jobs fail with WAR_EINVAL on any
    machine, an empty range succeeds without one."""
    import warlib
    for bad in (dict(n=1), dict(n=18, hi=1), dict(n=9, mode=warlib.CANON), dict(n=9, rule=2),
                dict(n=9, flags=warlib.F_SAMPLE), dict(n=9, flags=warlib.F_HALF), dict(n=9, hbins=5000),
                dict(n=17, hi=math.factorial(17) + 1), dict(n=9, lo=5, hi=4)):
        with pytest.raises(warlib.WarError) as e:
            warlib.enumerate_held(warlib.make_job(**bad))
        assert e.value.status == -1, bad
    r = warlib.enumerate_held(warlib.make_job(17, lo=123, hi=123, hbins=16))
    assert (r.done, r.cyc, r.hbins) == (0, 0, 16)
