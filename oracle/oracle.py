"""The oracle's Python face.  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it as the checker; the product never imports it.

* ``enumerate_job(job)``  -- liboracle.so (war_oracle.c), the C restatement of gpu/war_gpu.py.
* ``floyd_sample_job(job)`` -- the same sample played with Floyd (gpu/war_gpu_floyd.py:95-105).
* ``war24(job, det)``     -- the 5-bit program of gpu/war24.py (n <= 20, Floyd / streak test / Brent).
* ``ref_war(n, rule)``    -- the reference's own cpu/war.cpp, compiled unmodified into oracle/_ref/
                             (result line format cpu/war.cpp:59), when that binary is present.
* ``ref_distinct(n, t)``  -- cpu/distinct_cycles.c from oracle/_ref/ (output cpu/distinct_cycles.c:144-147).
"""
import ctypes
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

WAR_MAX_N = 16
WAR_HBINS_MAX = 4096
WAR_DBINS_MAX = 4096
WAR_EBINS = 1024
DEALS, CANON = 0, 1
F_HALF, F_DISTINCT, F_SHAPE, F_SAMPLE = 1, 2, 4, 8


class Job(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("mode", ctypes.c_int32), ("rule", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("hbins", ctypes.c_int32), ("dbins", ctypes.c_int32),
                ("blk", ctypes.c_int32), ("sample_ppm", ctypes.c_uint32),
                ("lo", ctypes.c_uint64), ("hi", ctypes.c_uint64), ("seed", ctypes.c_uint64)]


class Result(ctypes.Structure):
    _fields_ = [("cyc", ctypes.c_uint64), ("done", ctypes.c_uint64), ("maxfin", ctypes.c_uint64),
                ("turns", ctypes.c_uint64), ("shape_nonstd", ctypes.c_uint64),
                ("shape_unchecked", ctypes.c_uint64), ("oncycle", ctypes.c_uint64),
                ("distinct_min", ctypes.c_uint64), ("s_count", ctypes.c_uint64),
                ("s_cyc", ctypes.c_uint64), ("s_lamsum", ctypes.c_uint64),
                ("s_lensum", ctypes.c_uint64), ("s_maxfin", ctypes.c_uint64),
                ("units", ctypes.c_uint64), ("memo_lookups", ctypes.c_uint64), ("memo_hits", ctypes.c_uint64),
                ("memo_stores", ctypes.c_uint64), ("undetermined", ctypes.c_uint64), ("kernel_ms", ctypes.c_double),
                ("hbins", ctypes.c_int32), ("dbins", ctypes.c_int32), ("blk", ctypes.c_int32),
                ("status", ctypes.c_int32),
                ("hist", ctypes.c_uint64 * WAR_HBINS_MAX), ("dhist", ctypes.c_uint64 * WAR_DBINS_MAX),
                ("endhist", ctypes.c_uint64 * WAR_EBINS)]


_lib = None


def lib():
    """Loads liboracle.so, building it with make if it is missing."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, capture_output=True)
        _lib = ctypes.CDLL(path)
        _lib.oracle_enumerate.argtypes = [ctypes.POINTER(Job), ctypes.c_int, ctypes.POINTER(Result)]
        _lib.oracle_floyd_sample.argtypes = [ctypes.POINTER(Job), ctypes.c_int, ctypes.POINTER(Result)]
        _lib.oracle_enumerate_held.argtypes = [ctypes.POINTER(Job), ctypes.c_int, ctypes.POINTER(Result)]
        _lib.oracle_war24.argtypes = [ctypes.POINTER(Job), ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                                      ctypes.POINTER(Result)]
        _lib.oracle_play_one.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                         ctypes.POINTER(ctypes.c_uint64)]
        _lib.oracle_space_size.restype = ctypes.c_uint64
        _lib.oracle_space_size.argtypes = [ctypes.c_int, ctypes.c_int]
        _lib.oracle_result_size.restype = ctypes.c_size_t
        _lib.oracle_sample_pick.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64]
        assert _lib.oracle_result_size() == ctypes.sizeof(Result)
    return _lib


def make_job(n, mode=DEALS, rule=0, flags=0, lo=0, hi=None, hbins=0, dbins=0, blk=0, sample_ppm=0, seed=0):
    if hi is None:
        hi = space_size(n, mode)
    return Job(n, mode, rule, flags, hbins, dbins, blk, sample_ppm, lo, hi, seed)


def space_size(n, mode=DEALS):
    return lib().oracle_space_size(n, mode)


def to_dict(r, hbins=None, dbins=None):
    """The result as plain Python values; histograms as {bin: count} without zero bins."""
    out = {k: getattr(r, k) for k, _ in Result._fields_ if k not in ("hist", "dhist", "endhist")}
    hb = r.hbins if hbins is None else hbins
    db = r.dbins if dbins is None else dbins
    out["hist"] = {i: int(v) for i, v in enumerate(r.hist[:max(hb, 0)]) if v}
    out["dhist"] = {i: int(v) for i, v in enumerate(r.dhist[:max(db, 0)]) if v}
    out["endhist"] = {i: int(v) for i, v in enumerate(r.endhist) if v}
    return out


def enumerate_job(job, threads=0):
    r = Result()
    st = lib().oracle_enumerate(ctypes.byref(job), threads, ctypes.byref(r))
    if st != 0:
        raise ValueError("oracle_enumerate: status %d" % st)
    return r


def enumerate_held(job, threads=0):
    """The held-out-card program of gpu/war17.py on ranks [lo, hi) of the n! deals (n <= 17)."""
    r = Result()
    st = lib().oracle_enumerate_held(ctypes.byref(job), threads, ctypes.byref(r))
    if st != 0:
        raise ValueError("oracle_enumerate_held: status %d" % st)
    return r


DET_BRENT, DET_FLOYD, DET_STREAK = 0, 1, 2


def war24(job, det=DET_STREAK, window=1, cap=0, threads=0):
    """The 5-bit program of gpu/war24.py on ranks [lo, hi) of the n! deals (n <= 20): cyc, done, maxfin,
    undetermined, turns (steps played) and, with Brent, the cycle-length histogram."""
    r = Result()
    st = lib().oracle_war24(ctypes.byref(job), det, window, cap, threads, ctypes.byref(r))
    if st != 0:
        raise ValueError("oracle_war24: status %d" % st)
    return r


def floyd_sample_job(job, threads=0):
    r = Result()
    st = lib().oracle_floyd_sample(ctypes.byref(job), threads, ctypes.byref(r))
    if st != 0:
        raise ValueError("oracle_floyd_sample: status %d" % st)
    return r


def play_one(p1, p2, rule=0):
    """Plays one position given as card lists (top first).  Returns (cycles, rounds, lam)."""
    w1 = sum(c << (4 * i) for i, c in enumerate(p1))
    w2 = sum(c << (4 * i) for i, c in enumerate(p2))
    rounds, lam = ctypes.c_uint64(), ctypes.c_uint64()
    cyc = lib().oracle_play_one(w1, len(p1), w2, len(p2), rule, ctypes.byref(rounds), ctypes.byref(lam))
    return bool(cyc), rounds.value, lam.value


def sample_pick(seed, ppm, w1s, w2s):
    return bool(lib().oracle_sample_pick(seed, ppm, w1s, w2s))


def ref_available(name="war"):
    return os.access(os.path.join(REF_DIR, name), os.X_OK)


def ref_war(n, rule=0, threads=None, timeout=None):
    """Runs the reference's cpu/war.cpp (compiled unmodified) and parses its result line
    (cpu/war.cpp:59).  Returns (deals, cycling, longest_finite)."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    p = subprocess.run([os.path.join(REF_DIR, "war"), str(n), str(rule)], capture_output=True, text=True,
                       env=env, timeout=timeout, check=True)
    m = re.search(r"n=(\d+) mode=(\d+) deals=(\d+) cycling=(\d+) longest_finite=(\d+)", p.stdout)
    return int(m.group(3)), int(m.group(4)), int(m.group(5))


def ref_distinct(n, threads=1, timeout=None):
    """Runs the reference's cpu/distinct_cycles.c; returns (cycling, on_cycle, distinct, {len: cycles})."""
    p = subprocess.run([os.path.join(REF_DIR, "distinct_cycles"), str(n), str(threads)], capture_output=True,
                       text=True, timeout=timeout, check=True)
    m = re.search(r"never end (\d+); on a cycle (\d+); DISTINCT cycles up to swap (\d+)", p.stdout)
    lens = {int(a): int(b) for a, b in re.findall(r" (\d+):(\d+)", p.stdout.split("\n", 1)[1])}
    return int(m.group(1)), int(m.group(2)), int(m.group(3)), lens
