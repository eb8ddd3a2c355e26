"""ctypes binding of libwar.so, the sm_100a War enumerator (C ABI in include/war.h).

The library is built in place by build.py (nvcc, sm_100a).  Loading fails loudly when it is missing:
there is no CPU fallback anywhere in this package.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwar.so")

WAR_MAX_N = 16
WAR_HBINS_MAX = 4096
WAR_DBINS_MAX = 4096
WAR_EBINS = 1024
DEALS, CANON = 0, 1
F_HALF, F_DISTINCT, F_SHAPE, F_SAMPLE, F_MEMO_KEEP = 1, 2, 4, 8, 16

STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "timeout", -4: "out of memory",
          -5: "busy", -6: "not found", -7: "turn cap exceeded", -8: "no CUDA device", 1: "pending"}
PENDING = 1


class WarError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d: %s)" % (msg, status, STATUS.get(status, "?")))
        self.status = status


class Job(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("mode", ctypes.c_int32), ("rule", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("hbins", ctypes.c_int32), ("dbins", ctypes.c_int32),
                ("blk", ctypes.c_int32), ("sample_ppm", ctypes.c_uint32),
                ("lo", ctypes.c_uint64), ("hi", ctypes.c_uint64), ("seed", ctypes.c_uint64)]


class Tune(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32), ("games", ctypes.c_int32),
                ("block_m", ctypes.c_int32), ("window", ctypes.c_int32), ("defer", ctypes.c_int32),
                ("variant", ctypes.c_int32), ("memo_bits", ctypes.c_int32), ("chunk", ctypes.c_int32)]


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


class ServerCfg(ctypes.Structure):
    _fields_ = [("max_jobs", ctypes.c_int32), ("queue_cap", ctypes.c_int32), ("mem_budget", ctypes.c_uint64),
                ("tick_ranks", ctypes.c_uint64), ("threads", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("memo_bits", ctypes.c_int32), ("reserved", ctypes.c_int32 * 3)]


class JobStatus(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("status", ctypes.c_int32), ("submit_ms", ctypes.c_double),
                ("admit_ms", ctypes.c_double), ("finish_ms", ctypes.c_double)]


class WideCfg(ctypes.Structure):
    _fields_ = [("det", ctypes.c_int32), ("cap", ctypes.c_uint32), ("threads", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("block_m", ctypes.c_int32), ("window", ctypes.c_int32),
                ("defer", ctypes.c_int32), ("reserved", ctypes.c_int32)]


DET_BRENT, DET_FLOYD, DET_STREAK = 0, 1, 2


class DeviceInfo(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("sm_count", ctypes.c_int32), ("cc_major", ctypes.c_int32),
                ("cc_minor", ctypes.c_int32), ("clock_mhz", ctypes.c_int32), ("max_threads_per_sm", ctypes.c_int32),
                ("mem_free", ctypes.c_uint64), ("mem_total", ctypes.c_uint64), ("name", ctypes.c_char * 128)]


class Unit(ctypes.Structure):
    _fields_ = [("r", ctypes.c_uint64), ("j", ctypes.c_uint32), ("k0", ctypes.c_uint32), ("k1", ctypes.c_uint32),
                ("pad", ctypes.c_uint32)]


U64P = ctypes.POINTER(ctypes.c_uint64)
SYMBOLS = {
    "war_count_launch": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_uint64, U64P, U64P, U64P, U64P, ctypes.c_int32]),
    "war_canon_launch": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_uint64, U64P, U64P, U64P, U64P, ctypes.c_int32, U64P,
                                        ctypes.c_int32, U64P, ctypes.c_int32]),
    "war_enumerate_plain": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(Result)]),
    "war_enumerate": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(Tune), ctypes.POINTER(Result)]),
    "war_enumerate_held": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(Tune), ctypes.POINTER(Result)]),
    "war_enumerate_wide": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(WideCfg), ctypes.POINTER(Result)]),
    "war_floyd_sample": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(Result)]),
    "war_enumerate_noalloc": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(Tune), ctypes.POINTER(Result)]),
    "war_autotune": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(Tune), ctypes.c_double, ctypes.c_int32,
                                    ctypes.POINTER(Tune), ctypes.POINTER(ctypes.c_double)]),
    "war_server_create": (ctypes.c_int, [ctypes.POINTER(ServerCfg), ctypes.POINTER(ctypes.c_void_p)]),
    "war_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), U64P]),
    "war_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result), ctypes.POINTER(JobStatus)]),
    "war_server_drain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "war_server_stats": (ctypes.c_int, [ctypes.c_void_p, U64P, U64P, U64P]),
    "war_server_memo_info": (ctypes.c_int, [ctypes.c_void_p, U64P, U64P, ctypes.POINTER(ctypes.c_int32)]),
    "war_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "war_device_info_get": (ctypes.c_int, [ctypes.POINTER(DeviceInfo)]),
    "war_set_stream": (ctypes.c_int, [ctypes.c_void_p]),
    "war_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "war_launch_count": (ctypes.c_uint64, []),
    "war_sample_pick": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64]),
    "war_measure_int_peak": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "war_measure_gather_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "war_plan": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.c_int32, U64P, U64P, ctypes.POINTER(Unit), ctypes.c_int32]),
}

_lib = None


def lib():
    """The loaded libwar.so.  Raises if it has not been built: no fallback exists."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libwar.so is not built at %s: run python %s/build.py" % (LIB_PATH, HERE))
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SYMBOLS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    lib().war_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status, what):
    if status < 0:
        raise WarError(status, "%s: %s" % (what, last_error()))
    return status


def space_size(n, mode=DEALS):
    import math
    if mode == CANON:
        return 0 if n < 2 else math.factorial(n - 1) * (n - 1)
    return math.factorial(n)


def make_job(n, mode=DEALS, rule=0, flags=0, lo=0, hi=None, hbins=0, dbins=0, blk=0, sample_ppm=0, seed=0):
    if hi is None:
        hi = space_size(n, mode)
    return Job(n, mode, rule, flags, hbins, dbins, blk, sample_ppm, lo, hi, seed)


def make_tune(threads=0, blocks_per_sm=0, games=0, block_m=0, window=0, defer=0, variant=0, memo_bits=0, chunk=0):
    return Tune(threads, blocks_per_sm, games, block_m, window, defer, variant, memo_bits, chunk)


def enumerate_job(job, tune=None):
    """The persistent refill kernel over the job's ranks (war_enumerate)."""
    r = Result()
    check(lib().war_enumerate(ctypes.byref(job), ctypes.byref(tune) if tune is not None else None, ctypes.byref(r)),
          "war_enumerate")
    return r


def autotune_native(job, start=None, slice_ms=400.0, passes=2):
    """war_autotune: (best war_tune, its kernel ms) for the job's class, searched in the library."""
    best, ms = Tune(), ctypes.c_double()
    check(lib().war_autotune(ctypes.byref(job), ctypes.byref(start) if start is not None else None, slice_ms, passes,
                             ctypes.byref(best), ctypes.byref(ms)), "war_autotune")
    return best, ms.value


def enumerate_held(job, tune=None):
    """war_enumerate_held: deals of up to 17 cards with the held-out-card engine."""
    r = Result()
    check(lib().war_enumerate_held(ctypes.byref(job), ctypes.byref(tune) if tune is not None else None,
                                   ctypes.byref(r)), "war_enumerate_held")
    return r


def enumerate_wide(job, det=DET_BRENT, cap=0, threads=0, blocks_per_sm=0, block_m=0, window=0, defer=0):
    """war_enumerate_wide: deals of up to 20 cards with the 5-bit-pile engine (gpu/war24.py)."""
    r = Result()
    cfg = WideCfg(det, cap, threads, blocks_per_sm, block_m, window, defer, 0)
    check(lib().war_enumerate_wide(ctypes.byref(job), ctypes.byref(cfg), ctypes.byref(r)), "war_enumerate_wide")
    return r


def enumerate_noalloc(job, tune=None):
    """war_enumerate_noalloc: the same enumeration with the library's static scratch instead of allocated
    device memory, for callers that cannot allocate (see include/war.h)."""
    r = Result()
    check(lib().war_enumerate_noalloc(ctypes.byref(job), ctypes.byref(tune) if tune is not None else None,
                                      ctypes.byref(r)), "war_enumerate_noalloc")
    return r


def enumerate_plain(job):
    """The plain kernel (the reference's per-thread rank blocks) over the job (war_enumerate_plain)."""
    r = Result()
    check(lib().war_enumerate_plain(ctypes.byref(job), ctypes.byref(r)), "war_enumerate_plain")
    return r


def floyd_sample(job):
    """Floyd over the job's seeded sample (war_floyd_sample): fills the s_* fields."""
    r = Result()
    check(lib().war_floyd_sample(ctypes.byref(job), ctypes.byref(r)), "war_floyd_sample")
    return r


def count_launch(n, start, total, per, half_rule, threads, nthreads, acc, hist):
    """One launch of the plain deals kernel with the reference kernel's arguments; acc = [cyc, done, maxfin]
    and hist (list of hbins ints) are added to in place (gpu/war_gpu.py:121-124)."""
    c, d, m = ctypes.c_uint64(acc[0]), ctypes.c_uint64(acc[1]), ctypes.c_uint64(acc[2])
    h = (ctypes.c_uint64 * max(1, len(hist)))(*hist)
    check(lib().war_count_launch(n, start, total, per, half_rule, threads, nthreads, ctypes.byref(c),
                                 ctypes.byref(d), ctypes.byref(m), h, len(hist)), "war_count_launch")
    acc[:] = [c.value, d.value, m.value]
    hist[:] = list(h)[:len(hist)]


def device_info():
    d = DeviceInfo()
    check(lib().war_device_info_get(ctypes.byref(d)), "war_device_info_get")
    return d


def launch_count():
    return int(lib().war_launch_count())


def sample_pick(seed, ppm, w1s, w2s):
    return bool(lib().war_sample_pick(seed, ppm, w1s, w2s))


def to_dict(r, hbins=None, dbins=None):
    """A result as plain Python values; histograms as {bin: count} without empty bins."""
    out = {k: getattr(r, k) for k, _ in Result._fields_ if k not in ("hist", "dhist", "endhist")}
    hb = r.hbins if hbins is None else hbins
    db = r.dbins if dbins is None else dbins
    out["hist"] = {i: int(v) for i, v in enumerate(r.hist[:max(hb, 0)]) if v}
    out["dhist"] = {i: int(v) for i, v in enumerate(r.dhist[:max(db, 0)]) if v}
    out["endhist"] = {i: int(v) for i, v in enumerate(r.endhist) if v}
    return out


def plan(job, block_m):
    """The work units war_enumerate runs for a job: (main_base, main_count, [(r, j, k0, k1), ...])."""
    cap = 4096
    units = (Unit * cap)()
    mb, mc = ctypes.c_uint64(), ctypes.c_uint64()
    k = check(lib().war_plan(ctypes.byref(job), block_m, ctypes.byref(mb), ctypes.byref(mc), units, cap), "war_plan")
    return mb.value, mc.value, [(u.r, u.j, u.k0, u.k1) for u in units[:min(k, cap)]]


def measure_int_peak():
    """(issue, alu) integer thread-instructions per second measured on this GPU (war_measure_int_peak)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    check(lib().war_measure_int_peak(ctypes.byref(a), ctypes.byref(b)), "war_measure_int_peak")
    return a.value, b.value


def measure_gather_peak(table_bits=30, bucket_bytes=8):
    """Random lookups per second from a table of 2^table_bits words (war_measure_gather_peak)."""
    v = ctypes.c_double()
    check(lib().war_measure_gather_peak(table_bits, bucket_bytes, ctypes.byref(v)), "war_measure_gather_peak")
    return v.value


def set_stream(stream_handle):
    """Launch on this cudaStream_t (an int handle, e.g. torch.cuda.current_stream().cuda_stream); 0 = own stream."""
    check(lib().war_set_stream(ctypes.c_void_p(stream_handle or None)), "war_set_stream")
