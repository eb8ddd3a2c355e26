"""TEST INFRASTRUCTURE: the reference's own GPU path (gpu/war_gpu.py's kernels, compiled unmodified for
sm_100a by `make -C oracle ref-gpu`, driven by a restatement of run()'s launch loop) on this GPU.

    python oracle/ref_gpu.py 13 [--canon] [--hist 256] [--distinct] [--shape] [--rule R]

prints one JSON line with the reference's results and wall time (launch loop with a device
synchronisation after every launch, as CuPy does)."""
import argparse
import ctypes
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libwarref.so")


def available():
    return os.path.exists(LIB)


def run(n, canon=False, half=False, rule=0, hbins=0, dbins=0, shape=False, per=256, threads=256, batch_threads=1 << 18):
    L = ctypes.CDLL(LIB)
    out = (ctypes.c_ulonglong * 5)()
    h = (ctypes.c_ulonglong * max(hbins, 1))()
    d = (ctypes.c_ulonglong * max(dbins, 1))()
    ms = ctypes.c_double()
    blk = (n & -n) if (canon and shape) else 0
    st = L.ref_gpu_run(n, int(canon), int(half), rule, hbins, dbins if canon else 0, blk, per, threads,
                       ctypes.c_longlong(batch_threads), out, h, d, ctypes.byref(ms))
    if st != 0:
        raise RuntimeError("ref_gpu_run failed: %d" % st)
    return {"cyc": out[0], "done": out[1], "maxfin": out[2], "shape": [out[3], out[4]], "blk": blk,
            "hist": {i: int(v) for i, v in enumerate(h[:hbins]) if v},
            "dhist": {i: int(v) for i, v in enumerate(d[:dbins]) if v} if canon else {},
            "ms": ms.value}


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("n", type=int)
    ap.add_argument("--canon", action="store_true")
    ap.add_argument("--half", action="store_true")
    ap.add_argument("--rule", type=int, default=0)
    ap.add_argument("--hist", type=int, default=0)
    ap.add_argument("--distinct", action="store_true")
    ap.add_argument("--shape", action="store_true")
    a = ap.parse_args()
    r = run(a.n, a.canon, a.half, a.rule, a.hist, 4096 if a.distinct else 0, a.shape)
    space = (r["done"])
    r["rate_per_s"] = space / (r["ms"] * 1e-3) if r["ms"] else None
    r["impl"] = "reference gpu/war_gpu.py kernels (unmodified, nvcc sm_100a), run() launch loop restated"
    print(json.dumps(r))
