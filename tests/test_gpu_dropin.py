"""The drop-in program on the GPU engine (gpu/war_gpu.py:272-398): `war_gpu.main` prints the reference's
recorded output lines byte for byte apart from the time, for a(13), the n = 14 canonical scan and a(14) with
--half; an interrupted n = 13 run resumes from its progress file, keeping the cycle memo between the spans of
one process; and progress files written by the reference itself (tests/golden/progress_*_ref.json, in the
schema of gpu/war_gpu.py:331-338) resume to the recorded totals."""
import contextlib
import io
import json
import os
import re
import shutil

import pytest

pytestmark = pytest.mark.gpu

TIME = re.compile(r"  [0-9.]+s")
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def main_lines(argv):
    import war_gpu
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        war_gpu.main(argv)
    return [TIME.sub("  Xs", ln) for ln in buf.getvalue().splitlines()]


def strip(lines):
    return [TIME.sub("  Xs", ln) for ln in lines]


def test_a13_lines(wl, golden):
    """`war_gpu.py 13 --hist 256` (data/checks.txt:23-24)."""
    rec = golden["war_gpu_lines"]["deals_hist256"]
    i = next(k for k, ln in enumerate(rec) if ln.startswith("n=13 "))
    assert main_lines(["13", "--hist", "256"]) == strip(rec[i:i + 2])


def test_canon14_lines(wl, golden):
    """`war_gpu.py 14 --canon --distinct --shape --hist 256` (data/long_runs.txt:20-23)."""
    assert main_lines(["14", "--canon", "--distinct", "--shape", "--hist", "256"]) == \
        strip(golden["war_gpu_lines"]["long14_canon"])


def test_a14_half_lines(wl, golden):
    """`war_gpu.py 14 --half --hist 256` (data/long_runs.txt:14-15): 43,589,145,600 deals played, doubled."""
    assert main_lines(["14", "--half", "--hist", "256"]) == strip(golden["war_gpu_lines"]["long14_half"])


def test_interrupted_n13_resumes_with_memo_kept(wl, golden, monkeypatch, tmp_path):
    import warlib
    import war_gpu
    monkeypatch.setattr(war_gpu, "SPAN_RANKS", 1 << 30)            # 6 spans over the 13! deals
    real = warlib.enumerate_job
    calls = []

    def engine(job, tune=None, stop_after=None):
        calls.append((job.lo, job.hi, job.flags, tune.variant if tune is not None else None))
        if stop_after is not None and len(calls) > stop_after:
            raise KeyboardInterrupt("interrupted by the test")
        return real(job, tune)
    out = str(tmp_path / "n13")
    monkeypatch.setattr(warlib, "enumerate_job", lambda job, tune=None: engine(job, tune, stop_after=3))
    with pytest.raises(KeyboardInterrupt):
        war_gpu.run(13, out=out, hbins=256, quiet=True)
    with open(out + ".progress") as f:
        st = json.load(f)
    assert 0 < st["next_start"] < st["total"] and st["done"] == st["next_start"]
    assert calls[0][2] & warlib.F_MEMO_KEEP == 0 and all(c[2] & warlib.F_MEMO_KEEP for c in calls[1:])
    assert all(c[3] is not None and c[3] & 4 for c in calls)          # the memo tune from the cache
    first_resumed = len(calls)
    monkeypatch.setattr(warlib, "enumerate_job", lambda job, tune=None: engine(job, tune))
    c, d, mx, _, h, _, _ = war_gpu.run(13, out=out, resume=True, hbins=256, quiet=True)
    g = golden["deals_rule0"][13]
    assert (c, d, mx, h) == (g["cyc"], g["deals"], g["longest"], g["hist"])
    resumed = calls[first_resumed:]
    assert resumed[0][0] == st["next_start"] and resumed[0][2] & warlib.F_MEMO_KEEP == 0
    assert len(resumed) >= 2 and all(c[2] & warlib.F_MEMO_KEEP for c in resumed[1:])
    with open(out + ".progress") as f:
        assert json.load(f)["next_start"] == g["deals"]


@pytest.mark.parametrize("name,kw,key", [
    ("progress_deals13_ref.json", dict(hbins=256), "deals"),
    ("progress_canon13_ref.json", dict(canon=True, shape=True, dbins=4096), "canon"),
])
def test_resume_from_a_reference_progress_file(wl, golden, tmp_path, name, kw, key):
    """A progress file in the reference's schema, interrupted where the reference's launch loop would stop,
    resumes on the GPU engine to the recorded totals."""
    import war_gpu
    out = str(tmp_path / "run")
    shutil.copy(os.path.join(GOLDEN, name), out + ".progress")
    with open(out + ".progress") as f:
        before = json.load(f)
    c, d, mx, _, h, sh, dd = war_gpu.run(13, out=out, resume=True, quiet=True, **kw)
    if key == "deals":
        g = golden["deals_rule0"][13]
        assert (c, d, mx, h) == (g["cyc"], g["deals"], g["longest"], g["hist"])
    else:
        g = golden["canon_rule0"][13]
        assert (c, d, mx, dd) == (g["cycling"], g["positions"], g["longest"], g["dhist"])
        assert sh == (g["shape_nonstd"], g["shape_unchecked"], g["blk"])
        assert sum(v // k for k, v in dd.items()) == g["distinct"]
    with open(out + ".progress") as f:
        after = json.load(f)
    assert list(after) == list(before)                                 # the same schema, key for key
    assert after["next_start"] == after["total"] == before["total"]
