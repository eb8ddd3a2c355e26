"""The drop-in runner's host logic on the CPU (gpu/war_gpu.py:272-398): with the oracle standing in for
the engine, `war_gpu.main` prints the reference's recorded output lines byte for byte apart from the time,
an interrupted run resumes from its progress file to the same result, and every span of a run after its
first asks the engine to keep the cycle memo."""
import io
import json
import re
import contextlib

import pytest

TIME = re.compile(r"  [0-9.]+s")


def fake_engine(monkeypatch, oracle, calls=None, fail_after=None):
    """Replaces the engine entry points with the oracle on the same job (the oracle is the checker here:
    what is under test is the host code around the engine)."""
    import warlib
    import war_gpu

    def enum(job, tune=None):
        if calls is not None:
            calls.append((job.lo, job.hi, job.flags))
            if fail_after is not None and len(calls) > fail_after:
                raise KeyboardInterrupt("interrupted by the test")
        return oracle.enumerate_job(oracle.make_job(job.n, job.mode, job.rule, job.flags & ~warlib.F_MEMO_KEEP,
                                                    job.lo, job.hi, job.hbins, job.dbins, job.blk, job.sample_ppm,
                                                    job.seed))
    monkeypatch.setattr(warlib, "enumerate_job", enum)
    monkeypatch.setattr(warlib, "enumerate_plain", enum)
    monkeypatch.setattr(war_gpu, "_tune_for", lambda *a: None)


def main_lines(argv):
    import war_gpu
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        war_gpu.main(argv)
    return [TIME.sub("  Xs", ln) for ln in buf.getvalue().splitlines()]


def recorded(golden, name, nmax):
    out, keep = [], False
    for ln in golden["war_gpu_lines"][name]:
        if ln.startswith("n="):
            keep = int(ln.split()[0][2:]) <= nmax
        if keep:
            out.append(TIME.sub("  Xs", ln))
    return out


def test_deal_lines_match_the_recorded_output(monkeypatch, oracle, golden):
    """`war_gpu.py 11 --nmin 1 --hist 256` (data/checks.txt:5-24, n <= 11)."""
    fake_engine(monkeypatch, oracle)
    assert main_lines(["11", "--nmin", "1", "--hist", "256"]) == recorded(golden, "deals_hist256", 11)


def test_canonical_lines_match_the_recorded_output(monkeypatch, oracle, golden):
    """`war_gpu.py 10 --nmin 1 --canon --distinct --shape` (data/checks.txt:143-182, n <= 10)."""
    fake_engine(monkeypatch, oracle)
    assert main_lines(["10", "--nmin", "1", "--canon", "--distinct", "--shape"]) == \
        recorded(golden, "canon_distinct_shape", 10)


def test_interrupted_run_resumes_to_the_same_result(monkeypatch, oracle, tmp_path):
    import war_gpu
    monkeypatch.setattr(war_gpu, "SPAN_RANKS", 40000)
    full = None
    fake_engine(monkeypatch, oracle)
    kw = dict(hbins=64, per=16, batch_threads=256)      # spans of SPAN_RANKS deals
    full = war_gpu.run(9, quiet=True, **kw)

    calls = []
    fake_engine(monkeypatch, oracle, calls=calls, fail_after=3)
    out = str(tmp_path / "run9")
    with pytest.raises(KeyboardInterrupt):
        war_gpu.run(9, out=out, quiet=True, **kw)
    with open(out + ".progress") as f:
        st = json.load(f)
    assert st["n"] == 9 and 0 < st["next_start"] < 362880
    assert calls[0][2] & 16 == 0 and all(c[2] & 16 for c in calls[1:])   # WAR_F_MEMO_KEEP after the first span

    calls2 = []
    fake_engine(monkeypatch, oracle, calls=calls2)
    again = war_gpu.run(9, out=out, resume=True, quiet=True, **kw)
    assert calls2[0][0] == st["next_start"] and calls2[0][2] & 16 == 0   # a new process starts a new memo
    assert again[:3] == full[:3] and again[4] == full[4]
    with open(out + ".progress") as f:
        assert json.load(f)["next_start"] == 362880


def test_tune_override_fields(monkeypatch):
    import warlib
    import war_gpu
    t = war_gpu.override_tune(warlib.make_tune(threads=256, variant=31, memo_bits=30), {"memo_bits": 28})
    assert (t.threads, t.variant, t.memo_bits) == (256, 31, 28)
    with pytest.raises(ValueError):
        war_gpu.override_tune(None, {"no_such_field": 1})


TIME17 = re.compile(r"  [0-9.]+s  slowest launch [0-9.]+s")


def test_war17_lines_match_the_recorded_output(monkeypatch, oracle, golden):
    """`war17.py 11 --nmin 5` (data/checks.txt:81-91, n <= 11) with the oracle's gpu/war17.py restatement
    standing in for the held-out engine."""
    import warlib
    import war17

    def enum(job, tune=None):
        return oracle.enumerate_held(oracle.make_job(job.n, job.mode, job.rule, 0, job.lo, job.hi, job.hbins))
    monkeypatch.setattr(warlib, "enumerate_held", enum)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        war17.main(["11", "--nmin", "5"])
    got = [TIME17.sub("  X", ln) for ln in buf.getvalue().splitlines()]
    want = [TIME17.sub("  X", ln) for ln in golden["war_gpu_lines"]["war17_5_13"] if int(ln.split()[0][2:]) <= 11]
    assert got == want


def test_war17_resume(monkeypatch, oracle, tmp_path):
    import warlib
    import war17
    calls = []

    def enum(job, tune=None):
        calls.append(job.lo)
        if len(calls) == 3:
            raise KeyboardInterrupt("interrupted by the test")
        return oracle.enumerate_held(oracle.make_job(job.n, job.mode, job.rule, 0, job.lo, job.hi, job.hbins))
    monkeypatch.setattr(warlib, "enumerate_held", enum)
    monkeypatch.setattr(war17, "SPAN_RANKS", 50000)
    out = str(tmp_path / "n9")
    with pytest.raises(KeyboardInterrupt):
        war17.run(9, per=4, batch_threads=256, out=out)
    calls.append(None)   # no more interruptions
    r = war17.run(9, per=4, batch_threads=256, out=out, resume=True)
    assert r[:3] == (218680, 362880, 28)


def test_progress_file_schema_is_the_reference_one(monkeypatch, oracle, tmp_path):
    """The drop-in writes its progress file with exactly the keys of gpu/war_gpu.py:331-338, in the same order
    and with the same value types, as the reference's own files (tests/golden/progress_*_ref.json)."""
    import os
    import war_gpu
    fake_engine(monkeypatch, oracle)
    golden_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    for name, kw in (("progress_deals13_ref.json", dict(hbins=64)),
                     ("progress_canon13_ref.json", dict(canon=True, shape=True, dbins=4096))):
        with open(os.path.join(golden_dir, name)) as f:
            ref = json.load(f)
        out = str(tmp_path / name)
        war_gpu.run(8, out=out, quiet=True, **kw)
        with open(out + ".progress") as f:
            ours = json.load(f)
        assert list(ours) == list(ref)
        for k in ref:
            assert type(ours[k]) is type(ref[k]), k
        assert ours["next_start"] == ours["total"] and ours["n"] == 8


def test_war24_lines_and_checkpoint(monkeypatch, oracle, golden, tmp_path):
    """`war24.py n --det streak` for n = 5, 7, 9, 11 and `--det floyd` for n = 10 print the recorded lines
    (data/checks.txt:73-78) apart from the time, with the oracle's restatement of gpu/war24.py standing in for
    the engine; an interrupted run resumes from its checkpoint (pos, cyc, max, deals, und) to the same line."""
    import warlib
    import war24
    dets = {warlib.DET_BRENT: oracle.DET_BRENT, warlib.DET_FLOYD: oracle.DET_FLOYD, warlib.DET_STREAK: oracle.DET_STREAK}

    def enum(job, det=0, **kw):
        return oracle.war24(oracle.make_job(job.n, job.mode, job.rule, 0, job.lo, job.hi), dets[det])
    monkeypatch.setattr(warlib, "enumerate_wide", enum)
    tm = re.compile(r" time=[0-9.]+s")
    for e in [e for e in golden["war24"] if e["hi"] - e["lo"] <= 5 * 10 ** 7]:
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            war24.main([str(e["n"]), "--det", e["det"], "--dir", str(tmp_path)])
        assert tm.sub("", buf.getvalue().strip()) == tm.sub("", e["line"])
    # interrupted after two spans of 50,000 deals, then resumed
    monkeypatch.setattr(war24, "SPAN", 50000)
    monkeypatch.setattr(war24, "CKPT_EVERY_S", -1.0)             # a checkpoint after every span
    calls = []

    def enum_stop(job, det=0, **kw):
        calls.append(job.lo)
        if len(calls) == 3:
            raise KeyboardInterrupt("interrupted by the test")
        return enum(job, det)
    monkeypatch.setattr(warlib, "enumerate_wide", enum_stop)
    with pytest.raises(KeyboardInterrupt):
        war24.main(["9", "--dir", str(tmp_path), "--tag", "_t"])
    with open(tmp_path / "war24_n9_streak_0_362880_t.ckpt") as f:
        st = json.load(f)
    assert list(st) == ["pos", "cyc", "max", "deals", "und"] and st["pos"] == 100000 == st["deals"]
    calls.append(None)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        war24.main(["9", "--dir", str(tmp_path), "--tag", "_t", "--resume"])
    want = next(e for e in golden["war24"] if e["n"] == 9)
    assert tm.sub("", buf.getvalue().strip()) == tm.sub("", want["line"])
    assert calls[4] == 100000                                     # resumed at the checkpoint
