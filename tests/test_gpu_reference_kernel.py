"""The reference's own GPU kernels (gpu/war_gpu.py, compiled unmodified into oracle/_ref/libwarref.so) and
this repository's kernels give identical results on the same GPU."""
import os
import sys

import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import ref_gpu  # noqa: E402


@pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libwarref.so not built (needs the reference)")
@pytest.mark.parametrize("n,canon,rule", [(9, 0, 0), (10, 0, 1), (11, 0, 0), (12, 0, 0), (9, 1, 0), (10, 1, 1), (11, 1, 0)])
def test_same_results_as_reference_kernel(wl, n, canon, rule):
    ref = ref_gpu.run(n, canon=bool(canon), rule=rule, hbins=256, dbins=4096 if canon else 0, shape=bool(canon) and rule == 0)
    flags = (wl.F_DISTINCT | (wl.F_SHAPE if rule == 0 else 0)) if canon else 0
    job = wl.make_job(n, wl.CANON if canon else wl.DEALS, rule, flags, hbins=256, dbins=4096 if canon else 0)
    for r in (wl.enumerate_job(job), wl.enumerate_plain(job)):
        d = wl.to_dict(r)
        assert (d["cyc"], d["done"], d["maxfin"], d["hist"]) == (ref["cyc"], ref["done"], ref["maxfin"], ref["hist"])
        if canon:
            assert d["dhist"] == ref["dhist"]
            if ref["blk"]:
                assert [d["shape_nonstd"], d["shape_unchecked"]] == ref["shape"]


@pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libwarref.so not built (needs the reference)")
def test_half_matches_reference_kernel(wl):
    ref = ref_gpu.run(10, half=True, hbins=128)
    r = wl.to_dict(wl.enumerate_job(wl.make_job(10, flags=wl.F_HALF, hbins=128)))
    assert (r["cyc"], r["done"], r["maxfin"], r["hist"]) == (ref["cyc"], ref["done"], ref["maxfin"], ref["hist"])
