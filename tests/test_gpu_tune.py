"""Launch-shape tuning changes the time of a search, never its result."""
import numpy as np
import pytest

from conftest import search_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture
def restore_tuning(cuda):
    from gtls_b200 import _lib
    yield
    _lib.set_tuning()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_results_identical_for_every_tuning(cuda, restore_tuning, precision):
    from gtls_b200 import _lib
    from gtls_b200.core import CurveOnDevice
    s = search_inputs(seed=31, n=3000, span=9.0, use_dy=True)
    cur = CurveOnDevice(s["t"], s["y"], s["dy"], s["lc"], s["ov"])
    P = s["periods"][::4]
    out = []
    for cap, shift in [(0, 0), (256, 0), (1024, -1), (4096, -2), (24576, -3), (65536, 0)]:
        _lib.set_tuning(tile_cap_fp32=cap, tile_cap_fp64=cap, bucket_shift=shift)
        for pass_ in (_lib.GTLS_PASS_MAIN, _lib.GTLS_PASS_ALL):
            c, l = cur.search(P[::3] if pass_ == _lib.GTLS_PASS_ALL else P, 1e-5, 8, 7, pass_, precision,
                              want_loc=True)
            out.append((cap, shift, pass_, c.cpu().numpy(), l.cpu().numpy()))
    for cap, shift, pass_, c, l in out[2:]:
        ref = out[0] if pass_ == _lib.GTLS_PASS_MAIN else out[1]
        np.testing.assert_array_equal(c, ref[3], err_msg="cap %d shift %d" % (cap, shift))
        np.testing.assert_array_equal(l, ref[4], err_msg="cap %d shift %d" % (cap, shift))


def test_tuning_rejects_bad_values(cuda, restore_tuning):
    from gtls_b200 import _lib
    for bad in (dict(tile_cap_fp32=100), dict(tile_cap_fp64=70000), dict(bucket_shift=1), dict(bucket_shift=-4)):
        with pytest.raises(_lib.GtlsError):
            _lib.set_tuning(**bad)
    _lib.set_tuning(tile_cap_fp32=512)
    assert _lib.get_tuning()["tile_cap_fp32"] == 512


def test_autotune_picks_a_candidate(cuda, restore_tuning):
    from gtls_b200 import _lib, tune
    from gtls_b200.batch import CurveSetOnDevice
    s = search_inputs(seed=32, n=2500, span=8.0)
    prep = [dict(t=s["t"], y=s["y"], dy=s["dy"], periods=s["periods"],
                 span=float(np.float32(s["t"].max() - s["t"].min())), widths=s["widths"], overshoot=s["overshoot"],
                 durations=s["dur_u"], tmpl=s["templates"], maxd=int(s["maxd"]))]
    cs = CurveSetOnDevice(prep)
    tune._CACHE.clear()
    best = tune.tune_curve_set(cs, "fp32", n_sample=64)
    assert best["tile_cap_fp32"] in tune.TILE_CAPS["fp32"] and best["bucket_shift"] in tune.BUCKET_SHIFTS
    assert _lib.get_tuning() == best
