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
    for cap, shift, glob in [(0, 0, 0), (256, 0, 0), (1024, -1, 0), (4096, -2, 0), (24576, -3, 0), (65536, 0, 0),
                             (0, 0, 1), (256, -1, 1), (8192, 0, 1)]:
        _lib.set_tuning(tile_cap_fp32=cap, tile_cap_fp64=cap, bucket_shift=shift, records_global=glob)
        for pass_ in (_lib.GTLS_PASS_MAIN, _lib.GTLS_PASS_ALL):
            c, l = cur.search(P[::3] if pass_ == _lib.GTLS_PASS_ALL else P, 1e-5, 8, 7, pass_, precision,
                              want_loc=True)
            out.append((cap, shift, glob, pass_, c.cpu().numpy(), l.cpu().numpy()))
    for cap, shift, glob, pass_, c, l in out[2:]:
        ref = out[0] if pass_ == _lib.GTLS_PASS_MAIN else out[1]
        msg = "cap %d shift %d global %d" % (cap, shift, glob)
        np.testing.assert_array_equal(c, ref[4], err_msg=msg)
        np.testing.assert_array_equal(l, ref[5], err_msg=msg)


def test_tuning_rejects_bad_values(cuda, restore_tuning):
    from gtls_b200 import _lib
    for bad in (dict(tile_cap_fp32=100), dict(tile_cap_fp64=70000), dict(bucket_shift=1), dict(bucket_shift=-4),
                dict(records_global=2)):
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


def test_long_durations_read_records_from_global_memory(cuda):
    """A curve whose longest duration (14,400 samples) leaves no room for an
    FP64 shared-memory tile: the chi2 kernel reads the records from global
    memory, and the FP64 search still matches the oracle."""
    import tls_oracle as O
    from gtls_b200 import _lib
    from gtls_b200.core import CurveOnDevice
    s = search_inputs(seed=37, n=120000, span=30.0, step=1.3)
    assert s["maxd"] * 16 > 227 * 1024 - 4096
    cur = CurveOnDevice(s["t"], s["y"], s["dy"], s["lc"], s["ov"])
    P = s["periods"][::150]
    c, l = cur.search(P, 1e-5, 8, 3, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
    c_ref, l_ref = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                                    s["overshoot"], s["maxd"], 1e-5, 8, 3)
    np.testing.assert_allclose(c.cpu().numpy(), c_ref, rtol=1e-9)
    np.testing.assert_array_equal(l.cpu().numpy(), l_ref)
