"""End-to-end gtls(t, y, dy).power() against the oracle's full host flow."""
import numpy as np
import pytest

import tls_oracle as O
from conftest import search_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("use_dy", [False, True])
def test_power_matches_oracle(cuda, use_dy):
    from gtls_b200 import gtls
    s = search_inputs(seed=21, n=1500, span=6.0, use_dy=use_dy)
    P = s["periods"]
    batch = 12
    ref = O.search(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"], s["overshoot"],
                   s["dur_u"], s["maxd"], 1e-5, 0.125, 3, batch=batch)
    model = gtls(s["t"], s["y"], s["dy"] if use_dy else None, verbose=False)
    res = model.power(periods=P, batch_periods=batch, oversampling_factor=3)
    assert res.diagnostics["period_index"] == ref["period_index"]
    assert res.period == ref["period"]
    assert res.durationPoints == ref["width"]
    assert res.diagnostics["loc"] == ref["loc"]
    np.testing.assert_allclose(res.raw_chi2, ref["raw_chi2"], rtol=1e-9)
    np.testing.assert_allclose(np.ma.getdata(res.chi2), np.ma.getdata(ref["chi2"]), rtol=1e-9)
    assert list(res.possiblePeriodsIndices) == list(ref["candidates"])
    np.testing.assert_allclose([res.SDE, res.depth, res.T0, res.duration],
                               [ref["SDE"], ref["depth"], ref["T0"], ref["duration"]], rtol=1e-9)
    assert abs(res.period - 1.7) < 0.02


def test_power_fast_and_fp32(cuda):
    from gtls_b200 import gtls
    s = search_inputs(seed=22, n=1500, span=6.0)
    model = gtls(s["t"], s["y"], verbose=False)
    periods, power = model.power(periods=s["periods"], batch_periods=12, fast=True)
    assert len(periods) == len(power) == len(s["periods"])
    r64 = model.power(periods=s["periods"], batch_periods=12)
    r32 = model.power(periods=s["periods"], batch_periods=12, precision="fp32")
    assert r32.period == r64.period
    assert abs(r32.SDE / r64.SDE - 1) < 1e-4


def test_power_default_grid(cuda):
    """Default Ofir grid from the device and the reference's batch-size formula."""
    from gtls_b200 import gtls, synthetic
    t, y, _, truth = synthetic.light_curve_cfg1(seed=3, n=6000, period=2.2, depth=2000e-6)
    res = gtls(t, y, verbose=False).power()
    assert abs(res.period / truth["period"] - 1) < 2e-3
    assert res.SDE > 7
