"""Template tables built on the GPU (gtls_template_cache) against the host
construction that follows the reference's transit.py:8-160 (template.get_cache
+ device_templates): the same widths and durations, overshoot and template
rows within 1e-12, for the reference's "default", "grazing" and "box"
templates and curves of several lengths; and a batched search with device
templates returns what it returns with host templates."""
import types

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _opts(**kw):
    from gtls_b200.validate import validate_args
    o = types.SimpleNamespace()
    validate_args(o, dict(use_threads=1, **kw))
    return o


@pytest.mark.parametrize("kind", ["default", "grazing", "box"])
def test_device_templates_equal_host_construction(cuda, kind):
    from gtls_b200 import synthetic
    from gtls_b200.batch import CurveSetOnDevice, prepare_curve
    opts = _opts(transit_template=kind)
    curves = [synthetic.small_curve(seed=3, n=1500, span=6.0),
              synthetic.light_curve_cfg1(seed=2, n=5000)[:3],
              synthetic.light_curve_cfg1(seed=4, n=19728)[:3]]
    host = [prepare_curve(*c, opts, templates="host") for c in curves]
    dev = [prepare_curve(*c, opts, templates="device") for c in curves]
    cs_h = CurveSetOnDevice(host)
    cs_d = CurveSetOnDevice(dev)
    for h, d in zip(host, dev):
        np.testing.assert_array_equal(h["widths"], d["widths"])
        np.testing.assert_array_equal(h["durations"], d["durations"])
        assert h["maxd"] == d["maxd"]
        np.testing.assert_allclose(d["overshoot"], h["overshoot"], rtol=1e-12)
    np.testing.assert_array_equal(cs_h.tables["widths"].cpu().numpy(), cs_d.tables["widths"].cpu().numpy())
    np.testing.assert_allclose(cs_d.tables["overshoot"].cpu().numpy(), cs_h.tables["overshoot"].cpu().numpy(),
                               rtol=1e-12)
    np.testing.assert_allclose(cs_d.tables["templates"].cpu().numpy(), cs_h.tables["templates"].cpu().numpy(),
                               rtol=0, atol=1e-12)


def test_batched_search_with_device_templates_equals_host_templates(cuda):
    from gtls_b200 import synthetic
    from gtls_b200.batch import gtls_batch
    curves = [synthetic.small_curve(seed=s, n=1500 + 300 * s, span=6.0) for s in range(3)]
    kw = dict(precision="fp64", autotune=False, use_threads=1)
    a = gtls_batch(curves).power(templates="device", **kw)
    b = gtls_batch(curves).power(templates="host", **kw)
    for ra, rb in zip(a, b):
        assert ra.period_index == rb.period_index and ra.width == rb.width and ra.loc == rb.loc
        np.testing.assert_allclose([ra.SDE, ra.depth, ra.T0], [rb.SDE, rb.depth, rb.T0], rtol=1e-9)
        np.testing.assert_allclose(np.ma.getdata(ra.chi2), np.ma.getdata(rb.chi2), rtol=1e-9)
