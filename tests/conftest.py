import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libgtls_b200.so")


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gtls_b200 import _lib
    _lib.load()
    return torch


def search_inputs(seed=1, n=1200, span=6.0, use_dy=False, step=1.1):
    """Small seeded curve with its grid and template tables (host arrays)."""
    from gtls_b200 import synthetic, template, grid as G, validate as V
    import tls_oracle as O
    t, y, dy = synthetic.small_curve(seed=seed, n=n, span=span, dy=use_dy)
    t, y, dy = V.validate_inputs(t, y, dy)
    P = np.sort(O.period_grid(1, 1, t.max() - t.min()))
    durs = G.duration_grid(P, shortest=1 / len(t), log_step=step)
    mw = int(np.max(durs) * len(y))
    mw += mw % 2
    ov, lc = template.get_cache(durs, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    widths, os_, dd, tm, maxd = template.device_templates(lc, ov)
    return dict(t=t, y=y, dy=dy, periods=P, durations=durs, widths=widths, overshoot=os_, dur_u=dd,
                templates=tm, maxd=maxd, ov=ov, lc=lc)
