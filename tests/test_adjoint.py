"""Gradient of the limb-darkened model chi2: torch autograd vs central finite
differences (CPU), and the CUDA forward/adjoint kernels vs both (GPU); the
refinement of search peaks (GPU).

Bars.  Forward: the kernel's chi2 within 1e-12 relative of the torch model,
which equals gtls_b200.ldmodel (the template generator) to 1e-14.  Gradient:
torch autograd of the same discrete model within 1e-6 relative (the exact
check).  Central differences at h = 1e-6 relative: within 1e-6 relative plus
a roundoff floor for D, depth, u1 and u2.  P and T0 are stiff (a step in P
moves transit n by n*h, so chi2 varies on the scale of the ingress divided
by the number of transits): at h = 1e-6 relative the h^2 truncation error of
the central difference reaches 7% (P) and 1% (T0) on these curves, shrinking
100-fold per 10-fold smaller step, so they are checked at h = 1e-8 relative,
where truncation is below 1e-5, within 1e-5 relative plus the floor.
"""
import numpy as np
import pytest
import torch

import adjoint_reference as AR
from gtls_b200 import synthetic

RTOL_AUTOGRAD = 1e-6
STIFF = (0, 1)          # P, T0
H_SMOOTH, H_STIFF = 1e-6, 1e-8


def fd_floor(t, params, chi2, k, rel):
    """Roundoff floor of a central difference of chi2 for parameter k: the
    summation error of chi2 (~ eps * log2(n) * chi2, times 4 for safety) over
    the step."""
    return 4 * 2.2e-16 * np.log2(t.numel()) * chi2 / AR.fd_step(t, params, k, rel)


def check_against_fd(g, t, y, w, p, chi2):
    """g (6,) numpy gradient against central differences per the bars above."""
    fd_s = AR.finite_difference_grad(t, y, w, p, rel=H_SMOOTH).numpy()
    fd_t = AR.finite_difference_grad(t, y, w, p, rel=H_STIFF).numpy()
    for k in range(6):
        stiff = k in STIFF
        fd = fd_t[k] if stiff else fd_s[k]
        tol = (1e-5 if stiff else 1e-6) * abs(g[k]) + fd_floor(t, p, chi2, k, H_STIFF if stiff else H_SMOOTH)
        assert abs(g[k] - fd) <= tol, (k, g[k], fd, tol)


def _one(seed=0, n=20000, c=0):
    curves, truth, start, scales = synthetic.refinement_set(n_curves=c + 1, n=n, seed=seed)
    t, y, dy = curves[c]
    return (torch.from_numpy(t), torch.from_numpy(y), torch.from_numpy(1 / dy ** 2),
            torch.from_numpy(start[c]), torch.from_numpy(truth[c]))


def test_reference_model_is_the_template_model():
    """The differentiated model equals the light curves the synthetic sets
    inject (gtls_b200.ldmodel, the template generator's occultation)."""
    curves, truth, start, scales = synthetic.refinement_set(n_curves=3, n=20000, seed=1)
    for c in range(3):
        t = curves[c][0]
        P, T0, D, depth, u1, u2 = truth[c]
        ref = synthetic._transit(t, T0, P, depth, D, [u1, u2])
        m = AR.model(torch.from_numpy(t), torch.from_numpy(truth[c])).numpy()
        np.testing.assert_allclose(m, ref, rtol=0, atol=1e-14)
        assert 1 - ref.min() > 0.5 * depth


@pytest.mark.parametrize("c", [0, 3, 7])
def test_reference_autograd_matches_finite_differences(c):
    t, y, w, p0, _ = _one(seed=1, c=c)
    chi, g = AR.autograd_grad(t, y, w, p0)
    check_against_fd(g.numpy(), t, y, w, p0, float(chi))


@pytest.mark.gpu
def test_kernel_gradient_matches_autograd_and_finite_differences(cuda):
    from gtls_b200 import _lib, refine
    curves, truth, start, scales = synthetic.refinement_set(n_curves=16, n=20000, seed=1)
    t, y, w, off = refine.pack_curves(curves, "cuda")
    p = torch.from_numpy(start).cuda()
    chi = _lib.model_chi2(t, y, w, off, p)
    g = _lib.model_chi2_grad(t, y, w, off, p, torch.ones(16, dtype=torch.float64, device="cuda"))
    for c in range(16):
        tc, yc, dyc = (torch.from_numpy(a) for a in curves[c])
        wc = 1 / dyc ** 2
        pc = torch.from_numpy(start[c])
        c_ref, g_ref = AR.autograd_grad(tc, yc, wc, pc)
        assert abs(float(chi[c]) / float(c_ref) - 1) < 1e-12
        gk = g[c].cpu().numpy()
        np.testing.assert_allclose(gk, g_ref.numpy(), rtol=RTOL_AUTOGRAD)
        if c < 4:
            check_against_fd(gk, tc, yc, wc, pc, float(c_ref))


@pytest.mark.gpu
def test_autograd_function_and_refinement(cuda):
    from gtls_b200 import refine
    # deep transits with little noise: the period is fixed far below a grid step
    curves, truth, start, scales = synthetic.refinement_set(n_curves=64, n=20000, seed=2, noise=1e-4,
                                                            depth_range=(2000e-6, 5000e-6))
    t, y, w, off = refine.pack_curves(curves, "cuda")
    p0 = torch.from_numpy(start).cuda()
    sc = torch.from_numpy(scales).cuda()
    F = refine.model_chi2_function()
    p = p0.clone().requires_grad_(True)
    F.apply(p, t, y, w, off).sum().backward()
    assert torch.all(torch.isfinite(p.grad))
    out, chi, better = refine.refine(p0, sc, t, y, w, off, steps=50)
    chi0 = F.apply(p0, t, y, w, off)
    assert torch.all(chi <= chi0)
    assert better.float().mean() > 0.9
    # the period and the epoch move toward the truth
    for k in (0, 1):
        err0 = (p0[:, k].cpu().numpy() - truth[:, k]) / scales[:, k]
        err1 = (out[:, k].detach().cpu().numpy() - truth[:, k]) / scales[:, k]
        assert np.median(np.abs(err1)) < 0.5 * np.median(np.abs(err0)), k


@pytest.mark.gpu
def test_power_refine_moves_the_peak_below_grid_resolution(cuda):
    """gtls(...).power(refine=True): the refined period and T0 are closer to
    the injected ones than the grid's, the model chi2 decreased, and the grid
    result stays available; gtls_batch(...).power(refine=True) refines every
    curve in one batched run and agrees with the single-curve refinement."""
    from gtls_b200 import gtls
    from gtls_b200.batch import gtls_batch
    t, y, _, truth = synthetic.light_curve_cfg1(seed=5, n=12000, period=2.71, depth=3000e-6, noise=5e-4)
    res = gtls(t, y, verbose=False).power(period_min=0.5, period_max=10.0, refine=True)
    ref = res.diagnostics["refinement"]
    assert ref["improved"] and ref["chi2"] < ref["chi2_grid"]
    g = ref["grid"]
    assert abs(res.period - truth["period"]) < abs(g["period"] - truth["period"])
    t0_true = truth["t0"] + np.round((res.T0 - truth["t0"]) / truth["period"]) * truth["period"]
    assert abs(res.T0 - t0_true) < 2e-3
    assert res.period == ref["params"][0] and res.T0 == ref["params"][1]
    out = gtls_batch([(t, y)]).power(period_min=0.5, period_max=10.0, refine=True, precision="fp64",
                                     autotune=False)
    np.testing.assert_allclose(out[0].period, res.period, rtol=1e-9)
    assert out[0].refinement["improved"]
