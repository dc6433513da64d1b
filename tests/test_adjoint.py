"""Gradient of the model chi2: torch autograd vs central finite differences
(CPU), and the CUDA forward/adjoint kernels vs both (GPU)."""
import numpy as np
import pytest
import torch

import adjoint_reference as AR
from gtls_b200 import synthetic


def fd_floor(t, params, chi2, rel=1e-6):
    """Per-parameter roundoff floor of a central difference: summation error of
    chi2 (~ eps * log2(n) * chi2) over the step h_k = rel * |param_k| (T0: offset
    from the first sample), with a factor 4 for the Richardson combination."""
    n = t.numel()
    out = np.empty(6)
    for k in range(6):
        scale = abs(float(params[k]) - float(t[0])) if k == 1 else abs(float(params[k]))
        out[k] = 4 * 2.2e-16 * np.log2(n) * chi2 / (rel * scale)
    return out


def _one(seed=0, n=4000):
    curves, truth, start, scales = synthetic.refinement_set(n_curves=1, n=n, seed=seed)
    t, y, dy = curves[0]
    return (torch.from_numpy(t), torch.from_numpy(y), torch.from_numpy(1 / dy ** 2),
            torch.from_numpy(start[0]), torch.from_numpy(truth[0]))


def test_reference_autograd_matches_finite_differences():
    t, y, w, p0, _ = _one()
    _, g = AR.autograd_grad(t, y, w, p0)
    # central differences at h = 1e-6 relative carry an O(h^2) truncation error
    # of up to ~2e-4 on the sharp transit edges; Richardson's combination of h
    # and h/2 removes it down to O(h^4) (~1e-6); the exact bar (1e-6) is the
    # comparison with torch autograd
    fd = AR.finite_difference_grad(t, y, w, p0, rel=1e-6)
    np.testing.assert_allclose(g.numpy(), fd.numpy(), rtol=1e-3)
    rich = AR.richardson_grad(t, y, w, p0, rel=1e-6)
    floor = fd_floor(t, p0, float(AR.chi2(t, y, w, p0)))
    assert np.all(np.abs(g.numpy() - rich.numpy()) <= 5e-6 * np.abs(g.numpy()) + floor)


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
        c_ref, g_ref = AR.autograd_grad(tc, yc, wc, torch.from_numpy(start[c]))
        fd = AR.finite_difference_grad(tc, yc, wc, torch.from_numpy(start[c]), rel=1e-6)
        rich = AR.richardson_grad(tc, yc, wc, torch.from_numpy(start[c]), rel=1e-6)
        assert abs(float(chi[c]) / float(c_ref) - 1) < 1e-12
        np.testing.assert_allclose(g[c].cpu().numpy(), g_ref.numpy(), rtol=1e-6)
        np.testing.assert_allclose(g[c].cpu().numpy(), fd.numpy(), rtol=1e-2)   # truncation-limited
        floor = fd_floor(tc, torch.from_numpy(start[c]), float(c_ref))
        gk = g[c].cpu().numpy()
        assert np.all(np.abs(gk - rich.numpy()) <= 5e-6 * np.abs(gk) + floor), (gk, rich.numpy(), floor)


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
    # the period moves toward the truth on average
    err0 = (p0[:, 0].cpu().numpy() - truth[:, 0]) / scales[:, 0]
    err1 = (out[:, 0].detach().cpu().numpy() - truth[:, 0]) / scales[:, 0]
    assert np.median(np.abs(err1)) < np.median(np.abs(err0))


def test_pack_curves_weights_equal_the_host_formula():
    """refine.pack_curves forms w = 1 / (dy * dy) where the tensors live (here
    on the CPU): bitwise the host NumPy values, with t, y and the offsets
    concatenated in curve order."""
    from gtls_b200 import refine
    rng = np.random.default_rng(2)
    curves = [(np.sort(rng.uniform(0, 10, n)), rng.normal(1, 1e-3, n), rng.uniform(1e-4, 3e-3, n))
              for n in (5, 17, 1000)]
    t, y, w, off = refine.pack_curves(curves, "cpu")
    dy = np.concatenate([c[2] for c in curves])
    np.testing.assert_array_equal(w.numpy(), 1.0 / (dy * dy))
    np.testing.assert_array_equal(t.numpy(), np.concatenate([c[0] for c in curves]))
    np.testing.assert_array_equal(y.numpy(), np.concatenate([c[1] for c in curves]))
    np.testing.assert_array_equal(off.numpy(), [0, 5, 22, 1022])
