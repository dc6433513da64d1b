"""Torch-autograd and finite-difference references of the model chi2 -- TEST INFRASTRUCTURE ONLY.

The same model as the C-ABI's gtls_model_chi2 (defined in include/gtls_b200.h):
the quadratic limb-darkened occultation of a central (b = 0) circular-orbit
transit, evaluated with the quadrature of gtls_b200.ldmodel (96-node
Gauss-Legendre after the substitution r = m + h sin(theta)), written with
torch operations in float64 so that torch.autograd provides an independent
gradient of the same discrete formula, plus central finite differences.  Used
only by tests and the bench's checks.
"""
import numpy as np
import torch

GL_N = 96
_X, _W = np.polynomial.legendre.leggauss(GL_N)


def _moments(lo, hi, kind, z, p):
    """Quadrature of the three limb-darkening moments over r in [lo, hi]:
    int 2 pi r om^k dr ("inner") or int 2 r acos(c) om^k dr ("partial"),
    k = 0, 1, 2, om = 1 - sqrt(1 - r^2).  lo, hi, z: (m,) tensors."""
    theta = torch.as_tensor(0.5 * np.pi * _X, dtype=lo.dtype, device=lo.device)
    wts = torch.as_tensor(_W, dtype=lo.dtype, device=lo.device)
    mid = 0.5 * (lo + hi)
    half = 0.5 * (hi - lo)
    r = mid[:, None] + half[:, None] * torch.sin(theta)[None, :]
    jac = half[:, None] * torch.cos(theta)[None, :] * (0.5 * np.pi) * wts[None, :]
    one_r2 = 1.0 - r * r
    mu = torch.sqrt(torch.where(one_r2 > 0, one_r2, torch.ones_like(one_r2))) * (one_r2 > 0)
    om = 1.0 - mu
    if kind == "inner":
        f = 2.0 * np.pi * r
    else:
        zz = torch.clamp(z, min=1e-300)[:, None]
        c = (r * r + zz * zz - p * p) / (2.0 * r * zz)
        inside = (c > -1.0) & (c < 1.0)
        cc = torch.where(inside, c, torch.zeros_like(c))
        ac = torch.where(inside, torch.acos(cc), torch.where(c >= 1.0, torch.zeros_like(c), torch.full_like(c, np.pi)))
        f = 2.0 * r * ac
    return [torch.sum(f * om ** k * jac, dim=1) for k in range(3)]


def occulted_fraction(z, p, u1, u2):
    """gtls_b200.ldmodel.occulted_fraction as a differentiable torch function."""
    K = 1.0 - u1 / 3.0 - u2 / 6.0
    out = torch.zeros_like(z)
    hit = z < 1.0 + p
    if not bool(torch.any(hit)):
        return out
    zz = z[hit]
    inner = torch.clamp(p - zz, 0.0, 1.0)
    lo = torch.abs(zz - p)
    hi = torch.minimum(torch.ones_like(zz), zz + p)
    hi = torch.where(hi > lo, hi, lo)   # empty partial range: no contribution
    mi = _moments(torch.zeros_like(inner), inner, "inner", zz, p)
    mp = _moments(lo, hi, "partial", zz, p)
    N = (mi[0] + mp[0]) - u1 * (mi[1] + mp[1]) - u2 * (mi[2] + mp[2])
    return out.index_put((hit,), N / (np.pi * K))


def model(t, params):
    """t: (n,) float64 tensor; params: (6,) float64 tensor (P, T0, D, depth, u1, u2)
    -> model flux (n,)."""
    P, T0, D, depth, u1, u2 = params
    K = 1.0 - u1 / 3.0 - u2 / 6.0
    p = torch.sqrt(depth * K)
    a = (1.0 + p) / torch.sin(np.pi * D / P)
    x = t - T0
    q = x / P
    phi = 2.0 * np.pi * (q - torch.round(q.detach()))
    z = a * torch.abs(torch.sin(phi))
    behind = torch.cos(phi) < 0
    z = torch.where(behind, torch.full_like(z, 1e3) + a, z)
    return 1.0 - occulted_fraction(z, p, u1, u2)


def chi2(t, y, w, params):
    r = y - model(t, params)
    return torch.sum(w * r * r)


def autograd_grad(t, y, w, params):
    p = params.clone().detach().requires_grad_(True)
    c = chi2(t, y, w, p)
    (g,) = torch.autograd.grad(c, p)
    return c.detach(), g


def fd_step(t, params, k, rel):
    """Step of the central difference of parameter k: rel * |param| (T0: its
    offset from the first sample, so that the step is relative to the epoch
    within the data rather than to an absolute time stamp)."""
    scale = abs(float(params[k]) - float(t[0])) if k == 1 else abs(float(params[k]))
    return rel * max(scale, 1e-12)


def finite_difference_grad(t, y, w, params, rel=1e-6):
    """Central differences with step fd_step."""
    g = torch.empty_like(params)
    for k in range(params.numel()):
        h = fd_step(t, params, k, rel)
        pp = params.clone()
        pm = params.clone()
        pp[k] += h
        pm[k] -= h
        g[k] = (chi2(t, y, w, pp) - chi2(t, y, w, pm)) / (2 * h)
    return g


def richardson_grad(t, y, w, params, rel=1e-6):
    """Central differences at steps h and h/2 combined as (4 D(h/2) - D(h)) / 3,
    which cancels the h^2 truncation term."""
    d1 = finite_difference_grad(t, y, w, params, rel)
    d2 = finite_difference_grad(t, y, w, params, rel / 2)
    return (4 * d2 - d1) / 3
