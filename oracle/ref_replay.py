"""Replay of the reference's kernels, compiled for the CPU -- TEST INFRASTRUCTURE ONLY.

``oracle/Makefile`` compiles the reference's kernel source
(``src/gputls/GPUFun.cu``) with g++ into ``oracle/_ref/libgpufun_ref_*.so``.
This module launches those kernels in the order the reference's host code
launches them, per period:

* main pass: core.py:770-875 (foldFast, argsort, patchData,
  calcInverseSquaredPatchedDy, calcEdgeEffectCorrections, cumsum,
  calculate_base_error, cumsum, calcAllFullSum_v2, calculate_final_ootr_v3,
  calcAllLowestResidualsGPUB_SignalTiled_v2, argmin);
* candidate / single-period passes: core.py:1159-1237 and 1314-1418
  (calcAllFullSum, step1, cumsum, step2, ...NoSkipTemp or ...NoSkip).

cupy's argsort/cumsum/argmin are played by NumPy (stable argsort, sequential
cumsum, first-occurrence argmin).  ``r32`` uses the dtypes of the reference's
type-consistent caller ``_worker.py:100-147`` (FP64 time and periods, FP32
flux, weights and sums, int32 indices); ``r64`` promotes every float to
double.  The backend has the same interface as ``tls_oracle.NumpyBackend``
so ``tls_oracle.search`` can drive either.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def available(variant="r64_skip8"):
    return os.path.exists(os.path.join(REF_DIR, "libgpufun_ref_%s.so" % variant))


def _grid(size):
    """calcGridBlockSize (core.py:26-32)."""
    block = min(size, 128)
    return block, int((size / block) + 1)


class RefKernelBackend:
    """Per-period passes through the reference's own kernels on the CPU."""

    def __init__(self, precision="r64", skip_point=8):
        tag = "skip8" if skip_point == 8 else ("skipnever" if skip_point == 0x7F800000 else None)
        if tag is None:
            raise ValueError("reference kernels are built for SKIP_POINT 8 and 0x7f800000 only")
        self.name = "refkernels-%s-%s" % (precision, tag)
        self.skip_point = skip_point
        self.real = np.float64 if precision == "r64" else np.float32
        path = os.path.join(REF_DIR, "libgpufun_ref_%s_%s.so" % (precision, tag))
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run `make -C oracle`)")
        self.lib = ctypes.CDLL(path)

    # -- helpers ------------------------------------------------------------
    @staticmethod
    def _p(a):
        return a.ctypes.data_as(ctypes.c_void_p)

    def _i(self, v):
        return np.array([v], dtype=np.int32)

    def _launch(self, name, grid, block, *args):
        fn = getattr(self.lib, name)
        c_args = [ctypes.c_int(g) for g in grid] + [ctypes.c_int(b) for b in block]
        for a in args:
            c_args.append(self._p(a) if isinstance(a, np.ndarray) else ctypes.c_int(int(a)))
        fn(*c_args)

    def _prepare(self, t, y, dy, period, widths, tmpl, overshoot, maxd):
        R = self.real
        n = len(t)
        m = n + maxd
        tt = np.ascontiguousarray(t, dtype=np.float64)
        pp = np.array([period], dtype=np.float64)
        phase = np.empty(n, dtype=np.float64)
        b, g = _grid(n)
        self._launch("ref_foldFast", (g, 1, 1), (b, 1, 1), tt, pp, phase, self._i(1), self._i(n))
        order = np.argsort(phase, kind="stable").astype(np.int32)
        pd = np.empty(m, dtype=R)
        pdy = np.empty(m, dtype=R)
        b, g = _grid(m)
        self._launch("ref_patchData", (g, 1, 1), (b, 1, 1), pd, pdy, self._i(m), order, self._i(maxd),
                     np.ascontiguousarray(y, dtype=R), np.ascontiguousarray(dy, dtype=R), self._i(n))
        inv = np.empty(m, dtype=R)
        self._launch("ref_calcInverseSquaredPatchedDy", (g, 1, 1), (b, 1, 1), inv, pdy, self._i(m))
        edge = np.empty(1, dtype=R)
        self._launch("ref_calcEdgeEffectCorrections", (2, 1, 1), (1, 1, 1), edge, pd, inv, self._i(m),
                     self._i(maxd), self._i(1))
        cs = np.cumsum(pd).astype(R)
        dur = np.ascontiguousarray(widths, dtype=np.int32)
        D = len(dur)
        maxlen = int(np.max(dur))
        sig = np.ascontiguousarray(tmpl[:, :maxlen], dtype=R)
        os_ = np.ascontiguousarray(overshoot, dtype=R)
        return dict(n=n, m=m, pd=pd, inv=inv, edge=edge, cs=cs, dur=dur, D=D, maxlen=maxlen, sig=sig,
                    os=os_)

    def duration_ranges(self, periods, span, n_samples):
        """durationsGrid (GPUFun.py:47-86) with a float32 time span (_worker.py:107)."""
        P = np.ascontiguousarray(periods, dtype=np.float64)
        wmax = np.empty(len(P), dtype=np.int32)
        wmin = np.empty(len(P), dtype=np.int32)
        b, g = _grid(len(P))
        length = np.array([np.float32(span)], dtype=self.real)
        self._launch("ref_durationsGrid", (g, 1, 1), (b, 1, 1), P, wmax, wmin, length, self._i(n_samples),
                     self._i(len(P)))
        return wmin.astype(np.int64), wmax.astype(np.int64)

    # -- passes -------------------------------------------------------------
    def main_pass(self, t, y, dy, period, widths, tmpl, overshoot, maxd, depth_min, skip_point):
        if skip_point != self.skip_point:
            raise ValueError("backend built for SKIP_POINT %d" % self.skip_point)
        R = self.real
        s = self._prepare(t, y, dy, period, widths, tmpl, overshoot, maxd)
        n, m, D = s["n"], s["m"], s["D"]
        base = np.empty(m, dtype=R)
        self._launch("ref_calculate_base_error", ((m + 255) // 256, 1, 1), (256, 1, 1), base, s["pd"],
                     s["inv"], m, 1)
        eps = np.cumsum(base).astype(R)
        fs = np.empty(D, dtype=R)
        b, g = _grid(D)
        self._launch("ref_calcAllFullSum_v2", (g, 1, 1), (b, 1, 1), fs, eps, m, s["dur"], D, 1)
        ootr = np.empty(D * n, dtype=R)
        self._launch("ref_calculate_final_ootr_v3", ((n + 255) // 256, D, 1), (256, 1, 1), ootr, eps, fs,
                     s["dur"], n, m, D, 1)
        out = np.empty(D * n, dtype=R)
        b, g = _grid(n)
        self._launch("ref_lowest_v2", (g, D, 1), (b, 1, 1), out, self._i(n), s["pd"], self._i(m), s["dur"],
                     self._i(D), s["sig"], self._i(s["maxlen"]), s["inv"], s["os"], ootr, fs, s["edge"],
                     self._i(len(y)), s["cs"], np.array([depth_min], dtype=R))
        loc = int(np.argmin(out))
        return float(out[loc]), loc

    def noskip_pass(self, t, y, dy, period, widths, tmpl, overshoot, maxd, depth_min, single=False):
        R = self.real
        s = self._prepare(t, y, dy, period, widths, tmpl, overshoot, maxd)
        n, m, D = s["n"], s["m"], s["D"]
        fs = np.empty(D, dtype=R)
        b, g = _grid(D)
        self._launch("ref_calcAllFullSum", (g, 1, 1), (b, 1, 1), fs, s["pd"], s["inv"], self._i(m), s["dur"],
                     self._i(D), self._i(1))
        tmp = np.empty(D * n, dtype=R)
        b, g = _grid(n)
        self._launch("ref_step1", (g, D, 1), (b, 1, 1), tmp, s["pd"], s["dur"], self._i(D), s["inv"],
                     self._i(m), self._i(n))
        ootr = np.cumsum(tmp.reshape(D, n), axis=-1).astype(R).ravel()
        self._launch("ref_step2", (g, D, 1), (b, 1, 1), ootr, self._i(D), self._i(m), s["dur"], self._i(n), fs)
        out = np.empty(D * n, dtype=R)
        common = (out, self._i(n), s["pd"], self._i(m), s["dur"], self._i(D), s["sig"], self._i(s["maxlen"]),
                  s["inv"], s["os"], ootr, fs, s["edge"], self._i(len(y)), s["cs"])
        if single:
            # durationsMax/Min are read per duration index but not used in the arithmetic
            zeros = np.zeros(D, dtype=np.int32)
            self._launch("ref_lowest_noskip", (g, D, 1), (b, 1, 1), *common, zeros, zeros,
                         np.array([depth_min], dtype=R))
        else:
            self._launch("ref_lowest_noskip_temp", (g, D, 1), (b, 1, 1), *common,
                         np.array([depth_min], dtype=R))
        loc = int(np.argmin(out))
        return float(out[loc]), loc
