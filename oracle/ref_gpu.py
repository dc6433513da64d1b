"""The reference's kernels on the GPU -- BASELINE INFRASTRUCTURE ONLY.

``oracle/Makefile`` compiles the reference's kernel source
(``src/gputls/GPUFun.cu``, read where it lies) for sm_100a into
``oracle/_ref/libgpufun_ref_sm100.so``.  This module replays the main pass of
the reference's type-consistent caller, ``_worker.py:53-311``, launch by
launch: durationsGrid and durationBool over the whole grid; then per batch of
S periods the union of the batch's duration masks (one logical_or per period,
_worker.py:196-200), foldFast, the argsort of the phases in ten row chunks
(:224-226), patchData, calcInverseSquaredPatchedDy,
calcEdgeEffectCorrections, one cumsum per period row (:249-250),
calculate_base_error, the cumsum of the errors, calcAllFullSum_v2,
calculate_final_ootr_v3, calcAllLowestResidualsGPUB_SignalTiled_v2 and the
per-period argmin (:293-301).  cupy's array operations are played by torch on
the same stream; the dtypes are _worker.py's (FP64 times, periods and
phases; int32 sizes and indices; FP32 flux, weights and sums).  It is the
"reference kernels on the same B200" baseline of bench.py; nothing in the
product imports it.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libgpufun_ref_sm100.so")


def available():
    return os.path.exists(LIB)


def _grid(size):
    """calcGridBlockSize (_worker.py:17-23)."""
    block = min(size, 128)
    return block, int((size / block) + 1)


def reference_batch_size(total_periods, patched_size, n_durations, free_bytes):
    """singleCalcPeriods of _worker.py:73-88."""
    cap = free_bytes / (5 * (patched_size * 2 + 2 + n_durations * patched_size * 4 + 2 * n_durations))
    base = max(1, int(total_periods / 30))
    s = int(np.min([np.floor(cap), base]))
    if s < 15:
        s = int(s / 1.1)
    return max(1, s)


class RefGpuMainPass:
    """Main pass of the reference (``_worker.py``) on one light curve.

    ``lc_arr``/``lc_cache_overview`` are the template cache of ``get_cache``
    (transit.py:98-160 layout)."""

    def __init__(self, t, y, dy, lc_arr, lc_cache_overview, transit_depth_min=1e-5, device=0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda:%d" % device)
        self.lib = ctypes.CDLL(LIB)
        durations, indices = np.unique(lc_cache_overview["width_in_samples"], return_index=True)
        self.lc_arr = lc_arr[indices]
        self.overview = lc_cache_overview[indices]
        max_d = int(max(durations))
        if max_d % 2 != 0:
            max_d += 1
        self.durations = np.sort(durations)
        self.max_d = max_d
        self.n = len(t)
        self.m = self.n + max_d
        T = torch
        self.t = T.tensor(np.asarray(t, dtype=np.float64), device=self.dev)
        self.y = T.tensor(np.asarray(y, dtype=np.float32), device=self.dev)
        self.dy = T.tensor(np.asarray(dy, dtype=np.float32), device=self.dev)
        self.span = float(np.float32(np.max(t) - np.min(t)))
        self.depth_min = transit_depth_min

    def _i32(self, v):
        return self.torch.tensor([int(v)], dtype=self.torch.int32, device=self.dev)

    def _call(self, name, grid, block, *args):
        st = self.torch.cuda.current_stream(self.dev).cuda_stream
        c_args = [ctypes.c_int(int(g)) for g in grid] + [ctypes.c_int(int(block)), ctypes.c_void_p(st)]
        for a in args:
            if hasattr(a, "data_ptr"):
                c_args.append(ctypes.c_void_p(a.data_ptr()))
            else:
                c_args.append(ctypes.c_int(int(a)))
        rc = getattr(self.lib, "refgpu_" + name)(*c_args)
        if rc != 0:
            raise RuntimeError("reference kernel %s: CUDA error %d" % (name, rc))

    def prepare(self, periods, batch):
        """durationsGrid and durationBool over the whole grid (_worker.py:100-121)
        and the per-batch buffers (:135-147)."""
        T = self.torch
        P = np.asarray(periods, dtype=np.float64)
        self.periods = P
        self.batch = int(batch)
        nP = len(P)
        self.full_max = T.empty(nP, dtype=T.int32, device=self.dev)
        self.full_min = T.empty(nP, dtype=T.int32, device=self.dev)
        self.t_size = self._i32(self.n)
        self.t_len = T.tensor([self.span], dtype=T.float32, device=self.dev)
        pd = T.tensor(P, device=self.dev)
        b, g = _grid(nP)
        self._call("durationsGrid", (g, 1, 1), b, pd, self.full_max, self.full_min, self.t_len, self.t_size,
                   self._i32(nP))
        D = len(self.durations)
        self.dur_all = T.tensor(self.durations.astype(np.int32), device=self.dev)
        self.bool_all = T.empty((nP, D), dtype=T.bool, device=self.dev)
        self._call("durationBool", (g, D, 1), b, self.full_max, self.full_min, self._i32(D), self._i32(nP),
                   self.dur_all, self.bool_all)
        S, n, m = self.batch, self.n, self.m
        self.S_dev = self._i32(S)
        self.maxd_dev = self._i32(self.max_d)
        self.m_dev = self._i32(m)
        self.dp_dev = self._i32(n)
        self.depth_dev = T.tensor([self.depth_min], dtype=T.float32, device=self.dev)
        self.phases = T.empty((S, n), dtype=T.float64, device=self.dev)
        self.sort_idx = T.empty((S, n), dtype=T.int32, device=self.dev)
        self.pdata = T.empty((S, m), dtype=T.float32, device=self.dev)
        self.pdys = T.empty((S, m), dtype=T.float32, device=self.dev)
        self.edge = T.empty(S, dtype=T.float32, device=self.dev)
        self.inv = T.empty((S, m), dtype=T.float32, device=self.dev)
        self.csum = T.empty((S, m), dtype=T.float32, device=self.dev)
        self.base_err = T.empty((S, m), dtype=T.float32, device=self.dev)
        # the (S, D, n) buffers at the largest union, reused by every batch
        # (cupy's memory pool keeps them across the batches the same way)
        self.ootr_buf = T.empty(S * D * n, dtype=T.float32, device=self.dev)
        self.lowest_buf = T.empty(S * D * n, dtype=T.float32, device=self.dev)
        self.n_batches = (nP + S - 1) // S

    def run_batch(self, b):
        """Batch ``b`` (_worker.py:174-305); returns (chi2, loc) of its periods
        on the device, or None for a batch without durations."""
        T = self.torch
        S, n, m = self.batch, self.n, self.m
        nP = len(self.periods)
        s0, s1 = b * S, min((b + 1) * S, nP)
        cnt = s1 - s0
        single = self.periods[s0:s1]
        if cnt < S:
            single = np.append(single, np.full(S - cnt, single[-1]))
        temp = self.bool_all[s0]
        for i in range(s0 + 1, s1):
            temp = T.logical_or(temp, self.bool_all[i])
        sel = temp.cpu().numpy()
        single_d = self.durations[sel]
        if len(single_d) == 0:
            return None
        D = len(single_d)
        overshoot = T.tensor(np.asarray(self.overview["overshoot"][sel], dtype=np.float32), device=self.dev)
        periods = T.tensor(single, dtype=T.float64, device=self.dev)
        dmax = T.empty(S, dtype=T.int32, device=self.dev)
        dmin = T.empty(S, dtype=T.int32, device=self.dev)
        bl, g = _grid(S)
        self._call("durationsGrid", (g, 1, 1), bl, periods, dmax, dmin, self.t_len, self.t_size, self.S_dev)
        maxlen = int(np.max(single_d))
        sig = 1 - np.array([np.pad(x, (0, maxlen - len(x)), "constant") for x in self.lc_arr[sel]])
        sig_dev = T.tensor(sig.astype(np.float32), device=self.dev)
        maxlen_dev = self._i32(maxlen)
        dur = T.tensor(single_d.astype(np.int32), device=self.dev)
        dsize = self._i32(D)
        full_sum = T.empty((S, D), dtype=T.float32, device=self.dev)
        ootr = self.ootr_buf[:S * D * n].view(S, D, n)
        lowest = self.lowest_buf[:S * D * n].view(S, D, n)
        bl, g = _grid(n)
        self._call("foldFast", (g, S, 1), bl, self.t, periods, self.phases, self.S_dev, self.t_size)
        for i in range(1, 11):
            a, c = int((i - 1) * S / 10), int(i * S / 10)
            self.sort_idx[a:c] = T.argsort(self.phases[a:c], dim=-1).to(T.int32)
        bl, g = _grid(m)
        self._call("patchData", (g, S, 1), bl, self.pdata, self.pdys, self.m_dev, self.sort_idx, self.maxd_dev,
                   self.y, self.dy, self.t_size)
        self._call("calcInverseSquaredPatchedDy", (g, S, 1), bl, self.inv, self.pdys, self.m_dev)
        bl, g = _grid(S)
        self._call("calcEdgeEffectCorrections", (g, 1, 1), bl, self.edge, self.pdata, self.inv, self.m_dev,
                   self.maxd_dev, self.S_dev)
        for i in range(S):
            self.csum[i] = T.cumsum(self.pdata[i], dim=0)
        self._call("calculate_base_error", ((m + 255) // 256, S, 1), 256, self.base_err, self.pdata, self.inv, m, S)
        eps = T.cumsum(self.base_err, dim=1)
        bl, g = _grid(D)
        self._call("calcAllFullSum_v2", (g, S, 1), bl, full_sum, eps, m, dur, D, S)
        self._call("calculate_final_ootr_v3", ((n + 255) // 256, D, S), 256, ootr, eps, full_sum, dur, n, m, D, S)
        bl, g = _grid(n)
        self._call("lowest_v2", (g, D, S), bl, lowest, self.t_size, self.pdata, self.m_dev, dur, dsize, sig_dev,
                   maxlen_dev, self.inv, overshoot, ootr, full_sum, self.edge, self.dp_dev, self.csum,
                   self.depth_dev)
        flat = lowest[:cnt].reshape(cnt, -1)
        loc = T.argmin(flat, dim=-1)
        val = flat[T.arange(cnt, device=self.dev), loc]
        return val, loc
