"""Write tests/golden/cfg3_oracle.npz: the FP64 oracle's search results for
the 64 seeds of the mixed-precision workload (19,728 samples at 2-min
cadence over 27.4 d, depth log-U(100, 2000) ppm, P log-U(1, 500) d): for each
seed the best period index and period, the width, SDE, depth, T0 and
duration, and the chi2 spectrum (stored in float32), from the oracle's host flow
(oracle/tls_oracle.search, core.py:568-999) over the reference's kernels
compiled for the CPU in FP64 (oracle/_ref, R64).  Grid, templates and
duration-union batch size are the ones gtls().power() uses on a GPU whose
free memory does not bind the batch size (core.py:620-628).  bench.py
--workload cfg3 compares the FP32 form with these.

    python tests/golden/make_cfg3_oracle.py [n_seeds]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def oracle_inputs(seed):
    """The grid, templates and batch size of the seed's default search."""
    from gtls_b200 import core, grid as G, synthetic, template, validate as V
    t, y, dy, _ = synthetic.light_curve_cfg3(seed)
    t, y, dy = V.validate_inputs(t, y, dy)
    P = G.period_grid(1, 1, t.max() - t.min(), 0.5, 13.7, 3, 2, ascending=True)
    durs = G.duration_grid(P, shortest=1 / len(t))
    mw = int(np.max(durs) * len(y))
    mw += mw % 2
    ov, lc = template.get_cache(durs, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    widths, os_, dd, tm, maxd = template.device_templates(lc, ov)
    batch = core.reference_batch_size(len(P), len(t), maxd, len(widths), 1e15)
    return t, y, dy, P, widths, os_, dd, tm, maxd, batch


def main(n_seeds):
    import ref_replay as RR
    import tls_oracle as O
    be = RR.RefKernelBackend("r64", 8)
    out = {}
    for seed in range(n_seeds):
        t, y, dy, P, widths, os_, dd, tm, maxd, batch = oracle_inputs(seed)
        r = O.search(be, P, t, y, dy, widths, tm, os_, dd, maxd, 1e-5, 0.125, 3, batch=batch)
        out["seed%d_scalars" % seed] = np.array([r["period_index"], r["period"], r["width"], r["SDE"], r["depth"],
                                                 r["T0"], r["duration"], batch], dtype=np.float64)
        out["seed%d_chi2" % seed] = np.ma.getdata(r["chi2"]).astype(np.float32)   # ample for 2e-6 bars
        print("seed", seed, r["period_index"], r["SDE"], flush=True)
        np.savez_compressed(os.path.join(HERE, "cfg3_oracle.npz"), n_seeds=np.array(seed + 1), **out)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 64)
