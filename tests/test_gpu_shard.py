"""Sharded search through the public API on the GPU: two ranks (gloo for the
host-side all-gathers) share the one GPU of this machine; each runs the main
pass over its batch-aligned period range or its share of the curves, and
every rank must return exactly the unsharded result."""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _curves():
    from gtls_b200 import synthetic
    return [synthetic.small_curve(seed=41 + i, n=1400 + 300 * i, span=6.0 + i, period=1.3 + 0.3 * i, depth=4e-3)[:2]
            for i in range(3)]


KW = dict(precision="fp64", oversampling_factor=2, use_threads=1)


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from gtls_b200 import gtls
        from gtls_b200.batch import gtls_batch
        t, y = _curves()[1]
        r = gtls(t, y, verbose=False).power(distributed=True, batch_periods=20, **KW)
        np.save(os.path.join(out_dir, "single_%d.npy" % rank),
                np.concatenate([[r.period, r.SDE, r.depth, r.T0, r.duration], np.ma.filled(r.chi2, -1.0)]))
        # default batch size: rank 0's value is broadcast, so the ranks agree
        r2 = gtls(t, y, verbose=False).power(distributed=True, **KW)
        np.save(os.path.join(out_dir, "default_%d.npy" % rank), np.ma.filled(r2.chi2, -1.0))
        rb = gtls_batch(_curves()).power(distributed=True, batch_periods=20, **KW)
        np.save(os.path.join(out_dir, "batch_%d.npy" % rank),
                np.array([[x.period, x.SDE, x.depth, x.T0] for x in rb]))
    finally:
        dist.destroy_process_group()


def test_sharded_search_equals_unsharded(cuda):
    from gtls_b200 import gtls
    from gtls_b200.batch import gtls_batch
    t, y = _curves()[1]
    ref = gtls(t, y, verbose=False).power(batch_periods=20, **KW)
    refb = gtls_batch(_curves()).power(batch_periods=20, **KW)
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank_main, args=(2, _free_port(), d), nprocs=2, join=True)
        s = [np.load(os.path.join(d, "single_%d.npy" % r)) for r in range(2)]
        b = [np.load(os.path.join(d, "batch_%d.npy" % r)) for r in range(2)]
        dflt = [np.load(os.path.join(d, "default_%d.npy" % r)) for r in range(2)]
    np.testing.assert_array_equal(dflt[0], dflt[1])
    want = np.concatenate([[ref.period, ref.SDE, ref.depth, ref.T0, ref.duration], np.ma.filled(ref.chi2, -1.0)])
    np.testing.assert_array_equal(s[0], s[1])
    np.testing.assert_array_equal(s[0], want)
    np.testing.assert_array_equal(b[0], b[1])
    np.testing.assert_array_equal(b[0], np.array([[x.period, x.SDE, x.depth, x.T0] for x in refb]))


@pytest.mark.gpu
def test_power_with_several_device_ids_equals_one_device(cuda):
    """power(GPUDeviceIDs=[0, 0, 0]): the main pass in three batch-aligned
    ranges (on a one-GPU machine all on device 0, one after the other) gives
    exactly the single-device result."""
    from gtls_b200 import gtls
    from conftest import search_inputs
    s = search_inputs(seed=31, n=1500, span=6.0)
    one = gtls(s["t"], s["y"], verbose=False).power(periods=s["periods"], batch_periods=7)
    three = gtls(s["t"], s["y"], verbose=False).power(periods=s["periods"], batch_periods=7, GPUDeviceIDs=[0, 0, 0])
    np.testing.assert_array_equal(three.diagnostics["chi2_main"], one.diagnostics["chi2_main"])
    assert three.period == one.period and three.SDE == one.SDE
