"""Multi-rank sharding of the search (gtls_b200/shard.py) on the CPU: gloo,
world size 2, the oracle standing in for each rank's GPU main pass.

A sharded search must give every rank the result an unsharded search gives:
period ranges cut at whole duration-union batches reproduce the chi2 of
every period exactly, and the curve partition covers every curve once.
"""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, search_inputs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_balanced_partition_covers_and_balances():
    from gtls_b200 import shard
    rng = np.random.default_rng(3)
    costs = rng.lognormal(0.0, 1.0, 257)
    for world in (1, 2, 3, 8):
        parts = shard.balanced_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max() + 1e-9
    assert shard.balanced_partition([5.0, 5.0, 1.0], 2) == [[0, 2], [1]]


def test_aligned_ranges_cut_at_whole_batches():
    from gtls_b200 import shard
    for n, batch, world in [(100, 7, 2), (100, 7, 3), (5, 7, 2), (0, 3, 2), (64, 8, 8), (1000, 1, 3)]:
        rs = shard.aligned_ranges(n, batch, world)
        assert len(rs) == world and rs[0][0] == 0 and rs[-1][1] == n
        for (a0, a1), (b0, b1) in zip(rs, rs[1:]):
            assert a1 == b0 and a0 <= a1
        for a, b in rs[:-1]:
            assert b % batch == 0 or b == n
    with pytest.raises(ValueError):
        shard.aligned_ranges(10, 0, 2)


def _rank_main(rank, world, port, out_dir, case):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from gtls_b200 import shard
        if case == "periods":
            import tls_oracle as O
            from conftest import search_inputs as si
            s = si(seed=21, n=700, span=4.0)
            P = s["periods"][::9]

            def main_pass(p0, p1):
                c, _ = O.search_periods(O.NumpyBackend(), P[p0:p1], s["t"], s["y"], s["dy"], s["widths"],
                                        s["templates"], s["overshoot"], s["maxd"], 1e-5, 8, 7)
                return c

            full = shard.sharded_period_pass(len(P), 7, main_pass)
            np.save(os.path.join(out_dir, "periods_%d.npy" % rank), full.numpy())
        else:
            costs = [float(c) for c in np.arange(1, 12)]
            searched = []

            def search_subset(idx):
                searched.extend(idx)
                return [{"index": i, "value": 10.0 * i, "rank": rank} for i in idx]

            res = shard.sharded_curves(costs, search_subset)
            np.save(os.path.join(out_dir, "curves_%d.npy" % rank),
                    np.array([[r["index"], r["value"], r["rank"]] for r in res]))
            np.save(os.path.join(out_dir, "searched_%d.npy" % rank), np.array(searched, dtype=np.int64))
    finally:
        dist.destroy_process_group()


def _spawn(case, out_dir, world=2):
    mp.spawn(_rank_main, args=(world, _free_port(), out_dir, case), nprocs=world, join=True)


def test_sharded_period_pass_equals_unsharded():
    import tls_oracle as O
    s = search_inputs(seed=21, n=700, span=4.0)
    P = s["periods"][::9]
    ref, _ = O.search_periods(O.NumpyBackend(), P, s["t"], s["y"], s["dy"], s["widths"], s["templates"],
                              s["overshoot"], s["maxd"], 1e-5, 8, 7)
    with tempfile.TemporaryDirectory() as d:
        _spawn("periods", d)
        r0 = np.load(os.path.join(d, "periods_0.npy"))
        r1 = np.load(os.path.join(d, "periods_1.npy"))
    np.testing.assert_array_equal(r0, r1)
    np.testing.assert_array_equal(r0, ref)


def test_sharded_curves_cover_every_curve_once():
    with tempfile.TemporaryDirectory() as d:
        _spawn("curves", d)
        c0 = np.load(os.path.join(d, "curves_0.npy"))
        c1 = np.load(os.path.join(d, "curves_1.npy"))
        s0 = np.load(os.path.join(d, "searched_0.npy"))
        s1 = np.load(os.path.join(d, "searched_1.npy"))
    np.testing.assert_array_equal(c0, c1)
    np.testing.assert_array_equal(c0[:, 0], np.arange(11))
    np.testing.assert_array_equal(c0[:, 1], 10.0 * np.arange(11))
    assert sorted(np.concatenate([s0, s1]).tolist()) == list(range(11))
    assert len(s0) > 0 and len(s1) > 0


def test_multi_device_period_pass_concatenates_aligned_ranges_in_order():
    """GPUDeviceIDs in one process: one batch-aligned range per listed device,
    ranges of a repeated device run one after the other on its thread, and
    the chi2 segments come back concatenated in period order."""
    import threading
    from gtls_b200 import shard
    calls = []
    lock = threading.Lock()

    def main_pass(device, p0, p1):
        with lock:
            calls.append((device, p0, p1))
        return np.arange(p0, p1, dtype=np.float64) * 10 + device

    out = shard.multi_device_period_pass(103, 10, [0, 1, 0, 2], main_pass)
    ranges = shard.aligned_ranges(103, 10, 4)
    expect = np.concatenate([np.arange(a, b) * 10.0 + d for (a, b), d in zip(ranges, [0, 1, 0, 2])])
    np.testing.assert_array_equal(out, expect)
    assert sorted(calls) == sorted((d, a, b) for (a, b), d in zip(ranges, [0, 1, 0, 2]) if b > a)
    assert all(a % 10 == 0 for a, _ in ranges)
