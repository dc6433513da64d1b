"""Multi-GPU sharding of the search: one process per GPU, torch.distributed.

The units of work are independent (a (curve, period) chi2 needs nothing from
any other), so sharding needs no exchange during the search:

* many curves (``gtls_batch``): each rank searches a subset of the curves,
  chosen to balance the estimated work (samples x trial periods); the
  per-curve results, a few numbers and spectra each, are gathered at the end;
* one long curve (``gtls(...).power(distributed=True)``): each rank runs the
  main pass over a contiguous range of the period grid, the ranges cut at
  multiples of the duration-union batch so that every batch (and so every
  chi2 value) is the one an unsharded search computes; the chi2 spectrum
  (8 bytes per period) is then all-gathered and every rank finishes the
  search (spectra, candidate re-search, best period) identically.  This is
  the reference's multi-GPU mode (contiguous period ranges per GPU worker,
  core.py:318-564, gathered on the host) with the workers as ranks.

The collectives are plain all-gathers (NCCL for CUDA tensors, gloo on the
CPU); nothing here issues device code.
"""
import numpy as np


def balanced_partition(costs, world):
    """Indices of ``costs`` split into ``world`` lists of near-equal total cost.

    Longest-processing-time greedy: items in decreasing cost (ties by
    index) go to the currently lightest rank (ties by rank).  Deterministic;
    each list is returned in increasing index order."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def aligned_ranges(n, batch, world):
    """``world`` contiguous ranges covering [0, n) whose inner boundaries are
    multiples of ``batch`` (whole duration-union batches per rank), with the
    batches spread as evenly as possible.  Some ranges may be empty."""
    if n < 0 or batch < 1 or world < 1:
        raise ValueError("n >= 0, batch >= 1 and world >= 1 required")
    nb = (n + batch - 1) // batch
    out = []
    for r in range(world):
        b0 = nb * r // world
        b1 = nb * (r + 1) // world
        out.append((min(n, b0 * batch), min(n, b1 * batch)))
    return out


def _dist():
    import torch.distributed as dist
    return dist


def world_info(group=None):
    """(rank, world size) of the default or given process group; (0, 1)
    when torch.distributed is not initialised."""
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def gather_segments(local, ranges, group=None, device=None):
    """All-gather the 1-D float64 segments of every rank (rank r holds the
    values of ``ranges[r]``) into the full array, on every rank.  ``local``
    is a numpy array or a tensor; ``device`` is where the collective runs
    (a CUDA device for NCCL, None for CPU/gloo)."""
    import torch
    dist = _dist()
    rank, world = world_info(group)
    width = max(b - a for a, b in ranges) if ranges else 0
    t = torch.as_tensor(np.asarray(local, dtype=np.float64) if not torch.is_tensor(local) else local,
                        dtype=torch.float64)
    if device is not None:
        t = t.to(device)
    if t.numel() != ranges[rank][1] - ranges[rank][0]:
        raise ValueError("local segment does not match this rank's range")
    buf = torch.zeros(max(width, 1), dtype=torch.float64, device=t.device)
    buf[:t.numel()] = t
    bufs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    full = torch.cat([bufs[r][:ranges[r][1] - ranges[r][0]] for r in range(world)])
    return full


def sharded_period_pass(n_periods, batch, main_pass, group=None, device=None):
    """Run ``main_pass(p0, p1)`` (chi2 of periods [p0, p1), a 1-D array or
    tensor) on this rank's batch-aligned range and return the full chi2
    array (a tensor on ``device``) on every rank."""
    rank, world = world_info(group)
    ranges = aligned_ranges(n_periods, batch, world)
    p0, p1 = ranges[rank]
    local = main_pass(p0, p1)
    if world == 1:
        return local
    return gather_segments(local, ranges, group=group, device=device)


def sharded_curves(costs, search_subset, group=None):
    """Search the curves of this rank's share (``search_subset(indices)``
    returns one picklable result per index, in order) and return every
    curve's result, in the original order, on every rank."""
    dist = _dist()
    rank, world = world_info(group)
    parts = balanced_partition(costs, world)
    mine = parts[rank]
    local = list(search_subset(mine)) if mine else []
    if len(local) != len(mine):
        raise ValueError("search_subset returned %d results for %d curves" % (len(local), len(mine)))
    if world == 1:
        return local
    gathered = [None] * world
    dist.all_gather_object(gathered, list(zip(mine, local)), group=group)
    out = [None] * len(costs)
    for pairs in gathered:
        for i, res in pairs:
            out[i] = res
    return out


def multi_device_period_pass(n_periods, batch, devices, main_pass):
    """The reference's in-process multi-GPU mode (``power(GPUDeviceIDs=[...])``,
    core.py:318-564: contiguous period ranges per GPU, concatenated): the
    period list is cut into one batch-aligned range per entry of ``devices``
    (so every chi2 value is the unsharded one) and ``main_pass(device, p0,
    p1)`` (a host float64 array) runs for each, one host thread per distinct
    device so that the devices work at the same time (ranges of a repeated
    device run one after the other on it).  Returns the concatenated host
    array."""
    import threading
    ranges = aligned_ranges(n_periods, batch, len(devices))
    out = [None] * len(devices)
    errors = []
    by_device = {}
    for i, d in enumerate(devices):
        by_device.setdefault(int(d), []).append(i)

    def work(idx):
        try:
            for i in idx:
                a, b = ranges[i]
                out[i] = main_pass(int(devices[i]), a, b) if b > a else np.zeros(0)
        except Exception as e:   # re-raised on the calling thread
            errors.append(e)

    threads = [threading.Thread(target=work, args=(idx,)) for idx in by_device.values()]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    if errors:
        raise errors[0]
    return np.concatenate([np.asarray(o, dtype=np.float64) for o in out])
