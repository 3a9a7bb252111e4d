"""Disk-parallel sweeps over several GPUs.

Disks of a sweep are independent (nothing couples two disks inside a DT), so
the path shards by disk with no exchange in the data path: one process per
GPU (torch.distributed for the plumbing), each advancing its own batch of
disks.  Disks are assigned by greedy longest-processing-time on their cell
counts, the timed region is bracketed by barriers and reported as the
maximum device time over ranks, and per-disk results are gathered on rank 0
at the end.

A single disk is not decomposed: one disk runs on one GPU ("replicas only").
"""
import datetime
import os

import numpy as np


def lpt_partition(weights, nparts):
    """Greedy LPT: heaviest item first onto the lightest part.

    Deterministic (ties broken by index), so every rank computes the same
    partition without communicating.  Returns nparts lists of item indices,
    each in increasing order.
    """
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * nparts
    parts = [[] for _ in range(nparts)]
    for i in order:
        p = min(range(nparts), key=lambda k: (load[k], k))
        parts[p].append(i)
        load[p] += w[i]
    return [sorted(p) for p in parts]


def group_by_substeps(cells, nsub, ngroups):
    """Batches of disks with similar substep counts and balanced work.

    A batch advances until its slowest disk ends its DT, so a disk that
    needs few CFL substeps idles through the rest of its batch's DT.  Sorted
    by substep count (ties by index) and cut into `ngroups` contiguous runs,
    the disks of one batch need about as many substeps as each other; the
    cut points are chosen greedily so that the runs' work (sum of cells x
    substeps) is as even as possible (the batches advance concurrently on
    their own streams).  Returns ngroups sorted lists of disk indices."""
    cells = np.asarray(cells, dtype=np.float64)
    nsub = np.asarray(nsub, dtype=np.float64)
    n = len(cells)
    if ngroups < 1:
        raise ValueError("ngroups must be >= 1")
    ngroups = min(ngroups, n)
    order = sorted(range(n), key=lambda i: (nsub[i], i))
    w = (cells * nsub)[order]
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    cuts = [0]
    for g in range(1, ngroups):
        target = total * g / ngroups
        k = int(np.searchsorted(cum, target))
        # the nearer of the two candidate cut points, keeping every run non-empty
        if k > 0 and abs(cum[k - 1] - target) <= abs(cum[min(k, n)] - target):
            k -= 1
        k = max(k, cuts[-1] + 1)
        k = min(k, n - (ngroups - g))
        cuts.append(k)
    cuts.append(n)
    return [sorted(order[cuts[g]:cuts[g + 1]]) for g in range(ngroups)]


def disk_cells(params):
    return [int(p.NRAD) * int(p.NSEC) for p in params]


def shard_of(params, rank, world):
    """Indices of the disks that rank `rank` of `world` advances."""
    return lpt_partition(disk_cells(params), world)[rank]


def init_process_group(backend, timeout_s=120):
    """One process per GPU (or per CPU rank with gloo), from the launcher's
    RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT."""
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def reduce_timing(ms, units, device="cpu"):
    """(max over ranks of ms, sum over ranks of units); identity without a
    process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(ms), float(units)
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def gather_results(local):
    """Merge per-rank {disk index: result} dicts on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, local)
    merged = {}
    for part in out:
        merged.update(part)
    return merged


def run_sweep(params, planets, ndt, rank=0, world=1, make_batch=None, device=0):
    """Advance this rank's share of the sweep by ndt DTs and return every
    disk's scalars, gathered from all ranks: {disk index: scalars dict}.

    make_batch(params, planets, device) builds the engine for a list of disks
    (default: the CUDA batch of this package)."""
    if make_batch is None:
        from .disk import Batch

        def make_batch(p, l, dev):
            return Batch(p, l, device=dev)
    mine = shard_of(params, rank, world)
    local = {}
    if mine:
        b = make_batch([params[i] for i in mine], [planets[i] for i in mine], device)
        try:
            b.advance(ndt)
            for k, i in enumerate(mine):
                local[i] = b.scalars(k)
        finally:
            b.close()
    return gather_results(local)
