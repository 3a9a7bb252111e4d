"""The disk-parallel sweep over several ranks, on CPU with gloo.

Two ranks split a sweep of small disks by LPT on cell counts, advance their
shares and gather every disk's scalars; the result must equal one rank
running the whole sweep.  The oracle stands in for the CUDA batch (same
interface: advance(ndt), scalars(k), close()), so the partitioning, the
gather and the max/sum timing reduction are exercised without a GPU."""
import json
import multiprocessing as mp
import os
import socket
import tempfile

import numpy as np

from cudaprotoplanetarydisksfloat_b200 import shard
from tests.helpers import small

SIZES = [(16, 48), (24, 72), (32, 96), (20, 60), (12, 40)]


class OracleBatch:
    """A batch of disks advanced by the CPU oracle."""

    def __init__(self, params, planets, device):
        from oracle.oracle import Oracle
        self.disks = [Oracle(p, l) for p, l in zip(params, planets)]

    def advance(self, ndt):
        for o in self.disks:
            for _ in range(ndt):
                o.advance_dt()

    def scalars(self, k):
        s = self.disks[k].scalars()
        return {key: float(v) for key, v in s.items()}

    def close(self):
        for o in self.disks:
            o.close()


def _sweep():
    P, L = [], []
    for nrad, nsec in SIZES:
        p, l, _ = small("iso", nrad, nsec)
        P.append(p)
        L.append(l)
    return P, L


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist = shard.init_process_group("gloo", timeout_s=60)
    try:
        P, L = _sweep()
        res = shard.run_sweep(P, L, 2, rank=rank, world=world, make_batch=OracleBatch)
        ms, units = shard.reduce_timing(1.0 + rank, 10.0 * (rank + 1))
        if rank == 0:
            with open(out, "w") as f:
                json.dump({"res": {str(k): v for k, v in res.items()}, "ms": ms, "units": units}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_lpt_partition_covers_and_balances():
    w = [786432, 49152, 110592, 196608, 442368, 49152, 786432, 110592]
    for n in (1, 2, 3, 4, 8):
        parts = shard.lpt_partition(w, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(w) / n + max(w)
        assert parts == shard.lpt_partition(w, n)  # deterministic


def test_two_rank_sweep_matches_one_rank():
    P, L = _sweep()
    want = shard.run_sweep(P, L, 2, make_batch=OracleBatch)
    out = os.path.join(tempfile.mkdtemp(prefix="fargo_mr_"), "rank0.json")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    with open(out) as f:
        got = json.load(f)
    assert got["ms"] == 2.0 and got["units"] == 30.0  # max and sum over ranks
    assert sorted(int(k) for k in got["res"]) == list(range(len(SIZES)))
    for k, s in want.items():
        g = got["res"][str(k)]
        for key in ("nsub_total", "physical_time", "mass", "angular_momentum"):
            assert np.float64(g[key]) == np.float64(s[key]), (k, key)


def test_bench_batch_groups_cover_and_balance():
    import bench
    cells = [int(p["Nrad"]) * int(p["Nsec"]) for p, _ in __import__(
        "cudaprotoplanetarydisksfloat_b200").configs.c4(64, seed=42)]
    assert bench.batch_groups(cells, 4, plain=True) == [[d] for d in range(64)]
    assert bench.batch_groups(cells, 1, plain=False) == [list(range(64))]
    for g in (2, 4, 8):
        parts = bench.batch_groups(cells, g, plain=False)
        assert len(parts) == g
        assert sorted(d for p in parts for d in p) == list(range(64))
        loads = [sum(cells[d] for d in p) for p in parts]
        assert max(loads) <= sum(cells) / g + max(cells)


def test_group_by_substeps_cover_contiguous_balanced():
    """Batches by substep count: every disk once, each batch a contiguous run
    of the substep order, work (cells x substeps) evenly split."""
    from cudaprotoplanetarydisksfloat_b200 import shard
    rng = np.random.default_rng(3)
    nrad = rng.choice([128, 192, 256, 384, 512], 64)
    cells = nrad * 3 * nrad
    nsub = rng.integers(7, 55, 64)
    for G in (1, 2, 4, 6):
        gs = shard.group_by_substeps(cells, nsub, G)
        assert len(gs) == G and all(gs)
        assert sorted(sum(gs, [])) == list(range(64))
        # contiguous in substep order: no batch's range of counts overlaps another's interior
        spans = sorted((min(nsub[g]), max(nsub[g])) for g in gs)
        for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
            assert a1 <= b0
        work = [float((cells[g] * nsub[g]).sum()) for g in gs]
        # at most one disk's work above the even share
        assert max(work) <= sum(work) / G + float((cells * nsub).max())
