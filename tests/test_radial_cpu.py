"""Radial decomposition of one disk: the host logic, on CPU.

- partition(): cuts on whole CFL tiles, every stripe at least `ghost` rings.
- drive_dt() with the in-process exchange and with torch.distributed over
  gloo (2 and 3 ranks): a numpy stand-in of a stripe with the library's
  per-substep surface (forces -> block, substep from the gathered blocks,
  halo pack / unpack) must give, on its own rows, the bits of the same
  stand-in run undecomposed.  The stand-in's update has a radial reach per
  substep and a boundary rule at its local edges, so a ghost zone narrower
  than the reach, a halo sent the wrong way or blocks gathered out of order
  all change the result.  Its self-gravitating form also takes a term from
  every ring of the whole grid (the gathered own rows), as the library's
  stripes take the whole disk's convolution.
- fargo_stripe_create's argument checks (no GPU needed: they run first).
"""
import ctypes as C
import multiprocessing as mp
import os
import socket
import tempfile

import types

import numpy as np
import pytest
import torch

from cudaprotoplanetarydisksfloat_b200 import radial
from cudaprotoplanetarydisksfloat_b200._abi import FargoPlanets, lib
from tests.helpers import small

NRAD, NSEC, REACH, DT = 60, 16, 3, 1.0


def _init():
    rng = np.random.default_rng(11)
    return rng.random((NRAD + 1, NSEC)).astype(np.float32) + 1.0


class FakeStripe:
    """Numpy stand-in of radial.Stripe: rows lo..hi-1 own, `ghost` more on
    each side.  A substep: block = (minimum of a per-row limit, one partial
    per own row); the scalars from all blocks in stripe order; then REACH
    passes of a 3-row stencil plus the gathered total, with a boundary rule
    on the local edge rows (the cut edges' rule is not the disk's)."""

    def __init__(self, lo, hi, ghost, u0, sg=False):
        self.lo, self.hi, self.sg = lo, hi, sg
        self.params = types.SimpleNamespace(NSEC=NSEC)
        self.gterm = 0.0
        self.base = max(0, lo - ghost)
        top = min(NRAD, hi + ghost)
        self.own_lo, self.own_hi = lo - self.base, hi - self.base
        self.glo, self.ghi = lo - self.base, top - hi
        self.u = u0[self.base:top + 1].copy()
        self.block_doubles = radial._abi.FARGO_STRIPE_HEAD + (hi - lo)
        self.device, self.stream = torch.device("cpu"), None
        f = dict(dtype=torch.float32)
        self.send_lo = torch.zeros(max(1, self.glo * NSEC), **f)
        self.recv_lo = torch.zeros(max(1, self.glo * NSEC), **f)
        self.send_hi = torch.zeros(max(1, self.ghi * NSEC), **f)
        self.recv_hi = torch.zeros(max(1, self.ghi * NSEC), **f)
        self.history = []

    def set_stride(self, stride):
        self.stride = stride
        self.block = torch.zeros(stride, dtype=torch.float64)

    def set_sg_stride(self, stride):
        self.sg_send = torch.zeros(stride, dtype=torch.float32)

    def sg_rows(self):
        own = self.u[self.own_lo:self.own_hi].reshape(-1)
        self.sg_send[:own.size].copy_(torch.from_numpy(own.copy()))

    def sg_apply(self, gathered, nstripe, stride, cuts):
        g = gathered.numpy()
        whole = np.concatenate([g[k * stride:k * stride + (cuts[k + 1] - cuts[k]) * NSEC] for k in range(nstripe)])
        ring = whole.reshape(NRAD, NSEC).astype(np.float64).mean(axis=1)
        ring = np.append(ring, 0.0)  # the row at NRAD
        self.gterm = (1e-4 * ring[self.base:self.base + self.u.shape[0]]).astype(np.float32)[:, None]

    def dt_begin(self):
        self.dtemp = 0.0

    def forces(self):
        own = self.u[self.own_lo:self.own_hi]
        lim = 1.0 / (1.0 + np.abs(own).max(axis=1))
        b = self.block.numpy()
        b[0] = np.float32(lim.min()) * 0.25
        b[1] = self.hi - self.lo
        b[2] = 1
        b[3:3 + own.shape[0]] = own.astype(np.float64).sum(axis=1)

    def substep(self, blocks, nstripe, stride):
        blk = blocks.numpy()
        m = min(np.float32(blk[k * stride]) for k in range(nstripe))
        total = 0.0
        for k in range(nstripe):  # tiles in stripe order, summed in sequence
            n = int(blk[k * stride + 1])
            for t in range(n):
                total += blk[k * stride + 3 + t]
        dt = min(float(m), DT - self.dtemp)
        self.dtemp += dt
        self.history.append((dt, total))
        u = self.u
        for _ in range(REACH):
            v = u.copy()
            v[1:-1] = u[1:-1] + np.float32(0.2) * (u[:-2] - 2 * u[1:-1] + u[2:]) + np.float32(1e-6 * total)
            v = v + self.gterm
            v[0] = np.float32(0.5) * u[1]  # boundary rule at the local edges
            v[-1] = np.float32(0.5) * u[-2]
            u = np.roll(v, 1, axis=1)
        self.u = u
        self._more = 1 if self.dtemp < 0.999999 * DT else 0

    def pack(self):
        if self.glo:
            self.send_lo.copy_(torch.from_numpy(self.u[self.own_lo:self.own_lo + self.glo].reshape(-1)))
        if self.ghi:
            self.send_hi.copy_(torch.from_numpy(self.u[self.own_hi - self.ghi:self.own_hi].reshape(-1)))

    def more(self):
        return self._more

    def unpack(self):
        if self.glo:
            self.u[:self.glo] = self.recv_lo.numpy().reshape(self.glo, NSEC)
        if self.ghi:
            self.u[self.own_hi:self.own_hi + self.ghi] = self.recv_hi.numpy().reshape(self.ghi, NSEC)

    def own(self):
        top = self.own_hi + (1 if self.hi == NRAD else 0)
        return self.u[self.own_lo:top]


def _whole(ndt, sg=False):
    s = FakeStripe(0, NRAD, 1, _init(), sg)
    x = radial.LocalExchange([s])
    n = [radial.drive_dt([s], x) for _ in range(ndt)]
    return s.own(), n, s.history


def _assemble(stripes):
    out = np.zeros((NRAD + 1, NSEC), np.float32)
    for s in stripes:
        o = s.own()
        out[s.lo:s.lo + o.shape[0]] = o
    return out


def test_partition_cuts_on_whole_tiles():
    for nrad, nsec in [(2048, 6144), (512, 1536), (256, 768), (512, 1024), (384, 1152)]:
        g = radial.granule(nsec)
        assert (g * nsec) % 4096 == 0
        for n in (1, 2, 4, 8):
            parts = radial.partition(nrad, nsec, n)
            assert parts[0][0] == 0 and parts[-1][1] == nrad and len(parts) == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            assert all(lo % g == 0 for lo, _ in parts)
            assert all(hi - lo >= radial.GHOST for lo, hi in parts) or n == 1
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 2 * g
    with pytest.raises(ValueError):
        radial.partition(64, 384, 8)  # 32-ring granule: stripes of 0 or 32 rings


@pytest.mark.parametrize("sg", [False, True], ids=["plain", "self-gravity"])
def test_local_exchange_matches_whole(sg):
    want, nsub, hist = _whole(3, sg)
    for parts, ghost in ([[(0, 20), (20, 40), (40, 60)], 10], [[(0, 24), (24, 60)], 12]):
        ss = [FakeStripe(lo, hi, ghost, _init(), sg) for lo, hi in parts]
        x = radial.LocalExchange(ss)
        got = [radial.drive_dt(ss, x) for _ in range(3)]
        assert got == nsub
        assert all(s.history == hist for s in ss)
        assert np.array_equal(_assemble(ss), want)


def test_narrow_ghost_zone_is_detected():
    """A ghost zone narrower than the substep's reach lets the cut edges'
    boundary rule into the own rows: the stand-in then differs."""
    want, _, _ = _whole(2)
    ss = [FakeStripe(lo, hi, REACH - 1, _init()) for lo, hi in [(0, 30), (30, 60)]]
    x = radial.LocalExchange(ss)
    for _ in range(2):
        radial.drive_dt(ss, x)
    assert not np.array_equal(_assemble(ss), want)


def _rank_main(rank, world, port, out, sg):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        parts = radial.partition(NRAD, NSEC, world, ghost=REACH + 1, aligned=False)
        lo, hi = parts[rank]
        s = FakeStripe(lo, hi, REACH + 1, _init(), sg)
        x = radial.DistExchange([s], parts=parts)
        nsub = [radial.drive_dt([s], x) for _ in range(3)]
        np.savez(out % rank, own=s.own(), lo=lo, nsub=nsub, hist=np.array(s.history))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,sg", [(2, False), (3, False), (3, True)])
def test_gloo_ranks_match_whole(world, sg):
    want, nsub, hist = _whole(3, sg)
    out = os.path.join(tempfile.mkdtemp(prefix="fargo_radial_"), "rank%d.npz")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out, sg)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    got = np.zeros_like(want)
    for r in range(world):
        z = np.load(out % r)
        o, lo = z["own"], int(z["lo"])
        got[lo:lo + o.shape[0]] = o
        assert list(z["nsub"]) == nsub
        assert np.array_equal(z["hist"], np.array(hist))
    assert np.array_equal(got, want)


def test_stripe_create_checks_arguments():
    """Refusals that come before any device work (so they run without a GPU)."""
    P, L, _ = small("iso", 64, 128)
    cases = [(0, 0, 8), (10, 70, 8), (0, 32, 0), (0, 4, 8)]
    for lo, hi, ghost in cases:
        ctx = C.c_void_p()
        st = lib.fargo_stripe_create(C.byref(P), C.byref(L), None, lo, hi, ghost, 0, C.byref(ctx))
        assert st == 1, (lo, hi, ghost)  # FARGO_EINVAL
        assert lib.fargo_last_error(ctx)
        lib.fargo_destroy(ctx)
    op = type(P).from_buffer_copy(P)
    op.OpenInner = 1
    ctx = C.c_void_p()
    assert lib.fargo_stripe_create(C.byref(op), C.byref(FargoPlanets()), None, 0, 32, 8, 0, C.byref(ctx)) == 1
    assert b"RIGID" in lib.fargo_last_error(ctx)
    lib.fargo_destroy(ctx)
