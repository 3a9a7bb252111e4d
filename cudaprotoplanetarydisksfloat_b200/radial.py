"""Radial decomposition of one disk: stripes of rings on several GPUs.

The loop of AlgoGas (SourceEuler.cu:208-301) advances one grid; here the
rings are split into stripes, each a context of its own (fargo_stripe_* in
the C ABI) that computes its own rings plus ghost rings on each side.  Per
substep:

  1. every stripe forms its CFL minimum and disk-force partials over its own
     rings (fargo_stripe_forces) into a block;
  2. the blocks are gathered in stripe order (all-gather); every stripe
     derives the same dt, planet update and substep decision from them
     (fargo_stripe_substep), then runs the rest of the substep;
  3. the own rings next to each cut are sent to the neighbouring stripe,
     whose ghost rings they replace (halo exchange).
A self-gravitating disk first gathers every stripe's own density rings
(all-gather): each stripe runs the whole disk's convolution on the whole
density and keeps its own rings' accelerations (fargo_stripe_sg_*).

With the cuts on whole CFL tiles and ghost >= FARGO_STRIPE_GHOST the own
rings carry, after every substep, the bits of the same disk advanced whole.

Two ways to run it:
  DistStripes   one stripe per rank of torch.distributed (NCCL between the
                GPUs: all-gather of the blocks, send/recv of the halos)
  LocalStripes  every stripe in this process (one GPU or several), the
                exchange by device copies
Both drive the same per-DT sequence (drive_dt) through an exchange object
(DistExchange, LocalExchange) with two operations, gather and halo.
"""
import ctypes as C
import math

import numpy as np
import torch

from . import _abi
from ._abi import FargoStripeLayout, check, lib

GHOST = _abi.FARGO_STRIPE_GHOST


def granule(nsec):
    """Rings per whole number of CFL tiles: cuts at multiples of it keep the
    disk's tiles (and so its force sums) unchanged."""
    return _abi.FARGO_CFL_TILE // math.gcd(int(nsec), _abi.FARGO_CFL_TILE)


def partition(nrad, nsec, nstripes, ghost=GHOST, aligned=True):
    """[(lo, hi)] own rings of each stripe: near-equal shares, inner cuts at
    multiples of granule(nsec) (aligned) or of one ring, each stripe at
    least `ghost` rings."""
    if nstripes < 1:
        raise ValueError("nstripes must be >= 1")
    g = granule(nsec) if aligned else 1
    cuts = [0] + [int(round(k * nrad / nstripes / g)) * g for k in range(1, nstripes)] + [int(nrad)]
    parts = list(zip(cuts[:-1], cuts[1:]))
    if nstripes > 1:
        for lo, hi in parts:
            if hi - lo < ghost:
                raise ValueError("stripe [%d, %d) of a %d-ring disk has fewer own rings than the %d ghost rings "
                                 "(%d stripes, cuts at multiples of %d rings)" % (lo, hi, nrad, ghost, nstripes, g))
    return parts


def _vp(t):
    return C.c_void_p(t.data_ptr())


class Stripe:
    """One stripe: its context, its block and its four halo buffers (device
    tensors on the stripe's GPU, used by the library on its stream)."""

    def __init__(self, params, planets, lo, hi, ghost=GHOST, device=0, radii=None, index=0, count=1):
        self.params, self.lo, self.hi, self.index, self.count = params, lo, hi, index, count
        ctx = C.c_void_p()
        rp = None if radii is None else np.ascontiguousarray(radii, np.float64).ctypes.data_as(
            C.POINTER(C.c_double))
        st = lib.fargo_stripe_create(C.byref(params), C.byref(planets), rp, lo, hi, ghost, device, C.byref(ctx))
        self.ctx = ctx
        if st != 0:
            msg = lib.fargo_last_error(ctx).decode() if ctx else ""
            if ctx:
                lib.fargo_destroy(ctx)
                self.ctx = None
            raise _abi.FargoError("fargo_stripe_create failed: %s %s" % (_abi.STATUS.get(st, st), msg))
        L = FargoStripeLayout()
        self._chk(lib.fargo_stripe_info(self.ctx, C.byref(L)), "fargo_stripe_info")
        self.layout = {k: getattr(L, k) for k, _ in FargoStripeLayout._fields_}
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(lib.fargo_stream(self.ctx), device=self.device)
        self.block_doubles = L.block_doubles
        self.block = None  # allocated by set_stride
        self.sg = bool(params.SelfGravity)
        self.sg_send = None  # allocated by set_sg_stride
        f32 = dict(dtype=torch.float32, device=self.device)
        self.send_lo = torch.zeros(max(1, L.halo_floats_lo), **f32)
        self.recv_lo = torch.zeros(max(1, L.halo_floats_lo), **f32)
        self.send_hi = torch.zeros(max(1, L.halo_floats_hi), **f32)
        self.recv_hi = torch.zeros(max(1, L.halo_floats_hi), **f32)

    def _chk(self, st, what):
        check(st, what, ctx=self.ctx)

    def set_stride(self, stride):
        self.stride = stride
        self.block = torch.zeros(stride, dtype=torch.float64, device=self.device)

    def set_sg_stride(self, stride):
        self.sg_send = torch.zeros(stride, dtype=torch.float32, device=self.device)

    # rows of the whole grid this stripe holds, and the ones it owns (the
    # outer stripe also owns the v_r row at NRAD)
    def local_rows(self):
        b = self.layout["base"]
        return b, b + self.layout["nrad"] + 1

    def own_rows(self):
        b, L = self.layout["base"], self.layout
        top = L["own_hi"] + (1 if self.hi == self.params.NRAD else 0)
        return b + L["own_lo"], b + top

    def init_state(self, dens=None, energy=None):
        """Whole-grid (NRAD+1, NSEC) arrays, or None for the profiles."""
        d = None if dens is None else np.ascontiguousarray(dens, np.float32).reshape(-1)
        e = None if energy is None else np.ascontiguousarray(energy, np.float32).reshape(-1)
        self._chk(lib.fargo_stripe_init_state(self.ctx, _fptr(d), _fptr(e)), "fargo_stripe_init_state")

    def upload(self, dens=None, vrad=None, vtheta=None, energy=None):
        a, b = self.local_rows()
        arr = [None if x is None else np.ascontiguousarray(np.asarray(x, np.float32)[a:b]).reshape(-1)
               for x in (dens, vrad, vtheta, energy)]
        self._chk(lib.fargo_upload(self.ctx, *[_fptr(x) for x in arr]), "fargo_upload")

    def own_fields(self):
        """{field: (rows, NSEC)} of the own rows; and their first whole-grid row."""
        n = (self.layout["nrad"] + 1) * self.layout["nsec"]
        out = {k: np.empty(n, np.float32) for k in ("dens", "vrad", "vtheta", "energy")}
        self._chk(lib.fargo_download(self.ctx, _fptr(out["dens"]), _fptr(out["vrad"]), _fptr(out["vtheta"]),
                                     _fptr(out["energy"]), None, None), "fargo_download")
        a, b = self.own_rows()
        base = self.layout["base"]
        return {k: v.reshape(-1, self.layout["nsec"])[a - base:b - base] for k, v in out.items()}, a

    # the per-substep operations (asynchronous on the stripe's stream, but more)
    def dt_begin(self):
        self._chk(lib.fargo_stripe_dt_begin(self.ctx), "fargo_stripe_dt_begin")

    def sg_rows(self):
        self._chk(lib.fargo_stripe_sg_rows(self.ctx, _vp(self.sg_send)), "fargo_stripe_sg_rows")

    def sg_apply(self, gathered, nstripe, stride, cuts):
        c = (C.c_int * len(cuts))(*cuts)
        self._chk(lib.fargo_stripe_sg_apply(self.ctx, _vp(gathered), nstripe, stride, c), "fargo_stripe_sg_apply")

    def forces(self):
        self._chk(lib.fargo_stripe_forces(self.ctx, _vp(self.block)), "fargo_stripe_forces")

    def substep(self, blocks, nstripe, stride):
        self._chk(lib.fargo_stripe_substep(self.ctx, _vp(blocks), nstripe, stride), "fargo_stripe_substep")

    def pack(self):
        self._chk(lib.fargo_stripe_halo_pack(self.ctx, _vp(self.send_lo), _vp(self.send_hi)),
                  "fargo_stripe_halo_pack")

    def unpack(self):
        self._chk(lib.fargo_stripe_halo_unpack(self.ctx, _vp(self.recv_lo), _vp(self.recv_hi)),
                  "fargo_stripe_halo_unpack")

    def more(self):
        m = C.c_int(0)
        self._chk(lib.fargo_stripe_more(self.ctx, C.byref(m)), "fargo_stripe_more")
        return m.value

    def scalars(self):
        s = _abi.FargoScalars()
        self._chk(lib.fargo_get_scalars(self.ctx, C.byref(s)), "fargo_get_scalars")
        return {k: getattr(s, k) for k, _ in _abi.FargoScalars._fields_}

    def planets(self):
        pl = _abi.FargoPlanets()
        self._chk(lib.fargo_get_planets(self.ctx, C.byref(pl)), "fargo_get_planets")
        return pl

    def close(self):
        if self.ctx:
            torch.cuda.synchronize(self.device)
            lib.fargo_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def drive_dt(stripes, xfer):
    """One DT of the stripes held by this process (all of them, or this
    rank's one); returns the substeps taken.  Every stripe takes the same
    substeps: they decide from the same gathered blocks."""
    for s in stripes:
        s.dt_begin()
    nsub = 0
    sg = getattr(stripes[0], "sg", False)
    while True:
        if sg:
            xfer.sg(stripes)
        for s in stripes:
            s.forces()
        blocks = xfer.gather(stripes)
        for s, blk in zip(stripes, blocks):
            s.substep(blk, xfer.nstripe, xfer.stride)
        for s in stripes:
            s.pack()
        more = {s.more() for s in stripes}
        if len(more) != 1:
            raise RuntimeError("stripes disagree on the substep count")
        xfer.halo(stripes)
        for s in stripes:
            s.unpack()
        nsub += 1
        if not more.pop():
            return nsub


class LocalExchange:
    """Every stripe in this process: blocks concatenated on each stripe's
    device, halos copied between neighbours (after the stripes' streams are
    drained)."""

    def __init__(self, stripes):
        self.nstripe = len(stripes)
        self.stride = max(s.block_doubles for s in stripes)
        for s in stripes:
            s.set_stride(self.stride)
        if getattr(stripes[0], "sg", False):
            nsec = stripes[0].params.NSEC
            self.cuts = [s.lo for s in stripes] + [stripes[-1].hi]
            self.sg_stride = max(s.hi - s.lo for s in stripes) * nsec
            for s in stripes:
                s.set_sg_stride(self.sg_stride)

    def sg(self, stripes):
        for s in stripes:
            s.sg_rows()
        self._drain(stripes)
        out, cache = [], {}
        for s in stripes:
            if s.device not in cache:
                cache[s.device] = torch.cat([t.sg_send.to(s.device) for t in stripes])
            out.append(cache[s.device])
        self._sync(stripes)
        for s, g in zip(stripes, out):
            s.sg_apply(g, self.nstripe, self.sg_stride, self.cuts)
        self._sg = out  # alive until the stripes' streams are drained

    @staticmethod
    def _drain(stripes):
        for s in stripes:
            if s.stream is not None:
                s.stream.synchronize()

    @staticmethod
    def _sync(stripes):
        for s in stripes:
            if s.device.type == "cuda":
                torch.cuda.synchronize(s.device)

    def gather(self, stripes):
        self._drain(stripes)
        out, cache = [], {}
        for s in stripes:
            if s.device not in cache:
                cache[s.device] = torch.cat([t.block.to(s.device) for t in stripes])
            out.append(cache[s.device])
        self._sync(stripes)
        self._blocks = out  # alive until the next gather
        return out

    def halo(self, stripes):
        self._drain(stripes)
        for a, b in zip(stripes[:-1], stripes[1:]):
            b.recv_lo.copy_(a.send_hi.to(b.device))
            a.recv_hi.copy_(b.send_lo.to(a.device))
        self._sync(stripes)


class DistExchange:
    """One stripe per rank of `group`: all-gather of the blocks, and
    send/recv of the halos with the ranks below and above.  The collectives
    are issued on the stripe's own stream (torch.cuda.ExternalStream), so
    that they follow its kernels and precede its next ones."""

    def __init__(self, stripes, group=None, parts=None):
        import torch.distributed as dist
        (s,) = stripes
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.nstripe = dist.get_world_size(group)
        dev = s.device if s.device.type == "cuda" else torch.device("cpu")
        m = torch.tensor([s.block_doubles], dtype=torch.int64, device=dev)
        dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
        self.stride = int(m.item())
        s.set_stride(self.stride)
        self.out = torch.zeros(self.nstripe * self.stride, dtype=torch.float64, device=s.block.device)
        if getattr(s, "sg", False):
            nsec = s.params.NSEC
            self.cuts = [lo for lo, _ in parts] + [parts[-1][1]]
            self.sg_stride = max(hi - lo for lo, hi in parts) * nsec
            s.set_sg_stride(self.sg_stride)
            self.sg_out = torch.zeros(self.nstripe * self.sg_stride, dtype=torch.float32, device=s.sg_send.device)

    def sg(self, stripes):
        (s,) = stripes
        s.sg_rows()
        with self._on(s):
            self.dist.all_gather(list(self.sg_out.split(self.sg_stride)), s.sg_send, group=self.group)
        s.sg_apply(self.sg_out, self.nstripe, self.sg_stride, self.cuts)

    def _on(self, s):
        return torch.cuda.stream(s.stream) if s.stream is not None else _Null()

    def gather(self, stripes):
        (s,) = stripes
        with self._on(s):
            parts = list(self.out.split(self.stride))
            self.dist.all_gather(parts, s.block, group=self.group)
        return [self.out]

    def halo(self, stripes):
        (s,) = stripes
        d, r, n = self.dist, self.rank, self.nstripe
        ops = []
        if r > 0:
            ops += [d.P2POp(d.isend, s.send_lo, d.get_global_rank(self.group, r - 1) if self.group else r - 1,
                            self.group),
                    d.P2POp(d.irecv, s.recv_lo, d.get_global_rank(self.group, r - 1) if self.group else r - 1,
                            self.group)]
        if r < n - 1:
            ops += [d.P2POp(d.isend, s.send_hi, d.get_global_rank(self.group, r + 1) if self.group else r + 1,
                            self.group),
                    d.P2POp(d.irecv, s.recv_hi, d.get_global_rank(self.group, r + 1) if self.group else r + 1,
                            self.group)]
        if ops:
            with self._on(s):
                for w in d.batch_isend_irecv(ops):
                    w.wait()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class _StripedDisk:
    def _setup(self):
        for s in self.stripes:
            s.pack()
        for s in self.stripes:
            s.stream.synchronize()
        self.xfer.halo(self.stripes)
        for s in self.stripes:
            s.unpack()

    def init_state(self, dens=None, energy=None):
        """Whole-grid (NRAD+1, NSEC) arrays, or None for the reference's
        profiles; then the ghost rings are exchanged once."""
        for s in self.stripes:
            s.init_state(dens, energy)
        self._setup()

    def upload(self, dens=None, vrad=None, vtheta=None, energy=None):
        for s in self.stripes:
            s.upload(dens, vrad, vtheta, energy)
        self._setup()

    def advance_dt(self):
        return drive_dt(self.stripes, self.xfer)

    def scalars(self):
        return self.stripes[0].scalars()

    def planets(self):
        return self.stripes[0].planets()

    def close(self):
        for s in self.stripes:
            s.close()


class LocalStripes(_StripedDisk):
    """A disk split into `nstripes` stripes held by this process, on
    `devices` (one per stripe; all on cuda:0 by default)."""

    def __init__(self, params, planets, nstripes, ghost=GHOST, devices=None, radii=None, parts=None):
        self.params = params
        self.parts = parts or partition(params.NRAD, params.NSEC, nstripes, ghost)
        devices = devices or [0] * len(self.parts)
        self.stripes = [Stripe(params, planets, lo, hi, ghost, dev, radii, k, len(self.parts))
                        for k, ((lo, hi), dev) in enumerate(zip(self.parts, devices))]
        self.xfer = LocalExchange(self.stripes)

    def fields(self):
        """Whole-grid {field: (NRAD+1, NSEC)} assembled from the own rows."""
        out = {k: np.zeros((self.params.NRAD + 1, self.params.NSEC), np.float32)
               for k in ("dens", "vrad", "vtheta", "energy")}
        for s in self.stripes:
            f, a = s.own_fields()
            for k, v in f.items():
                out[k][a:a + v.shape[0]] = v
        return out


class DistStripes(_StripedDisk):
    """This rank's stripe of a disk split over the ranks of `group` (one
    stripe per rank, on this rank's GPU)."""

    def __init__(self, params, planets, group=None, ghost=GHOST, device=None, radii=None, parts=None):
        import torch.distributed as dist
        self.params, self.group = params, group
        n, r = dist.get_world_size(group), dist.get_rank(group)
        self.parts = parts or partition(params.NRAD, params.NSEC, n, ghost)
        lo, hi = self.parts[r]
        if device is None:
            device = torch.cuda.current_device()
        self.stripes = [Stripe(params, planets, lo, hi, ghost, device, radii, r, n)]
        self.xfer = DistExchange(self.stripes, group, self.parts)

    def fields(self):
        """Whole-grid {field: (NRAD+1, NSEC)} on every rank (all-gather of
        the own rows, padded to the largest stripe)."""
        import torch.distributed as dist
        s = self.stripes[0]
        f, a = s.own_fields()
        nsec = self.params.NSEC
        rows = max(hi - lo for lo, hi in self.parts) + 1
        out = {}
        for k, v in f.items():
            buf = torch.zeros(rows, nsec, dtype=torch.float32, device=s.device)
            buf[:v.shape[0]] = torch.from_numpy(v).to(s.device)
            allb = [torch.empty_like(buf) for _ in self.parts]
            dist.all_gather(allb, buf, group=self.group)
            g = np.zeros((self.params.NRAD + 1, nsec), np.float32)
            for (lo, hi), t in zip(self.parts, allb):
                m = hi - lo + (1 if hi == self.params.NRAD else 0)
                g[lo:lo + m] = t[:m].cpu().numpy()
            out[k] = g
        return out
