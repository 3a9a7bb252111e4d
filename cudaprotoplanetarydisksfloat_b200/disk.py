"""Host-side interface of the library: one disk (Disk) or many (Batch).

Mirrors the reference's run structure: parameters come from a .par file
(ReadVariables), planets from a .cfg (InitPlanetarySystem), then each
advance_dt() is one AlgoGas call.  All computation happens on the GPU through
the C ABI; this module only moves host buffers.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._abi import FargoParams, FargoPlanets, FargoScalars, check, lib

_fp = C.POINTER(C.c_float)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_fp)


def read_params(par_path):
    p = FargoParams()
    check(lib.fargo_params_read(par_path.encode(), C.byref(p)), "fargo_params_read(%s)" % par_path)
    return p


def read_planets(cfg_path, params):
    pl = FargoPlanets()
    check(lib.fargo_planets_read(cfg_path.encode(), C.byref(params), C.byref(pl)),
          "fargo_planets_read(%s)" % cfg_path)
    return pl


def grid_radii(params):
    r = np.zeros(params.NRAD + 1, dtype=np.float64)
    check(lib.fargo_grid_radii(C.byref(params), r.ctypes.data_as(C.POINTER(C.c_double))), "fargo_grid_radii")
    return r


def planets_dict(pl):
    n = pl.nb
    return {k: np.array(getattr(pl, k)[:n]) for k in ("mass", "x", "y", "vx", "vy")}


class Disk:
    """One disk on one GPU."""

    def __init__(self, params, planets, device=0, radii=None):
        self.params = params
        self.nrad, self.nsec = params.NRAD, params.NSEC
        ctx = C.c_void_p()
        rp = None if radii is None else np.ascontiguousarray(radii, np.float64).ctypes.data_as(
            C.POINTER(C.c_double))
        st = lib.fargo_create(C.byref(params), C.byref(planets), rp, device, C.byref(ctx))
        self.ctx = ctx
        if st != 0:
            msg = lib.fargo_last_error(ctx).decode() if ctx else ""
            if ctx:
                lib.fargo_destroy(ctx)
                self.ctx = None
            raise _abi.FargoError("fargo_create failed: %s %s" % (_abi.STATUS.get(st, st), msg))

    @classmethod
    def from_par(cls, par_path, cfg_path=None, device=0):
        p = read_params(par_path)
        pl = read_planets(cfg_path or p.PLANETCONFIG.decode(), p)
        return cls(p, pl, device=device)

    @property
    def size_grid(self):
        return (self.nrad + 1) * self.nsec

    def _chk(self, st, what):
        check(st, what, ctx=self.ctx)

    def init_state(self, dens=None, energy=None):
        d = None if dens is None else np.ascontiguousarray(dens, np.float32).reshape(-1)
        e = None if energy is None else np.ascontiguousarray(energy, np.float32).reshape(-1)
        self._chk(lib.fargo_init_state(self.ctx, _ptr(d), _ptr(e)), "fargo_init_state")

    def upload(self, dens=None, vrad=None, vtheta=None, energy=None):
        a = [None if x is None else np.ascontiguousarray(x, np.float32).reshape(-1)
             for x in (dens, vrad, vtheta, energy)]
        self._chk(lib.fargo_upload(self.ctx, *[_ptr(x) for x in a]), "fargo_upload")

    def fields(self, temperature=False, qplus=False):
        n = self.size_grid
        out = {k: np.empty(n, np.float32) for k in ("dens", "vrad", "vtheta", "energy")}
        t = np.empty(n, np.float32) if temperature else None
        q = np.empty(n, np.float32) if qplus else None
        self._chk(lib.fargo_download(self.ctx, _ptr(out["dens"]), _ptr(out["vrad"]), _ptr(out["vtheta"]),
                                     _ptr(out["energy"]), _ptr(t), _ptr(q)), "fargo_download")
        if temperature:
            out["temperature"] = t
        if qplus:
            out["qplus"] = q
        return {k: v.reshape(self.nrad + 1, self.nsec) for k, v in out.items()}

    def advance_dt(self):
        n = C.c_int(0)
        self._chk(lib.fargo_advance_dt(self.ctx, C.byref(n)), "fargo_advance_dt")
        return n.value

    def advance(self, ndt):
        self._chk(lib.fargo_advance(self.ctx, ndt), "fargo_advance")

    def advance_async(self, ndt):
        self._chk(lib.fargo_advance_async(self.ctx, ndt), "fargo_advance_async")

    def sync(self):
        self._chk(lib.fargo_sync(self.ctx), "fargo_sync")

    def planets(self):
        pl = FargoPlanets()
        self._chk(lib.fargo_get_planets(self.ctx, C.byref(pl)), "fargo_get_planets")
        return pl

    def set_planets(self, pl):
        self._chk(lib.fargo_set_planets(self.ctx, C.byref(pl)), "fargo_set_planets")

    def scalars(self):
        s = FargoScalars()
        self._chk(lib.fargo_get_scalars(self.ctx, C.byref(s)), "fargo_get_scalars")
        return {k: getattr(s, k) for k, _ in FargoScalars._fields_}

    def substep_log(self, cap=2048):
        ns = np.zeros(cap * self.nrad, np.int32)
        dt = np.zeros(cap, np.float64)
        n = C.c_int(0)
        self._chk(lib.fargo_get_substep_log(self.ctx, cap, ns.ctypes.data_as(C.POINTER(C.c_int)),
                                            dt.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)),
                  "fargo_get_substep_log")
        k = min(n.value, cap)
        return ns[:k * self.nrad].reshape(k, self.nrad), dt[:k]

    def disk_force(self, x, y, rsmoothing, mass):
        gf = np.zeros(4 * _abi.FARGO_DIMFXY, np.float64)
        self._chk(lib.fargo_disk_force(self.ctx, x, y, rsmoothing, mass, _abi.FARGO_DIMFXY,
                                       gf.ctypes.data_as(C.POINTER(C.c_double))), "fargo_disk_force")
        return gf

    def sg_accelerations(self):
        """(accr, acct), each (NRAD, NSEC) float32: the self-gravity
        accelerations of the current density (between DTs)."""
        n = self.nrad * self.nsec
        ar, at = np.empty(n, np.float32), np.empty(n, np.float32)
        self._chk(lib.fargo_sg_accelerations(self.ctx, _ptr(ar), _ptr(at)), "fargo_sg_accelerations")
        return ar.reshape(self.nrad, self.nsec), at.reshape(self.nrad, self.nsec)

    def set_graph_mode(self, on):
        self._chk(lib.fargo_set_graph_mode(self.ctx, 1 if on else 0), "fargo_set_graph_mode")

    def set_max_substeps(self, n):
        """Substeps one DT may take before it stops with FARGO_ETIMEOUT."""
        self._chk(lib.fargo_set_max_substeps(self.ctx, n), "fargo_set_max_substeps")

    def set_precision(self, mode):
        """0 (FARGO_PRECISION_REFERENCE): the reference's arithmetic;
        1 (FARGO_PRECISION_ACCURATE): closer to FP64 (see the header)."""
        self._chk(lib.fargo_set_precision(self.ctx, int(mode)), "fargo_set_precision")

    def autotune(self, reps=3):
        """Pick the transport segment width by timing (between DTs); returns it."""
        seg = C.c_int(0)
        self._chk(lib.fargo_autotune(self.ctx, reps, C.byref(seg)), "fargo_autotune")
        return seg.value

    def checkpoint(self):
        """The device state as bytes (between DTs)."""
        n = lib.fargo_checkpoint_bytes(self.ctx)
        buf = C.create_string_buffer(n)
        self._chk(lib.fargo_checkpoint_save(self.ctx, buf, n), "fargo_checkpoint_save")
        return buf.raw

    def restore(self, data):
        """Load a state saved by checkpoint()."""
        buf = C.create_string_buffer(data, len(data))
        self._chk(lib.fargo_checkpoint_load(self.ctx, buf, len(data)), "fargo_checkpoint_load")

    def close(self):
        if self.ctx:
            lib.fargo_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent disks advanced together (one launch per kernel)."""

    def __init__(self, params_list, planets_list, device=0):
        n = len(params_list)
        P = (FargoParams * n)(*params_list)
        L = (FargoPlanets * n)(*planets_list)
        b = C.c_void_p()
        st = lib.fargo_batch_create(n, P, L, device, C.byref(b))
        self.b = b
        self.n = n
        self.shapes = [(p.NRAD, p.NSEC) for p in params_list]
        if st != 0:
            msg = lib.fargo_batch_last_error(b).decode() if b else ""
            if b:
                lib.fargo_batch_destroy(b)
                self.b = None
            raise _abi.FargoError("fargo_batch_create failed: %s %s" % (_abi.STATUS.get(st, st), msg))

    def _chk(self, st, what):
        check(st, what, batch=self.b)

    def init_state(self, disk, dens=None, energy=None):
        d = None if dens is None else np.ascontiguousarray(dens, np.float32).reshape(-1)
        e = None if energy is None else np.ascontiguousarray(energy, np.float32).reshape(-1)
        self._chk(lib.fargo_batch_init_state(self.b, disk, _ptr(d), _ptr(e)), "fargo_batch_init_state")

    def fields(self, disk):
        nrad, nsec = self.shapes[disk]
        n = (nrad + 1) * nsec
        out = {k: np.empty(n, np.float32) for k in ("dens", "vrad", "vtheta", "energy")}
        self._chk(lib.fargo_batch_download(self.b, disk, _ptr(out["dens"]), _ptr(out["vrad"]),
                                           _ptr(out["vtheta"]), _ptr(out["energy"])), "fargo_batch_download")
        return {k: v.reshape(nrad + 1, nsec) for k, v in out.items()}

    def upload(self, disk, dens=None, vrad=None, vtheta=None, energy=None):
        a = [None if x is None else np.ascontiguousarray(x, np.float32).reshape(-1)
             for x in (dens, vrad, vtheta, energy)]
        self._chk(lib.fargo_batch_upload(self.b, disk, *[_ptr(x) for x in a]), "fargo_batch_upload")

    def advance(self, ndt):
        self._chk(lib.fargo_batch_advance(self.b, ndt), "fargo_batch_advance")

    def advance_async(self, ndt):
        self._chk(lib.fargo_batch_advance_async(self.b, ndt), "fargo_batch_advance_async")

    def set_graph_mode(self, on):
        self._chk(lib.fargo_batch_set_graph_mode(self.b, 1 if on else 0), "fargo_batch_set_graph_mode")

    def set_precision(self, mode):
        self._chk(lib.fargo_batch_set_precision(self.b, int(mode)), "fargo_batch_set_precision")

    def autotune(self, reps=3):
        """Pick the transport segment width by timing (between DTs); returns it."""
        seg = C.c_int(0)
        self._chk(lib.fargo_batch_autotune(self.b, reps, C.byref(seg)), "fargo_batch_autotune")
        return seg.value

    def segments(self):
        """The transport segment width of each disk (autotuned per class)."""
        out = (C.c_int * self.n)()
        self._chk(lib.fargo_batch_segments(self.b, self.n, out), "fargo_batch_segments")
        return list(out)

    def sync(self):
        self._chk(lib.fargo_batch_sync(self.b), "fargo_batch_sync")

    def scalars(self, disk):
        s = FargoScalars()
        self._chk(lib.fargo_batch_get_scalars(self.b, disk, C.byref(s)), "fargo_batch_get_scalars")
        return {k: getattr(s, k) for k, _ in FargoScalars._fields_}

    def planets(self, disk):
        pl = FargoPlanets()
        self._chk(lib.fargo_batch_get_planets(self.b, disk, C.byref(pl)), "fargo_batch_get_planets")
        return pl

    def launches(self):
        return lib.fargo_batch_count_launches(self.b)

    def close(self):
        if self.b:
            lib.fargo_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
