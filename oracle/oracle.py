"""ctypes wrapper of the CPU oracle (fargo_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The product never uses it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


class FargoScalarsO(C.Structure):
    _fields_ = [("physical_time", C.c_float), ("omega_frame", C.c_float), ("mdcp1", C.c_float),
                ("lost_mass", C.c_float), ("nsub_last_dt", C.c_int), ("nsub_total", C.c_int),
                ("mass", C.c_double), ("angular_momentum", C.c_double), ("last_dt", C.c_double)]


_libs = {}


def _lib(prec):
    if prec in _libs:
        return _libs[prec]
    path = os.path.join(BUILD, "liboracle_%s.so" % prec)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    vp, fp, dp = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double)
    lib.orc_create.restype = C.c_int
    lib.orc_create.argtypes = [vp, vp, dp, C.POINTER(vp)]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_init_state.argtypes = [vp, fp, fp]
    lib.orc_set_fields_f32.argtypes = [vp, fp, fp, fp, fp]
    lib.orc_get_fields_f32.argtypes = [vp, fp, fp, fp, fp, fp, fp]
    lib.orc_set_fields.argtypes = [vp, vp, vp, vp, vp]
    lib.orc_get_fields.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    lib.orc_advance_dt.restype = C.c_int
    lib.orc_advance_dt.argtypes = [vp]
    lib.orc_substep_log.restype = C.c_int
    lib.orc_substep_log.argtypes = [vp, C.c_int, C.POINTER(C.c_int), dp]
    lib.orc_disk_force.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, dp]
    lib.orc_get_scalars.argtypes = [vp, C.POINTER(FargoScalarsO)]
    lib.orc_get_planets.argtypes = [vp, vp]
    lib.orc_set_planets.argtypes = [vp, vp]
    lib.orc_get_table.argtypes = [vp, C.c_int, dp]
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_set_precision.argtypes = [vp, C.c_int]
    lib.orc_sg_accelerations.restype = C.c_int
    lib.orc_sg_accelerations.argtypes = [vp, dp, dp]
    lib.orc_real_size.restype = C.c_int
    _libs[prec] = lib
    return lib


def set_threads(n, prec="f32"):
    _lib(prec).orc_set_threads(n)


class Oracle:
    """CPU restatement of one disk; prec 'f32' (reference typing), 'f64', or
    'f32fma' (the float build with a*b+c fused: a second FP32 build whose
    distance from 'f32' is the rounding-order floor)."""

    def __init__(self, params, planets, prec="f32", radii=None):
        self.lib = _lib(prec)
        self.prec = prec
        self.nrad, self.nsec = params.NRAD, params.NSEC
        self._params, self._planets = params, planets
        h = C.c_void_p()
        rp = None if radii is None else np.ascontiguousarray(radii, np.float64).ctypes.data_as(
            C.POINTER(C.c_double))
        st = self.lib.orc_create(C.addressof(params), C.addressof(planets), rp, C.byref(h))
        if st != 0:
            raise RuntimeError("orc_create failed")
        self.h = h

    @property
    def size_grid(self):
        return (self.nrad + 1) * self.nsec

    def init_state(self, dens=None, energy=None):
        """Re-run the initialisation with a perturbed density (as fargo_init_state)."""
        fp = C.POINTER(C.c_float)
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1) for a in (dens, energy)]
        self.lib.orc_init_state(self.h, *[None if a is None else a.ctypes.data_as(fp) for a in arrs])

    def set_fields(self, dens=None, vrad=None, vtheta=None, energy=None):
        fp = C.POINTER(C.c_float)
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1) for a in
                (dens, vrad, vtheta, energy)]
        self.lib.orc_set_fields_f32(self.h, *[None if a is None else a.ctypes.data_as(fp) for a in arrs])

    def set_fields_native(self, dens=None, vrad=None, vtheta=None, energy=None):
        dt = np.float32 if self.prec in ("f32", "f32fma") else np.float64
        arrs = [None if a is None else np.ascontiguousarray(a, dt).reshape(-1) for a in
                (dens, vrad, vtheta, energy)]
        self.lib.orc_set_fields(self.h, *[None if a is None else a.ctypes.data for a in arrs])

    def fields(self, native=False):
        n = self.size_grid
        dt = (np.float32 if self.prec in ("f32", "f32fma") else np.float64) if native else np.float32
        out = {k: np.empty(n, dt) for k in ("dens", "vrad", "vtheta", "energy", "temperature", "qplus")}
        if native:
            self.lib.orc_get_fields(self.h, *[out[k].ctypes.data for k in
                                              ("dens", "vrad", "vtheta", "energy", "temperature", "qplus")])
        else:
            fp = C.POINTER(C.c_float)
            self.lib.orc_get_fields_f32(self.h, *[out[k].ctypes.data_as(fp) for k in
                                                  ("dens", "vrad", "vtheta", "energy", "temperature", "qplus")])
        return {k: v.reshape(self.nrad + 1, self.nsec) for k, v in out.items()}

    def advance_dt(self):
        return self.lib.orc_advance_dt(self.h)

    def substep_log(self, cap=4096):
        ns = np.zeros(cap * self.nrad, np.int32)
        dt = np.zeros(cap, np.float64)
        n = self.lib.orc_substep_log(self.h, cap, ns.ctypes.data_as(C.POINTER(C.c_int)),
                                     dt.ctypes.data_as(C.POINTER(C.c_double)))
        k = min(n, cap)
        return ns[:k * self.nrad].reshape(k, self.nrad), dt[:k]

    def planets(self):
        pl = type(self._planets)()
        self.lib.orc_get_planets(self.h, C.addressof(pl))
        return pl

    def set_planets(self, pl):
        self.lib.orc_set_planets(self.h, C.addressof(pl))

    def scalars(self):
        s = FargoScalarsO()
        self.lib.orc_get_scalars(self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in FargoScalarsO._fields_}

    def disk_force(self, x, y, rs, mass, dimfxy=11):
        gf = np.zeros(4 * dimfxy, np.float64)
        self.lib.orc_disk_force(self.h, x, y, rs, mass, dimfxy, gf.ctypes.data_as(C.POINTER(C.c_double)))
        return gf

    def set_precision(self, mode):
        """0: the reference's arithmetic; 1: accurate mode."""
        self.lib.orc_set_precision(self.h, int(mode))

    def sg_accelerations(self):
        """(accr, acct) of the current density, each (NRAD, NSEC) float64."""
        n = self.nrad * self.nsec
        ar, at = np.zeros(n), np.zeros(n)
        st = self.lib.orc_sg_accelerations(self.h, ar.ctypes.data_as(C.POINTER(C.c_double)),
                                           at.ctypes.data_as(C.POINTER(C.c_double)))
        if st != 0:
            raise RuntimeError("no self-gravity in this run")
        return ar.reshape(self.nrad, self.nsec), at.reshape(self.nrad, self.nsec)

    def table(self, which):
        out = np.zeros(self.nrad + 1, np.float64)
        self.lib.orc_get_table(self.h, which, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
