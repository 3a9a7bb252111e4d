"""Shared helpers of the test-suite (the oracle is the checker)."""
import os
import tempfile

import numpy as np

from cudaprotoplanetarydisksfloat_b200 import configs, read_params, read_planets

SEED = 20261203

# Relative-L2 bounds on the fields after 10 DTs.
#
# FIELD_TOL: the CUDA path against the oracle (the CPU restatement of the
# reference's algorithm, with the reference's expression typing and no
# contraction of a*b+c into fused multiply-adds).  Measured on the parity
# cases (32x64 .. 128x384, 5-10 DTs): Sigma <= 8.1e-6, v_r <= 1.8e-4,
# v_theta <= 5.7e-7, energy <= 1.3e-5.
#
# REF_TOL: anything against the reference's own build (its fixtures and its
# output files).  That build contracts a*b+c into fused multiply-adds where
# its compiler chooses, and sits Sigma 1.03e-5, v_r 1.2e-4, v_theta 5e-7,
# energy 1.8e-5 from the oracle on the golden cases: the rounding-order floor
# between two FP32 builds of the same algorithm (the oracle built with and
# without contraction differs by the same amounts), so the bound is twice it.
# The reference algorithm's FP32-vs-FP64 gap is larger (Sigma 1.2-1.9e-5,
# v_r 1.6-1.9e-4 after 5 DTs).  v_r is a near-zero field (|v_r| ~ 3e-3
# |v_theta|), hence its larger relative bound.  The integer outcomes of the
# step (substep count, every substep's dt, every ring's FARGO shift) are
# compared exactly in both cases.
FIELD_TOL = {"dens": 1e-5, "vrad": 2.5e-4, "vtheta": 1e-6, "energy": 2e-5, "temperature": 1e-5}
REF_TOL = {"dens": 2e-5, "vrad": 3e-4, "vtheta": 2e-6, "energy": 4e-5, "temperature": 2e-5}


def planet_err(a, b):
    """Largest difference of a planet quantity, relative to its scale."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def make(params, planets, name="t"):
    d = tempfile.mkdtemp(prefix="fargo_%s_" % name)
    par, cfg, out = configs.materialise(params, planets, d, name)
    P = read_params(par)
    L = read_planets(cfg, P)
    return P, L, d


def small(kind, nrad=32, nsec=96, **over):
    p, pl = configs.small(kind, nrad, nsec)
    p = dict(p, **over)
    return make(p, pl, kind)


def floor_tol(P, L, start, ndt, f32_after, keys=("dens", "vrad", "vtheta", "energy"), precision=0):
    """Field tolerances of one case, scaled by its own rounding-order floor.

    REF_TOL was measured on the small grids; on other physics (the C4
    sweep's thin, low-alpha disks, C5's first substeps, where v_r is still
    near zero) two FP32 builds of the same algorithm drift further apart.
    The floor is measured live: the oracle's FMA-contracted build advanced
    `ndt` DTs from the same `start` fields as the plain float build, whose
    result is `f32_after`.  tol[k] = max(REF_TOL[k], 2 * rel_l2(fma, f32))."""
    from oracle.oracle import Oracle
    o = Oracle(P, L, "f32fma")
    if precision:
        o.set_precision(precision)
    o.set_fields(dens=start["dens"], vrad=start["vrad"], vtheta=start["vtheta"], energy=start["energy"])
    for _ in range(ndt):
        o.advance_dt()
    g = o.fields()
    o.close()
    nrad = P.NRAD
    tol = {}
    for k in keys:
        fl = rel_l2(g[k][:nrad], f32_after[k][:nrad]) if np.any(f32_after[k][:nrad]) else 0.0
        tol[k] = max(REF_TOL[k], 2.0 * fl)
    return tol
