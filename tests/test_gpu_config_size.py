"""The benchmark configurations at their own sizes, on the GPU.

- C3 (512x1024, self-gravity): the accelerations of the CUDA path (cuFFT in
  FP32) against the FP64 oracle's (FP64 DFT) in both precision modes, and
  one DT against the FP32 oracle (integer outcomes exact, fields within
  FIELD_TOL).
- C4: four disks of the 64-disk sweep, the 512x1536 one among them, batched
  give the same bits as each disk alone, and the batch matches the oracle
  disk by disk after 2 DTs.
- C5 (2048x6144, adiabatic, self-gravity, three live planets): the grid and
  physics of C5 with DT shortened to 0.002 (two substeps): the CPU oracle
  takes ~10 s per C5 substep on 16 host cores, and a standard C5 DT of
  0.314 is ~190 substeps.  Against the FP32 oracle: substep count, dt and
  every Nshift exact, fields within tolerance; against the FP64 oracle: the
  per-field error is reported and may not exceed 1.5 times the FP32
  oracle's own distance from FP64 (plus the FP32 tolerance).

Field tolerances at these sizes are FIELD_TOL or, where the case's own
rounding-order floor is wider, twice the measured distance between the
oracle's plain and FMA-contracted FP32 builds (tests/helpers.py floor_tol):
on the sweep's thin, low-alpha disks and in C5's first substeps, where v_r
is still near zero, two FP32 builds of the same algorithm differ by up to
~6e-4 in v_r.

C2 (256x768) and the 512x1536 disk are also checked against the reference's
own build, through the fixtures of test_gpu_reference.py."""
import os

import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Batch, Disk, configs, noise, planets_dict
from oracle.oracle import Oracle, set_threads
from tests.helpers import FIELD_TOL, SEED, floor_tol, make, planet_err, rel_l2

pytestmark = pytest.mark.gpu

CORES = os.cpu_count() or 1


def _noisy_disk(p, pl, name, seed=SEED):
    P, L, _ = make(p, pl, name)
    d = Disk(P, L)
    f0 = d.fields()
    d.init_state(dens=noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, seed))
    return P, L, d


def _oracle_from(P, L, d, prec="f32"):
    for pr in (prec, "f32fma"):
        set_threads(CORES, pr)
    o = Oracle(P, L, prec)
    g = d.fields()
    o.set_fields(dens=g["dens"], vrad=g["vrad"], vtheta=g["vtheta"], energy=g["energy"])
    return o


def _exact_step(d, o):
    n1, n2 = d.advance_dt(), o.advance_dt()
    assert n1 == n2
    ns1, dt1 = d.substep_log()
    ns2, dt2 = o.substep_log()
    assert np.array_equal(ns1, ns2), "FARGO shift counts differ"
    assert np.array_equal(dt1, dt2), "substep dt differ"
    return n1


@pytest.mark.parametrize("mode", [0, 1], ids=["reference", "accurate"])
def test_c3_sg_accelerations_vs_fp64(gpu, mode):
    p, pl = configs.c3()
    P, L, d = _noisy_disk(p, pl, "c3acc")
    d.set_precision(mode)
    o64 = _oracle_from(P, L, d, "f64")
    ar, at = d.sg_accelerations()
    wr, wt = o64.sg_accelerations()
    er, et = rel_l2(ar, wr), rel_l2(at, wt)
    print("\nC3 self-gravity (%s mode), CUDA (cuFFT FP32) vs FP64 oracle: rel-L2 g_r %.2e, g_phi %.2e"
          % (["reference", "accurate"][mode], er, et))
    # g_r: the FP32 floor of the reference's method (~1e-5).  g_phi of a
    # near-axisymmetric disk is a small residual driven by the 1e-3 noise:
    # with the reference's float kernel table part of the axisymmetric
    # density leaks into it (5% at this size); the FP64 table of the
    # accurate mode removes that part, leaving the FP32 FFT's rounding.
    # measured: reference mode g_r 7.3e-6, g_phi 5.0e-2; accurate mode g_r
    # 2.0e-7, g_phi 1.4e-4
    assert er <= (3e-5 if mode == 0 else 1e-6)
    assert et <= (0.1 if mode == 0 else 1e-3)
    d.close()


def test_c3_one_dt_parity(gpu):
    p, pl = configs.c3()
    P, L, d = _noisy_disk(p, pl, "c3dt")
    o = _oracle_from(P, L, d)
    _exact_step(d, o)
    a, b = d.fields(), o.fields()
    errs = {k: rel_l2(a[k][:P.NRAD], b[k][:P.NRAD]) for k in ("dens", "vrad", "vtheta")}
    print("\nC3 one DT, CUDA vs oracle: %s" % {k: "%.2e" % e for k, e in errs.items()})
    for k, e in errs.items():
        assert e <= FIELD_TOL[k], (k, e)
    pa, pb = planets_dict(d.planets()), planets_dict(o.planets())
    for k in ("x", "y"):
        assert planet_err(pa[k], pb[k]) <= 1e-5
    d.close()


def test_c4_real_disks_batched_equal_single_and_oracle(gpu, tmp_path):
    sweep = configs.c4(64, seed=42)
    pick = []
    for nrad in (128, 256, 384, 512):
        pick.append(next(k for k, (p, _) in enumerate(sweep) if int(p["Nrad"]) == nrad))
    built = [make(sweep[k][0], sweep[k][1], "c4d%02d" % k) for k in pick]
    P = [b[0] for b in built]
    L = [b[1] for b in built]
    batch = Batch(P, L)
    singles = [Disk(p, l) for p, l in zip(P, L)]
    oracles, starts = [], []
    for i, (k, p, s) in enumerate(zip(pick, P, singles)):
        f = s.fields()
        dens = noise.perturb_density(f["dens"].reshape(-1), p.NRAD, p.NSEC, SEED + k)
        s.init_state(dens=dens)
        batch.init_state(i, dens=dens)
        starts.append(s.fields())
        oracles.append(_oracle_from(p, L[i], s))
    batch.advance(2)
    for s in singles:
        s.advance(2)
    for o in oracles:
        for _ in range(2):
            o.advance_dt()
    for i, (p, s, o) in enumerate(zip(P, singles, oracles)):
        a, b = batch.fields(i), s.fields()
        for key in ("dens", "vrad", "vtheta"):
            assert np.array_equal(a[key], b[key]), (pick[i], key)
        c = o.fields()
        tol = floor_tol(p, L[i], starts[i], 2, c, keys=("dens", "vrad", "vtheta"))
        for key in ("dens", "vrad", "vtheta"):
            e = rel_l2(a[key][:p.NRAD], c[key][:p.NRAD])
            assert e <= tol[key], (pick[i], key, e, tol[key])
        assert batch.scalars(i)["nsub_total"] == o.scalars()["nsub_total"]
    batch.close()


def test_c5_short_dt_vs_fp32_and_fp64(gpu):
    p, pl = configs.c5()
    p = dict(p, DT="0.002")
    P, L, d = _noisy_disk(p, pl, "c5")
    start = d.fields()
    o32 = _oracle_from(P, L, d, "f32")
    n = _exact_step(d, o32)
    a, b = d.fields(), o32.fields()
    keys = ("dens", "vrad", "vtheta", "energy")
    tol = floor_tol(P, L, start, 1, b, keys=keys)
    for k in keys:
        e = rel_l2(a[k][:P.NRAD], b[k][:P.NRAD])
        assert e <= tol[k], (k, e, tol[k])
    # the same start against the FP64 oracle: the CUDA path may be no
    # further from it than the FP32 oracle is
    o64 = _oracle_from(P, L, d, "f64")
    o64.set_fields(dens=start["dens"], vrad=start["vrad"], vtheta=start["vtheta"], energy=start["energy"])
    assert o64.advance_dt() == n
    c = o64.fields()
    errs = {k: rel_l2(a[k][:P.NRAD], c[k][:P.NRAD]) for k in keys}
    gap = {k: rel_l2(b[k][:P.NRAD], c[k][:P.NRAD]) for k in keys}
    pa, pb = planets_dict(d.planets()), planets_dict(o64.planets())
    perr = max(planet_err(pa[k], pb[k]) for k in ("x", "y", "vx", "vy"))
    print("\nC5 (%d substeps) vs FP64 oracle: CUDA %s; FP32 oracle %s; planets %.1e" % (
        n, ", ".join("%s %.2e" % kv for kv in errs.items()), ", ".join("%s %.2e" % kv for kv in gap.items()), perr))
    for k in keys:
        assert errs[k] <= 1.5 * gap[k] + tol[k], (k, errs[k], gap[k])
    assert perr <= 1e-6
    o32.close()
    o64.close()
    d.close()
