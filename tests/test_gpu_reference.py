"""The CUDA path against the reference's own CUDA build.

Fixtures tests/golden/ref_*.npz come from the reference compiled from its
unmodified sources and run on a B200 with seeded noisy initial conditions
(tests/golden/make_ref_golden.py).  This library, initialised from the same
parameters and the same noise, must reproduce the reference's initial
fields, its substep counts, dt and FARGO shift counts exactly, its planet
orbits, and its fields after 10 DTs within REF_TOL, twice the rounding-order floor between two FP32 builds."""
import glob
import os

import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Disk, noise, planets_dict
from tests.golden import make_ref_golden as G
from oracle.oracle import Oracle, set_threads
from tests.helpers import REF_TOL, floor_tol, make, rel_l2

set_threads(os.cpu_count() or 1)
set_threads(os.cpu_count() or 1, "f32fma")

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))

# rel-L2 after 10 DTs.  Same compiler, same FP32 expressions and contraction
# as the reference; the only arithmetic differences are the FP64 (here) vs
# FP32 (reference) force sums and the summation order of those sums.
TOL = REF_TOL


@pytest.mark.skipif(not FIXTURES, reason="no reference fixtures")
@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_matches_reference(gpu, path):
    z = np.load(path)
    name = os.path.basename(path)[:-4]
    p, pl, seed, ndt = G.cases()[name]
    P, L, _ = make(dict(p, Ntot=str(ndt), Ninterm=str(ndt)), pl, name)
    d = Disk(P, L)
    if seed is not None:
        f = d.fields()
        d.init_state(dens=noise.perturb_density(f["dens"].reshape(-1), P.NRAD, P.NSEC, seed))
    nrad = P.NRAD
    f0 = d.fields(temperature=True)
    start = {k: v.copy() for k, v in d.fields().items()}
    for k in ("dens", "vrad", "vtheta", "energy"):
        if k + "0" in z:
            assert rel_l2(f0[k][:nrad], z[k + "0"]) <= 1e-7, k
    s = 0
    big = z["bigplanet"]
    for t in range(ndt):
        # bigplanet line t is written before AlgoGas(t): planet state after t DTs
        pd = planets_dict(d.planets())
        for k in range(pd["x"].size):
            assert abs(np.float32(pd["x"][k]) - big[k, t, 1]) <= 1e-6 * max(1.0, abs(big[k, t, 1]))
            assert abs(np.float32(pd["y"][k]) - big[k, t, 2]) <= 1e-6 * max(1.0, abs(big[k, t, 1]))
        n = d.advance_dt()
        ns, dt = d.substep_log()
        assert np.array_equal(ns, z["sub_nshift"][s:s + n]), "FARGO shift counts differ from the reference"
        assert np.array_equal(dt.astype(np.float32), z["sub_dt"][s:s + n].astype(np.float32))
        s += n
        # CircumPlanetaryMass after the DT (SourceEuler.cu:539-553): bigplanet
        # column 9 of the next line (Output.cu:85-86); FP64 sum here, the
        # reference's FP32 tree sum, of densities within REF_TOL
        want = big[0, t + 1, 9]
        assert abs(d.scalars()["mdcp1"] - want) <= 1e-4 * abs(want), (t, d.scalars()["mdcp1"], want)
    f1 = d.fields(temperature=True)
    tol = dict(TOL)
    if nrad * P.NSEC >= G.BIG:
        # the benchmark sizes: bound by this case's own rounding-order floor
        # between two FP32 builds, measured with the oracle (floor_tol)
        o = Oracle(P, L)
        o.set_fields(dens=start["dens"], vrad=start["vrad"], vtheta=start["vtheta"], energy=start["energy"])
        for _ in range(ndt):
            o.advance_dt()
        tol.update(floor_tol(P, L, start, ndt, o.fields()))
        tol["temperature"] = max(tol["temperature"], tol["dens"])
    errs = {}
    for k in TOL:
        if k + "1" in z:
            errs[k] = rel_l2(f1[k][:nrad], z[k + "1"])
    print("\nCUDA vs the reference's build %dx%d after %d DTs: %s" % (nrad, P.NSEC, ndt,
                                                                      {k: "%.2e" % e for k, e in errs.items()}))
    for k, e in errs.items():
        assert e <= tol[k], (k, e, errs, tol)
