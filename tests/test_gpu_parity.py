"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Same seeded inputs, small grids that the oracle finishes in seconds:
substep counts, every substep's dt and every ring's FARGO shift count
exact; fields within FIELD_TOL (tests/helpers.py, the measured rounding-order
floor between two FP32 builds); planets bit-for-bit up to 1e-9 when they do
not feel the disk, within 1e-6 of their scale when they do (their kick sums
per-cell FP32 forces that differ at the rounding floor) and 1e-5 with self
gravity (cuFFT FP32 transforms here, an FP64 DFT in the oracle).  The oracle
starts from the state the GPU initialised, so the step is compared alone;
test_init_parity compares the initialisation."""
import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Batch, Disk, noise, planets_dict
from oracle.oracle import Oracle
from tests.helpers import FIELD_TOL, SEED, planet_err, rel_l2, small

pytestmark = pytest.mark.gpu

TOL = FIELD_TOL


def _pair(kind, nrad, nsec, seed=SEED, **over):
    P, L, _ = small(kind, nrad, nsec, **over)
    d = Disk(P, L)
    f0 = d.fields()
    dens = noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, seed)
    d.init_state(dens=dens)
    g = d.fields()
    o = Oracle(P, L)
    o.set_fields(dens=g["dens"], vrad=g["vrad"], vtheta=g["vtheta"], energy=g["energy"])
    return P, L, d, o, dens


def _compare(P, d, o, ndt, fields=("dens", "vrad", "vtheta"), tol=TOL, scale=1.0, planet_rtol=1e-9):
    for _ in range(ndt):
        n1 = d.advance_dt()
        n2 = o.advance_dt()
        assert n1 == n2
        ns1, dt1 = d.substep_log()
        ns2, dt2 = o.substep_log()
        assert np.array_equal(ns1, ns2), "FARGO shift counts differ"
        assert np.array_equal(dt1, dt2), "substep dt differ"
    a, b = d.fields(), o.fields()
    errs = {k: rel_l2(a[k][:P.NRAD], b[k][:P.NRAD]) for k in fields}
    print("\nCUDA vs oracle %dx%d after %d DTs: %s" % (P.NRAD, P.NSEC, ndt,
                                                      {k: "%.2e" % e for k, e in errs.items()}))
    for k, e in errs.items():
        assert e <= tol[k] * scale, (k, e, errs)
    pa, pb = planets_dict(d.planets()), planets_dict(o.planets())
    for k in ("x", "y", "vx", "vy"):
        assert planet_err(pa[k], pb[k]) <= planet_rtol, (k, pa[k], pb[k])
    # CircumPlanetaryMass of planet 0 (SourceEuler.cu:539-553), both summed in FP64
    if pa["x"].size:
        m1, m2 = d.scalars()["mdcp1"], o.scalars()["mdcp1"]
        assert abs(m1 - m2) <= 1e-4 * abs(m2) + 1e-30, (m1, m2)
    return errs


@pytest.mark.parametrize("nrad,nsec,ndt", [(32, 96, 10), (48, 130, 10), (128, 384, 5)])
def test_isothermal_step_parity(gpu, nrad, nsec, ndt):
    P, L, d, o, _ = _pair("iso", nrad, nsec)
    _compare(P, d, o, ndt)


# NSEC 126 is not a multiple of 4: the cell kernels' per-cell path and the
# transport's 4-byte row staging
@pytest.mark.parametrize("nrad,nsec", [(32, 96), (64, 192), (40, 126)])
def test_adiabatic_two_live_planets_parity(gpu, nrad, nsec):
    P, L, d, o, _ = _pair("adi", nrad, nsec)
    _compare(P, d, o, 10, fields=("dens", "vrad", "vtheta", "energy"), planet_rtol=1e-6)


def test_standard_transport_and_exclude_hill(gpu):
    P, L, d, o, _ = _pair("iso", 32, 96, Transport="STANDARD", ExcludeHill="YES", ForcedCircular="NO")
    _compare(P, d, o, 5, planet_rtol=1e-6)


def test_cooling_branch(gpu):
    P, L, d, o, _ = _pair("adi", 32, 96, Cooling="YES", CoolingTime0="31.4")
    _compare(P, d, o, 5, fields=("dens", "vrad", "vtheta", "energy"), planet_rtol=1e-6)


def test_self_gravity_parity(gpu):
    # the FFT is FP32 (cuFFT) here and FP64 in the oracle
    P, L, d, o, _ = _pair("sg", 32, 64)
    _compare(P, d, o, 5, planet_rtol=1e-5)


# Non-rigid boundaries (ApplyBoundaryCondition, called three times per
# substep).  NONREFLECTING on an adiabatic disk with alpha viscosity also
# refreshes the sound speed and the viscosity at every call; EVANESCENT in a
# corotating frame meets CorrectVtheta; OPEN accumulates the mass lost
# through the inner edge.
def test_nonreflecting_adiabatic_alpha_parity(gpu):
    P, L, d, o, _ = _pair("adi", 48, 160, InnerBoundary="NONREFLECTING")
    _compare(P, d, o, 10, fields=("dens", "vrad", "vtheta", "energy"), planet_rtol=1e-6)


def test_nonreflecting_isothermal_parity(gpu):
    P, L, d, o, _ = _pair("iso", 48, 160, InnerBoundary="NONREFLECTING")
    _compare(P, d, o, 10)


def test_evanescent_corotating_parity(gpu):
    P, L, d, o, _ = _pair("adi", 48, 160, InnerBoundary="EVANESCENT", Frame="COROTATING")
    _compare(P, d, o, 10, fields=("dens", "vrad", "vtheta", "energy"), planet_rtol=1e-6)


def test_open_boundary_parity_and_lost_mass(gpu):
    # Sigma rising outwards: ring 1 sits above SigmaMed[0], so the open edge lets gas out
    P, L, d, o, _ = _pair("iso", 48, 160, InnerBoundary="OPEN", SigmaSlope="-0.5")
    _compare(P, d, o, 10)
    # LostMass integrates the density flux through the inner edge, i.e. v_r on
    # the first rings, where the rounding-order differences of v_r are largest
    # (the field bound is 3e-4 in rel-L2 over the whole grid)
    a, b = d.scalars()["lost_mass"], o.scalars()["lost_mass"]
    assert b != 0.0
    assert abs(a - b) <= 2e-3 * abs(b), (a, b)


def test_nonreflecting_rejects_narrow_grid(gpu):
    P, L, _ = small("adi", 32, 96, InnerBoundary="NONREFLECTING")
    with pytest.raises(Exception, match="NSEC > 128"):
        Disk(P, L)


def test_init_parity(gpu):
    """GPU initialisation (device sound speed and velocities) vs the oracle's."""
    for kind in ("iso", "adi"):
        P, L, _ = small(kind, 32, 96)
        d = Disk(P, L)
        o = Oracle(P, L)
        a, b = d.fields(), o.fields()
        for k in ("dens", "vrad", "vtheta", "energy"):
            assert rel_l2(a[k][:P.NRAD], b[k][:P.NRAD]) <= 1e-6, (kind, k)


def test_disk_force_matches_oracle(gpu):
    P, L, d, o, _ = _pair("iso", 48, 130)
    d.advance_dt()
    o.advance_dt()
    a = d.disk_force(1.0, 0.01, 0.03, 1e-3)
    b = o.disk_force(1.0, 0.01, 0.03, 1e-3)
    assert rel_l2(a, b) <= 1e-6
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6 * np.abs(b).max())


def test_batched_equals_single(gpu):
    """A batch of uneven disks of every kind (isothermal, adiabatic, each with
    and without self-gravity: one Substep1 instance per kind) gives the same
    bits as each disk alone."""
    cases = [("iso", 32, 96), ("iso", 48, 144), ("adi", 40, 120), ("sg", 32, 64), ("adisg", 32, 64)]
    built = [small(k, nr, ns) for k, nr, ns in cases]
    P = [b[0] for b in built]
    L = [b[1] for b in built]
    batch = Batch(P, L)
    singles = [Disk(p, l) for p, l in zip(P, L)]
    for i, (p, s) in enumerate(zip(P, singles)):
        f = s.fields()
        dens = noise.perturb_density(f["dens"].reshape(-1), p.NRAD, p.NSEC, SEED + i)
        s.init_state(dens=dens)
        batch.init_state(i, dens=dens)
    batch.advance(4)
    for s in singles:
        s.advance(4)
    for i, s in enumerate(singles):
        a, b = batch.fields(i), s.fields()
        for k in ("dens", "vrad", "vtheta", "energy"):
            assert np.array_equal(a[k], b[k]), (i, k)


def test_graph_and_host_loop_identical(gpu):
    P, L, d1, _, dens = _pair("iso", 32, 96)
    P2, L2, d2, _, _ = _pair("iso", 32, 96)
    d2.set_graph_mode(False)
    d1.advance(3)
    d2.advance(3)
    a, b = d1.fields(), d2.fields()
    for k in ("dens", "vrad", "vtheta"):
        assert np.array_equal(a[k], b[k])


def test_deterministic(gpu):
    P, L, d1, _, _ = _pair("adi", 32, 96)
    _, _, d2, _, _ = _pair("adi", 32, 96)
    d1.advance(3)
    d2.advance(3)
    a, b = d1.fields(), d2.fields()
    for k in ("dens", "vrad", "vtheta", "energy"):
        assert np.array_equal(a[k], b[k])


def test_autotune_keeps_results(gpu):
    # the segment width only regroups the transport's work: the result of
    # every cell is the same, bit for bit, whatever width the tuner picks
    P, L, d1, _, _ = _pair("adi", 64, 320)
    _, _, d2, _, _ = _pair("adi", 64, 320)
    d1.advance(1)
    seg = d1.autotune(reps=2)
    assert 96 <= seg <= 248
    d1.advance(2)
    d2.advance(3)
    a, b = d1.fields(), d2.fields()
    for k in ("dens", "vrad", "vtheta", "energy"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("kind,nrad,nsec", [("iso", 64, 192), ("adi", 48, 160), ("sg", 32, 64)])
def test_accurate_mode_parity(gpu, kind, nrad, nsec):
    """The accurate precision mode against the oracle's accurate mode (the
    same restatement with the FP64 star-potential gradient, Kahan ring means
    and the FP64 self-gravity kernel): integer outcomes exact, fields within
    FIELD_TOL."""
    P, L, _ = small(kind, nrad, nsec)
    d = Disk(P, L)
    d.set_precision(1)
    f0 = d.fields()
    d.init_state(dens=noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, SEED))
    g = d.fields()
    o = Oracle(P, L)
    o.set_precision(1)
    o.set_fields(dens=g["dens"], vrad=g["vrad"], vtheta=g["vtheta"], energy=g["energy"])
    fields = ("dens", "vrad", "vtheta", "energy") if kind == "adi" else ("dens", "vrad", "vtheta")
    _compare(P, d, o, 5, fields=fields, planet_rtol=1e-5 if kind != "iso" else 1e-9)
