"""Radial decomposition of one disk on the GPU (stripes held by one process).

The stripes, advanced through the stripe entry points with their ghost
rings refreshed after every substep, must give the bits of the same disk
advanced whole by fargo_advance_dt: the substep count of every DT, every
row of every field and the planets.
- C1's grid (128x384, isothermal, viscosity 1e-5, one planet on a fixed
  circular orbit) in 2 and 3 stripes;
- C2 (256x768, adiabatic, alpha viscosity, two live planets that feel the
  disk) in 2 and 4 stripes.
- C3 (512x1024, self-gravity) in 2 and 4 stripes, and C5's grid and physics
  (2048x6144, adiabatic, self-gravity, three live planets; DT shortened to
  0.004, a few substeps) in 2 stripes: every stripe gathers the whole
  density before each substep and runs the whole disk's convolution.
Cuts off the CFL tile grid group the force sums differently: the result
then stays within the FP32 rounding floor of the whole disk (FIELD_TOL).
A NaN in one stripe's own rings stops every stripe's DT with
FARGO_ENONFINITE (every stripe sees the gathered minimum)."""
import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Disk, configs, noise, radial
from cudaprotoplanetarydisksfloat_b200._abi import FargoError
from tests.helpers import FIELD_TOL, SEED, make, planet_err, rel_l2

pytestmark = pytest.mark.gpu

KEYS = ("dens", "vrad", "vtheta", "energy")


def _start(p, pl, name):
    P, L, _ = make(p, pl, name)
    whole = Disk(P, L)
    f0 = whole.fields()
    dens = noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, SEED).reshape(P.NRAD + 1, P.NSEC)
    whole.init_state(dens=dens)
    return P, L, whole, dens


def _planets(pl):
    n = pl.nb
    return np.array([[getattr(pl, k)[i] for k in ("x", "y", "vx", "vy", "mass")] for i in range(n)])


def _run_pair(cfg, name, nstripes, ndt, parts=None):
    p, pl = cfg
    P, L, whole, dens = _start(p, pl, name)
    st = radial.LocalStripes(P, L, nstripes, parts=parts)
    st.init_state(dens=dens)
    n_whole, n_str = [], []
    for _ in range(ndt):
        n_whole.append(whole.advance_dt())
        n_str.append(st.advance_dt())
    a, b = whole.fields(), st.fields()
    pa, pb = _planets(whole.planets()), _planets(st.planets())
    sa, sb = whole.scalars(), st.scalars()
    whole.close()
    st.close()
    return P, n_whole, n_str, a, b, pa, pb, sa, sb


@pytest.mark.parametrize("nstripes", [2, 3])
def test_c1_stripes_bit_identical(gpu, nstripes):
    P, nw, ns, a, b, pa, pb, sa, sb = _run_pair(configs.c1(), "rad_c1", nstripes, 3)
    assert nw == ns
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(pa, pb)
    assert sa["physical_time"] == sb["physical_time"] and sa["last_dt"] == sb["last_dt"]


@pytest.mark.parametrize("nstripes", [2, 4])
def test_c2_stripes_bit_identical(gpu, nstripes):
    P, nw, ns, a, b, pa, pb, sa, sb = _run_pair(configs.c2(), "rad_c2", nstripes, 3)
    assert nw == ns
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(pa, pb)


@pytest.mark.parametrize("nstripes", [2, 4])
def test_c3_self_gravity_stripes_bit_identical(gpu, nstripes):
    P, nw, ns, a, b, pa, pb, _, _ = _run_pair(configs.c3(), "rad_c3", nstripes, 2)
    assert nw == ns
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(pa, pb)


def test_c5_stripes_bit_identical(gpu):
    p, pl = configs.c5()
    p = dict(p, DT="0.004")
    P, nw, ns, a, b, pa, pb, _, _ = _run_pair((p, pl), "rad_c5", 2, 1)
    print("\nC5 in 2 stripes: %d substeps" % ns[0])
    assert nw == ns
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(pa, pb)


def test_c2_unaligned_cuts_within_floor(gpu):
    """A cut at ring 171 (NSEC 768: C2's 1024-cell CFL tiles are 4 rings)
    splits a CFL tile: the FP64 force sums group differently, the planets
    move by rounding, and the fields stay within the FP32 floor."""
    P, nw, ns, a, b, pa, pb, _, _ = _run_pair(configs.c2(), "rad_c2u", 3, 3,
                                               parts=[(0, 100), (100, 171), (171, 256)])
    assert nw == ns
    nrad = P.NRAD
    for k in KEYS:
        e = rel_l2(b[k][:nrad], a[k][:nrad])
        assert e <= FIELD_TOL[k], (k, e)
    assert planet_err(pb[:, :4], pa[:, :4]) < 1e-9


def test_nan_in_one_stripe_stops_all(gpu):
    p, pl = configs.c1()
    P, L, whole, dens = _start(p, pl, "rad_nan")
    whole.close()
    st = radial.LocalStripes(P, L, 3)
    st.init_state(dens=dens)
    f = st.fields()
    lo, hi = st.parts[1]
    f["vtheta"][(lo + hi) // 2, 5] = np.nan
    st.upload(**f)
    with pytest.raises(FargoError, match="ENONFINITE"):
        st.advance_dt()
    for s in st.stripes:  # the DT stopped on every stripe, not only the first to report
        with pytest.raises(FargoError, match="ENONFINITE"):
            s.more()
    st.close()
