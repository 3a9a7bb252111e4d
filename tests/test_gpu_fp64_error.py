"""Error of the FP32 CUDA step against an FP64 run of the same algorithm.

The oracle built in double (every float of the reference's arithmetic
promoted) starts from the state the GPU initialised and both advance 10 DTs,
in both precision modes of the library:

- reference (default): the reference's FP32 arithmetic, bit-exact integer
  outcomes.  Its Sigma error is ~2e-5 after 10 DTs, most of it from the
  star's potential: Substep1 differences two FP32 values of -G/r across a
  ring spacing of ~1%.
- accurate (FARGO_PRECISION_ACCURATE): that term as an FP64-derived
  difference quotient, Kahan ring means.  On C1 the Sigma error drops to
  ~1.0e-5 after 10 DTs (the oracle's accurate mode, without fused
  multiply-adds: 9.85e-6).  That is the floor of FP32 storage: the FP64
  oracle with every stored intermediate of the substep rounded to FP32 and
  nothing else changed lands at 8.6e-6.  On C2 (adiabatic, alpha viscosity,
  two live planets) the same storage floor is ~7e-5 and both modes sit on
  it: no arithmetic change inside an FP32-storage design removes it.

Reported per case (run with -s): rel-L2 of Sigma, v_r, v_theta and energy,
the planets' position error relative to their orbital radius, the error of
the disk force on planet 0 at all Hill-cut levels, and the mass and
angular-momentum drift of each run (relative change over the 10 DTs)."""
import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Disk, configs, noise, planets_dict
from oracle.oracle import Oracle, set_threads
from tests.helpers import SEED, make, rel_l2

pytestmark = pytest.mark.gpu

# loose bounds for every case: they catch a broken path, not rounding
BOUND = {"dens": 1e-4, "vrad": 2e-3, "vtheta": 1e-5, "energy": 2e-4}
# the accurate mode on C1 (isothermal, one fixed planet): the target of
# 1e-5 after 10 DTs, at the FP32 storage floor (9.99e-6 measured on the B200,
# with the accurate mode's kernels built without fused multiply-adds)
C1_ACCURATE_SIGMA = 1e-5


def _case(name):
    p, pl = configs.c1() if name == "C1" else configs.c2()
    return make(p, pl, "fp64" + name)


@pytest.mark.parametrize("mode", [0, 1], ids=["reference", "accurate"])
@pytest.mark.parametrize("name", ["C1", "C2"])
def test_error_vs_fp64(gpu, name, mode):
    P, L, _ = _case(name)
    d = Disk(P, L)
    d.set_precision(mode)
    f0 = d.fields()
    d.init_state(dens=noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, SEED))
    g = d.fields()
    set_threads(16, "f64")
    o = Oracle(P, L, prec="f64")
    o.set_fields(dens=g["dens"], vrad=g["vrad"], vtheta=g["vtheta"], energy=g["energy"])
    s0, q0 = d.scalars(), o.scalars()
    for _ in range(10):
        d.advance_dt()
        o.advance_dt()
    a, b = d.fields(), o.fields(native=True)
    nrad = P.NRAD
    err = {k: rel_l2(a[k][:nrad], b[k][:nrad]) for k in ("dens", "vrad", "vtheta")}
    if P.Adiabatic:
        err["energy"] = rel_l2(a["energy"][:nrad], b["energy"][:nrad])
    pa, pb = planets_dict(d.planets()), planets_dict(o.planets())
    r = np.hypot(pb["x"], pb["y"])
    orbit = float(np.max(np.hypot(pa["x"] - pb["x"], pa["y"] - pb["y"]) / r))
    x, y, m = float(pb["x"][0]), float(pb["y"][0]), float(pb["mass"][0])
    rs = 0.6 * 0.05 * float(r[0])
    torque = rel_l2(d.disk_force(x, y, rs, m), o.disk_force(x, y, rs, m))
    s1, q1 = d.scalars(), o.scalars()
    drift = {"mass_f32": (s1["mass"] - s0["mass"]) / s0["mass"], "mass_f64": (q1["mass"] - q0["mass"]) / q0["mass"],
             "am_f32": (s1["angular_momentum"] - s0["angular_momentum"]) / s0["angular_momentum"],
             "am_f64": (q1["angular_momentum"] - q0["angular_momentum"]) / q0["angular_momentum"]}
    print("\n%s %s: rel-L2 vs FP64 after 10 DTs %s; planet orbit %.2e; disk force %.2e; drift %s" % (
        name, ["reference", "accurate"][mode], {k: "%.2e" % v for k, v in err.items()}, orbit, torque,
        {k: "%.2e" % v for k, v in drift.items()}))
    for k, e in err.items():
        assert e <= BOUND[k], (k, e)
    if name == "C1" and mode == 1:
        assert err["dens"] <= C1_ACCURATE_SIGMA, err
    assert orbit <= 1e-5
    assert torque <= 1e-3
    # mass and angular momentum: the FP32 run drifts as the FP64 run does
    assert abs(drift["mass_f32"] - drift["mass_f64"]) <= 1e-5
    assert abs(drift["am_f32"] - drift["am_f64"]) <= 1e-5
