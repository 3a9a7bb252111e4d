"""Error of the FP32 CUDA step against an FP64 run of the same algorithm.

The oracle built in double (every float of the reference's arithmetic
promoted) starts from the state the GPU initialised and both advance 10 DTs.
Reported per case (run with -s to see the table): rel-L2 of Sigma, v_r,
v_theta and energy, the planets' position error relative to their orbital
radius, the error of the disk force on planet 0 at all Hill-cut levels, and
the mass and angular-momentum drift of each run.  The bounds asserted here
are loose (they catch a broken path, not rounding): the reference
algorithm's own FP32-vs-FP64 gap after 10 DTs is ~1-2e-5 in Sigma and
~1-2e-4 in v_r, because the seeded noise is advected and amplified."""
import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Disk, configs, noise, planets_dict
from oracle.oracle import Oracle
from tests.helpers import SEED, make, rel_l2

pytestmark = pytest.mark.gpu

BOUND = {"dens": 1e-4, "vrad": 1e-3, "vtheta": 1e-5, "energy": 2e-4}


def _case(name):
    if name == "C1 128x384 isothermal":
        p, pl = configs.c1()
    else:
        p, pl = configs.small("adi", 128, 384)
    return make(p, pl, "fp64")


@pytest.mark.parametrize("name", ["C1 128x384 isothermal", "adiabatic 128x384, two live planets"])
def test_error_vs_fp64(gpu, name):
    P, L, _ = _case(name)
    d = Disk(P, L)
    f0 = d.fields()
    d.init_state(dens=noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, SEED))
    g = d.fields()
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
    print("\n%s: rel-L2 vs FP64 after 10 DTs %s; planet orbit %.2e; disk force %.2e; drift %s" % (
        name, {k: "%.2e" % v for k, v in err.items()}, orbit, torque, {k: "%.2e" % v for k, v in drift.items()}))
    for k, e in err.items():
        assert e <= BOUND[k], (k, e)
    assert orbit <= 1e-5
    assert torque <= 1e-3
    assert abs(drift["mass_f32"] - drift["mass_f64"]) <= 1e-5
