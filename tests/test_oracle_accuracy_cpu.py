"""The oracle's accurate precision mode against its FP64 build (CPU).

The FP32 restatement with the FP64 star-potential gradient and Kahan ring
means (orc_set_precision(1), the same mode as the library's
FARGO_PRECISION_ACCURATE) must stay within 1e-5 relative-L2 of the FP64
build in Sigma after 10 DTs of C1 (128x384), where the reference's own FP32
arithmetic is ~2e-5 away."""
import os

from cudaprotoplanetarydisksfloat_b200 import configs, noise
from oracle.oracle import Oracle, set_threads
from tests.helpers import SEED, make, rel_l2


def test_accurate_mode_meets_1e5_on_c1():
    p, pl = configs.c1()
    P, L, _ = make(p, pl, "acc")
    n = os.cpu_count() or 1
    set_threads(n, "f32")
    set_threads(n, "f64")
    ref, acc, o64 = Oracle(P, L, "f32"), Oracle(P, L, "f32"), Oracle(P, L, "f64")
    acc.set_precision(1)
    f = ref.fields()
    ref.init_state(dens=noise.perturb_density(f["dens"].reshape(-1), P.NRAD, P.NSEC, SEED))
    g = ref.fields()
    for o in (acc, o64):
        o.set_fields(dens=g["dens"], vrad=g["vrad"], vtheta=g["vtheta"], energy=g["energy"])
    for _ in range(10):
        for o in (ref, acc, o64):
            o.advance_dt()
    a, r, b = acc.fields(), ref.fields(), o64.fields()
    e_acc = rel_l2(a["dens"][:P.NRAD], b["dens"][:P.NRAD])
    e_ref = rel_l2(r["dens"][:P.NRAD], b["dens"][:P.NRAD])
    assert e_acc <= 1e-5, e_acc
    assert e_ref > 1.5 * e_acc, (e_ref, e_acc)
