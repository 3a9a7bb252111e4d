"""The transport tile autotuner (fargo_batch_autotune).

- Results do not depend on the segment widths it picks: a tuned batch and an
  untuned one advanced from the same state give the same bits.
- It tunes each class of disk (NSEC) on its own: the widths it reports per
  disk are candidates of the search, equal within a class.
- Its choices are kept for the process: a batch created afterwards with
  disks of the tuned classes starts from the tuned widths."""
import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Batch, noise
from tests.helpers import SEED, small

pytestmark = pytest.mark.gpu

CAND = {96, 128, 160, 192, 224, 244}
SIZES = [(64, 384), (48, 768), (64, 384), (40, 1280)]


def _batch(P, L):
    b = Batch(P, L)
    for k, p in enumerate(P):
        f = b.fields(k)
        b.init_state(k, dens=noise.perturb_density(f["dens"].reshape(-1), p.NRAD, p.NSEC, SEED + k))
    return b


def test_autotune_per_class_cached_and_exact(gpu):
    P, L = [], []
    for nrad, nsec in SIZES:
        p, l, _ = small("iso", nrad, nsec)
        P.append(p)
        L.append(l)
    tuned, plain = _batch(P, L), _batch(P, L)
    seg = tuned.autotune(reps=2)
    segs = tuned.segments()
    print("\nsegment widths per disk:", segs, "(largest class:", seg, ")")
    assert set(segs) <= CAND
    assert segs[0] == segs[2]  # one class, one width
    for b in (tuned, plain):
        b.advance(2)
    for k in range(len(P)):
        a, c = tuned.fields(k), plain.fields(k)
        for f in ("dens", "vrad", "vtheta"):
            assert np.array_equal(a[f], c[f]), (k, f)
    later = Batch(P[:2], L[:2])
    assert later.segments() == segs[:2]
    for b in (tuned, plain, later):
        b.close()
