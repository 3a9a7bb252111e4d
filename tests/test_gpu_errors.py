"""Error paths of the step, made on the host: no GPU fault is involved.

- A NaN in an uploaded field makes the CFL step non-finite: the DT stops on
  the device and the call returns FARGO_ENONFINITE.
- A substep limit below what the DT needs stops the DT after that many
  substeps: FARGO_ETIMEOUT (the reference has no limit; the library's
  default, 100000, only guards against a DT that would never end).
In both cases the context stays usable: restored from the checkpoint taken
before the failed DT, the next DT runs and gives the same bits as a fresh
context restored from it.
Both the CUDA graph (device-driven loop) and the host loop are covered."""
import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Disk, noise
from cudaprotoplanetarydisksfloat_b200._abi import FARGO_MAX_SUBSTEPS, FargoError
from tests.helpers import SEED, small

pytestmark = pytest.mark.gpu


def _disk(graph):
    P, L, _ = small("iso", 32, 96)
    d = Disk(P, L)
    f0 = d.fields()
    d.init_state(dens=noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, SEED))
    d.set_graph_mode(graph)
    return P, L, d


def _same_as_fresh(P, L, d, blob):
    """Restore the checkpoint taken before the failed DT; the next DT must
    give the bits a fresh context restored from it gives."""
    d.restore(blob)
    ref = Disk(P, L)
    ref.restore(blob)
    n1, n2 = d.advance_dt(), ref.advance_dt()
    assert n1 == n2 > 0
    a, b = d.fields(), ref.fields()
    for k in ("dens", "vrad", "vtheta"):
        assert np.array_equal(a[k], b[k]), k
    ref.close()


@pytest.mark.parametrize("graph", [True, False])
def test_nan_in_state_gives_enonfinite(gpu, graph):
    P, L, d = _disk(graph)
    blob = d.checkpoint()
    good = d.fields()
    bad = {k: v.copy() for k, v in good.items()}
    bad["vtheta"][P.NRAD // 2, 7] = np.nan
    d.upload(dens=bad["dens"], vrad=bad["vrad"], vtheta=bad["vtheta"], energy=bad["energy"])
    with pytest.raises(FargoError, match="ENONFINITE"):
        d.advance_dt()
    _same_as_fresh(P, L, d, blob)
    d.close()


@pytest.mark.parametrize("graph", [True, False])
def test_substep_limit_gives_etimeout(gpu, graph):
    P, L, d = _disk(graph)
    blob = d.checkpoint()
    probe = Disk(P, L)
    probe.restore(blob)
    need = probe.advance_dt()
    probe.close()
    assert need > 2
    d.set_max_substeps(need - 1)
    with pytest.raises(FargoError, match="ETIMEOUT"):
        d.advance_dt()
    assert d.scalars()["nsub_last_dt"] == need - 1
    d.set_max_substeps(FARGO_MAX_SUBSTEPS)
    _same_as_fresh(P, L, d, blob)
    d.close()
