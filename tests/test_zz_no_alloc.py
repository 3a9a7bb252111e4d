"""fargo_disk_force_noalloc against fargo_disk_force, on one disk state.

fargo_disk_force_noalloc serves programs that keep their disk in their own
device arrays (the reference's layout: Dens, CellAbscissa, CellOrdinate,
Surf, Rmed) and may not allocate device memory in the middle of a step,
because they manage device memory themselves or cannot afford cudaMalloc's
device-wide synchronisation.  It takes no context and uses only a fixed
static scratch array.  Two calls in a row must each agree with the
context-based entry point and with the CPU oracle within the disk-force
tolerance of the parity tests; the second call must leave free device
memory unchanged, and an NRAD beyond the scratch must be refused with a
clear message.

The file name makes pytest collect it last."""
import ctypes as C

import numpy as np
import pytest
import torch

from cudaprotoplanetarydisksfloat_b200 import Disk, grid_radii, noise
from cudaprotoplanetarydisksfloat_b200._abi import FARGO_DIMFXY, FARGO_NOALLOC_MAXRAD, lib
from oracle.oracle import Oracle
from tests.helpers import SEED, rel_l2, small

pytestmark = pytest.mark.gpu

FARGO_EINVAL = 1


def _device_arrays(d, P):
    """The disk's density and the reference's geometry arrays, on the GPU."""
    nrad, nsec = P.NRAD, P.NSEC
    r = grid_radii(P)
    # the library's ring tables: FP64 formulas of FillPolar1DArrays rounded to float
    rmed = (2.0 / 3.0 * (r[1:] ** 3 - r[:-1] ** 3) / (r[1:] ** 2 - r[:-1] ** 2)).astype(np.float32)
    surf = (np.pi * (r[1:] ** 2 - r[:-1] ** 2) / nsec).astype(np.float32)
    # CellAbscissa / CellOrdinate: Rmed * cosf(2 pi j / NSEC) in float
    ang = (2.0 * np.pi * np.arange(nsec) / nsec).astype(np.float32)
    cell_x = rmed[:, None] * np.cos(ang)[None, :]
    cell_y = rmed[:, None] * np.sin(ang)[None, :]
    dens = d.fields()["dens"][:nrad].reshape(nrad, nsec).astype(np.float32)
    dev = torch.device("cuda", 0)
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev)
            for k, v in (("dens", dens), ("cell_x", cell_x), ("cell_y", cell_y), ("surf", surf), ("rmed", rmed))}


def _noalloc(T, nrad, nsec, x, y, rs, mass):
    gf = np.zeros(4 * FARGO_DIMFXY, np.float64)
    err = C.create_string_buffer(512)
    stream = torch.cuda.current_stream(0).cuda_stream
    st = lib.fargo_disk_force_noalloc(T["dens"].data_ptr(), T["cell_x"].data_ptr(), T["cell_y"].data_ptr(),
                                      T["surf"].data_ptr(), T["rmed"].data_ptr(), nrad, nsec, x, y, rs, mass,
                                      FARGO_DIMFXY, gf.ctypes.data_as(C.POINTER(C.c_double)), stream, err, 512)
    return st, gf, err.value.decode()


def test_noalloc_disk_force_matches_context_entry_point(gpu):
    P, L, _ = small("adi", 64, 192)
    d = Disk(P, L)
    f0 = d.fields()
    d.init_state(dens=noise.perturb_density(f0["dens"].reshape(-1), P.NRAD, P.NSEC, SEED))
    d.advance(2)
    T = _device_arrays(d, P)
    # the CPU oracle on the same density (the checker of every disk force)
    o = Oracle(P, L)
    o.set_fields(dens=d.fields()["dens"])
    torch.cuda.synchronize()
    bodies = [(1.0, 0.0, 0.03, 1e-3), (0.3, -0.9, 0.05, 3e-4)]
    for n, (x, y, rs, m) in enumerate(bodies):
        before = torch.cuda.mem_get_info(0)[0]
        st, got, msg = _noalloc(T, P.NRAD, P.NSEC, x, y, rs, m)
        after = torch.cuda.mem_get_info(0)[0]
        assert st == 0, msg
        if n == 1:
            # the second call (set-up done by the first) allocates nothing
            assert after == before
        want = d.disk_force(x, y, rs, m)
        assert rel_l2(got, want) <= 1e-6
        assert np.allclose(got, want, rtol=1e-5, atol=1e-6 * np.abs(want).max())
        assert rel_l2(got, o.disk_force(x, y, rs, m)) <= 1e-6
    d.close()


def test_noalloc_rejects_grid_beyond_scratch(gpu):
    T = {k: torch.zeros(1, device="cuda") for k in ("dens", "cell_x", "cell_y", "surf", "rmed")}
    st, _, msg = _noalloc(T, FARGO_NOALLOC_MAXRAD + 1, 8, 1.0, 0.0, 0.03, 1e-3)
    assert st == FARGO_EINVAL
    assert "exceeds" in msg and str(FARGO_NOALLOC_MAXRAD) in msg
