"""Host side of the drop-in boundary (no GPU): .par/.cfg parsing and the
command-line driver against the reference's own parse (its -vn output,
tests/golden/pars/*.vn.txt made by tests/golden/make_vn_golden.py)."""
import glob
import os
import subprocess

import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import _abi, configs, grid_radii, read_params, read_planets
from cudaprotoplanetarydisksfloat_b200._abi import FargoError

HERE = os.path.dirname(os.path.abspath(__file__))
PARS = os.path.join(HERE, "golden", "pars")
DRIVER = os.path.join(os.path.dirname(HERE), "cudaprotoplanetarydisksfloat_b200", "fargo_b200")


@pytest.mark.parametrize("par", sorted(glob.glob(os.path.join(PARS, "*.par"))), ids=os.path.basename)
def test_driver_parse_output_matches_reference(par):
    """`fargo_b200 -vn file.par` prints exactly what the reference prints."""
    got = subprocess.run([DRIVER, "-vn", os.path.basename(par)], cwd=PARS, stdout=subprocess.PIPE,
                         stderr=subprocess.STDOUT).stdout
    want = open(par[:-4] + ".vn.txt", "rb").read()
    assert got == want


def test_params_values_and_quirks():
    p = read_params(os.path.join(PARS, "quirks.par"))
    assert p.NRAD == 128 and p.NSEC == 384          # "#NRAD 999" is a comment; "Nsec:=> 200" is key "Nsec:=>"
    assert p.LogGrid == 0 and p.FastTransport == 0  # ARITHMETIC, STANDARD
    assert p.Adiabatic == 0                         # AdiabaticIndex 1 turns it off
    assert p.Write_DivV == 0                        # assigned from a number in the reference
    assert p.RocheSmoothing == 1 and abs(p.ROCHESMOOTHING - 0.5) < 1e-7
    assert p.Corotating == 1 and p.GuidingCenter == 1
    c = read_params(os.path.join(PARS, "c2.par"))
    assert c.ViscosityAlpha == 1 and c.Adiabatic == 1 and c.Write_Temperature == 1
    assert np.float32(c.ALPHAVISCOSITY) == np.float32(1e-3)


def test_params_errors():
    with pytest.raises(FargoError, match="EIO"):
        read_params("/nonexistent/file.par")
    with pytest.raises(FargoError, match="EINVAL"):
        read_params(os.path.join(PARS, "both_viscosities.par"))
    with pytest.raises(FargoError, match="EINVAL"):
        read_params(os.path.join(PARS, "quirks_colon.par"))


def test_planets_cfg():
    p = read_params(os.path.join(PARS, "c2.par"))
    pl = read_planets(os.path.join(PARS, "c2.cfg"), p)
    assert pl.nb == 2
    assert pl.x[1] == 1.6 and pl.mass[1] == 3e-4
    assert pl.feeldisk[0] == 1 and pl.feelothers[1] == 1
    # Psys.cu:196-199
    assert pl.vy[0] == np.sqrt(1.0 * (1.0 + 1e-3) / 1.0)
    assert pl.vx[0] == -0.0000000001 * pl.vy[0]


def test_grid_radii_log_and_arith():
    p, pl = configs.c1()
    import tempfile
    d = tempfile.mkdtemp()
    par, cfg, out = configs.materialise(p, pl, d)
    P = read_params(par)
    r = grid_radii(P)
    i = np.arange(P.NRAD + 1)
    want = np.float32(0.4) * np.exp(i / P.NRAD * np.log(np.float64(np.float32(2.5)) / np.float64(np.float32(0.4))))
    assert np.allclose(r, want, rtol=1e-15, atol=0)


def test_library_exports_every_header_symbol():
    import re
    hdr = open(os.path.join(os.path.dirname(HERE), "include", "fargo_b200.h")).read()
    declared = set(re.findall(r"\b(fargo_[a-z_0-9]+)\s*\(", hdr))
    lib = _abi.lib
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_abi.EXPORTS) >= declared
    assert lib.fargo_abi_version() == 1


def test_create_without_gpu_fails_loudly():
    from tests.conftest import have_gpu
    if have_gpu():
        pytest.skip("a GPU is present")
    from cudaprotoplanetarydisksfloat_b200 import Disk
    p = read_params(os.path.join(PARS, "c1.par"))
    pl = read_planets(os.path.join(PARS, "c1.cfg"), p)
    with pytest.raises(FargoError, match="ENODEV"):
        Disk(p, pl)
