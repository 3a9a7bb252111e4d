"""The drop-in driver end to end: outputs, checkpoints and -s restart.

A run of 4 DTs with an output every 2 writes outputs 0, 1, 2 and a
checkpoint with each; a second run restarted from output 1 (`-s 1`, which the
reference parses but never acts on, Main.cu:147-155) must write output 2
bit for bit as the uninterrupted run did.  The Disk API's checkpoint /
restore is checked the same way."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import Disk, configs
from tests.helpers import small

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(os.path.dirname(HERE), "cudaprotoplanetarydisksfloat_b200", "fargo_b200")


def _run(args, cwd):
    r = subprocess.run([DRIVER] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def _par(tmp, name, **over):
    p, pl = configs.small("adi", 32, 96)
    p = dict(p, Ntot="4", Ninterm="2", WriteEnergy="YES", **over)
    return configs.materialise(p, pl, os.path.join(tmp, name), "run")


def test_driver_restart_continues_bit_for_bit(gpu, tmp_path):
    tmp = str(tmp_path)
    par_a, _, out_a = _par(tmp, "a")
    stdout = _run([par_a], tmp)
    assert "*** OUTPUT 2 ***" in stdout
    for k in range(3):
        for fld in ("dens", "vrad", "vtheta", "energy"):
            assert os.path.getsize(os.path.join(out_a, fld, "%s%d.dat" % (fld, k))) == 32 * 96 * 4
        assert os.path.exists(os.path.join(out_a, "checkpoint%d.bin" % k))
    par_b, _, out_b = _par(tmp, "b")
    shutil.copy(os.path.join(out_a, "checkpoint1.bin"), out_b)
    stdout = _run(["-s", "1", par_b], tmp)
    assert "*** OUTPUT 1 ***" in stdout and "*** OUTPUT 0 ***" not in stdout
    for fld in ("dens", "vrad", "vtheta", "energy"):
        a = np.fromfile(os.path.join(out_a, fld, "%s2.dat" % fld), np.float32)
        b = np.fromfile(os.path.join(out_b, fld, "%s2.dat" % fld), np.float32)
        assert np.array_equal(a, b), fld


def test_checkpoint_restore_api(gpu):
    P, L, _ = small("iso", 32, 96)
    d1, d2 = Disk(P, L), Disk(P, L)
    d1.advance(2)
    blob = d1.checkpoint()
    d1.advance(2)
    d2.restore(blob)
    d2.advance(2)
    a, b = d1.fields(), d2.fields()
    for k in ("dens", "vrad", "vtheta"):
        assert np.array_equal(a[k], b[k]), k
    pa, pb = d1.planets(), d2.planets()
    assert pa.x[0] == pb.x[0] and pa.y[0] == pb.y[0]


def test_driver_output_files_match_reference(gpu, tmp_path):
    """The drop-in driver on C1 (128x384, no noise) for 10 DTs against the
    reference's own run of the same .par (tests/golden/ref_c1_128x384.npz):
    used_rad.dat (SourceEuler.cu:159-171) identical; bigplanet0.dat
    (Output.cu:70-88) line by line: planet to 1e-6 of its scale, mass,
    PhysicalTime and OmegaFrame exact, CircumPlanetaryMass to 1e-4;
    tqwk0.dat (UpdateLog, Force.cu:76-138) torques and powers within 1e-4 of
    each column's largest value (FP64 force sums here, FP32 tree sums in the
    reference, of fields within REF_TOL); the fields after 10 DTs within
    REF_TOL (tests/helpers.py)."""
    from tests.golden import make_ref_golden as G
    from tests.helpers import REF_TOL, rel_l2
    z = np.load(os.path.join(HERE, "golden", "ref_c1_128x384.npz"))
    p, pl, seed, ndt = G.cases()["ref_c1_128x384"]
    assert seed is None
    d = str(tmp_path / "c1")
    p = dict(p, Ntot=str(ndt), Ninterm=str(ndt))
    configs.materialise(p, pl, d, "run", relative=True)
    _run(["run.par"], d)
    out = os.path.join(d, "run_out")
    used = np.loadtxt(os.path.join(out, "used_rad.dat"))
    assert np.array_equal(used, z["used_rad"])
    big = np.loadtxt(os.path.join(out, "bigplanet0.dat"), ndmin=2)
    ref = z["bigplanet"][0]
    assert big.shape == ref.shape
    for c in (1, 2, 3, 4):
        assert np.abs(big[:, c] - ref[:, c]).max() <= 1e-6 * np.abs(ref[:, c]).max(), c
    for c in (0, 5, 6, 7, 8):
        assert np.array_equal(big[:, c], ref[:, c]), c
    assert np.allclose(big[:, 9], ref[:, 9], rtol=1e-4, atol=0)
    tq = np.loadtxt(os.path.join(out, "tqwk0.dat"), ndmin=2)
    rq = z["tqwk"][0]
    assert tq.shape == rq.shape
    assert np.array_equal(tq[:, 0], rq[:, 0]) and np.array_equal(tq[:, 9], rq[:, 9])
    for c in range(1, 9):
        assert np.abs(tq[:, c] - rq[:, c]).max() <= 1e-4 * np.abs(rq[:, c]).max(), c
    nrad, nsec = int(z["nrad"]), int(z["nsec"])
    for fld in ("dens", "vrad", "vtheta"):
        a = np.fromfile(os.path.join(out, fld, "%s1.dat" % fld), np.float32).reshape(nrad, nsec)
        assert rel_l2(a, z[fld + "1"]) <= REF_TOL[fld], fld
