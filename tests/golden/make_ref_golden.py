"""Golden data from the reference's own CUDA implementation.

oracle/ref/Makefile.ref compiles the reference's unmodified sources into
oracle/_ref/fargo_ref (with link-level hooks that add the seeded density
noise right after InitGasDensity and dump dt + Nshift after every Transport,
see oracle/ref/ref_hooks.cu).  This script runs it and packs the outputs:

  on a GPU box:   python tests/golden/make_ref_golden.py run <rawdir> [case ...]
  here:           python tests/golden/make_ref_golden.py collect <rawdir> [case ...]

`collect` writes tests/golden/<case>.npz with the reference's output fields
after 0 and NDT time steps (dens/vrad/vtheta/energy/temperature dumps,
Output.cu:104-170; only after NDT steps for grids of BIG cells or more), the
per-substep dt and Nshift, the bigplanet and tqwk log lines
(Output.cu:70-88, Force.cu:76-138) and used_rad.dat.
"""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cudaprotoplanetarydisksfloat_b200 import configs  # noqa: E402

SEED = 20261203
NDT = 10

# name: (params, planets, noise seed or None, DTs)
def cases():
    out = {}
    p, pl = configs.small("iso", 128, 256)
    out["ref_iso_128x256"] = (p, pl, SEED, NDT)
    p, pl = configs.small("adi", 128, 256)
    p = dict(p, WriteEnergy="YES")
    out["ref_adi_128x256"] = (p, pl, SEED + 1, NDT)
    p, pl = configs.c1()
    out["ref_c1_128x384"] = (p, pl, None, NDT)
    # the non-rigid boundaries (ApplyBoundaryCondition, SideEuler.cu:172-182)
    p, pl = configs.small("adi", 128, 256)
    p = dict(p, InnerBoundary="NONREFLECTING", WriteEnergy="YES")
    out["ref_nr_adi_128x256"] = (p, pl, SEED + 2, NDT)
    p, pl = configs.small("adi", 128, 256)
    p = dict(p, InnerBoundary="EVANESCENT", WriteEnergy="YES", Cooling="YES", CoolingTime0="31.4")
    out["ref_ev_adi_128x256"] = (p, pl, SEED + 3, NDT)
    p, pl = configs.small("iso", 128, 256)
    p = dict(p, InnerBoundary="OPEN")
    out["ref_open_iso_128x256"] = (p, pl, SEED + 4, NDT)
    # the benchmark configurations at their own size: C2 (adiabatic, alpha
    # viscosity, two live planets) and the largest disk size of the C4 sweep
    # (the sweep's first 512-ring disk, with the noise seed the sweep gives it)
    p, pl = configs.c2()
    p = dict(p, WriteEnergy="YES")
    out["ref_c2_256x768"] = (p, pl, SEED + 5, NDT)
    k, (p, pl) = c4_disk(512)
    out["ref_c4d%02d_512x1536" % k] = (p, pl, SEED + k, NDT)
    return out


def c4_disk(nrad):
    """(index, (params, planets)) of the first disk of the 64-disk sweep with
    `nrad` rings."""
    for k, d in enumerate(configs.c4(64, seed=42)):
        if int(d[0]["Nrad"]) == nrad:
            return k, d
    raise ValueError(nrad)


# fixtures of this many cells or more store only the fields after NDT DTs
# (the initial fields are rebuilt from the parameters and the seed, and the
# small cases already pin that initialisation to the reference's)
BIG = 150000


def _selected(names):
    return {k: v for k, v in cases().items() if not names or k in names}


def run(rawdir, names=()):
    rawdir = os.path.abspath(rawdir)
    exe = os.path.join(ROOT, "oracle", "_ref", "fargo_ref")
    if not os.path.exists(exe):
        raise SystemExit("build the reference first: make -f oracle/ref/Makefile.ref")
    status = 0
    for name, (p, pl, seed, ndt) in _selected(names).items():
        d = os.path.join(rawdir, name)
        p = dict(p, Ntot=str(ndt), Ninterm=str(ndt))
        par, cfg, out = configs.materialise(p, pl, d, "run", relative=True)
        env = dict(os.environ, FARGO_REF_DUMP="dump_")
        if seed is not None:
            env["FARGO_REF_NOISE_SEED"] = str(seed)
        with open(os.path.join(d, "stdout.txt"), "w") as f:
            r = subprocess.run([exe, "run.par"], cwd=d, env=env, stdout=f, stderr=subprocess.STDOUT, timeout=1200)
        print(name, "exit", r.returncode)
        status |= r.returncode
    return status


def _read_field(path, nrad, nsec):
    return np.fromfile(path, dtype=np.float32).reshape(nrad, nsec)


def collect(rawdir, names=()):
    rawdir = os.path.abspath(rawdir)
    for name, (p, pl, seed, ndt) in _selected(names).items():
        d = os.path.join(rawdir, name)
        out = os.path.join(d, "run_out")
        nrad, nsec = int(p["Nrad"]), int(p["Nsec"])
        z = {"nrad": nrad, "nsec": nsec, "ndt": ndt, "seed": -1 if seed is None else seed}
        big = nrad * nsec >= BIG
        for fld in ("dens", "vrad", "vtheta", "energy", "temperature"):
            if big and fld == "temperature":
                continue
            for k in ((1,) if big else (0, 1)):
                f = os.path.join(out, fld, "%s%d.dat" % (fld, k))
                if os.path.exists(f):
                    z["%s%d" % (fld, k)] = _read_field(f, nrad, nsec)
        raw = np.fromfile(os.path.join(d, "dump_nshift.bin"), dtype=np.uint8)
        rec = 8 + 4 * nrad
        nrec = raw.size // rec
        raw = raw[:nrec * rec].reshape(nrec, rec)
        z["sub_dt"] = raw[:, :8].copy().view(np.float64).reshape(-1)
        z["sub_nshift"] = raw[:, 8:].copy().view(np.int32).reshape(nrec, nrad)
        rows = []
        for k in range(len(pl)):
            f = os.path.join(out, "bigplanet%d.dat" % k)
            rows.append(np.loadtxt(f, ndmin=2))
        z["bigplanet"] = np.stack(rows)
        tq = []
        for k in range(len(pl)):
            f = os.path.join(out, "tqwk%d.dat" % k)
            tq.append(np.loadtxt(f, ndmin=2))
        z["tqwk"] = np.stack(tq)
        z["used_rad"] = np.loadtxt(os.path.join(out, "used_rad.dat"))
        alg = np.loadtxt(os.path.join(d, "dump_algogas.txt"), ndmin=2)
        z["algogas_seconds"] = alg[:, 1]
        np.savez_compressed(os.path.join(ROOT, "tests", "golden", name + ".npz"), **z)
        print(name, {k: np.shape(v) for k, v in z.items()})


if __name__ == "__main__":
    if len(sys.argv) < 3 or sys.argv[1] not in ("run", "collect"):
        raise SystemExit(__doc__)
    if sys.argv[1] == "run":
        sys.exit(run(sys.argv[2], sys.argv[3:]))
    collect(sys.argv[2], sys.argv[3:])
