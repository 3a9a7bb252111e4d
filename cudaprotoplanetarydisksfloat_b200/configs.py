"""The benchmark workloads as reference .par/.cfg files.

C1..C5 are the five configurations of the reference's headline benchmark
(small isothermal disk, adiabatic two-planet disk, self-gravitating disk,
64-disk batched sweep, high-resolution production run); `small_*` are
reduced versions of the same physics used by the parity tests.  Everything
is written as text files in the reference's format and parsed by the
library's own ReadVariables (fargo_params_read), so a config means the same
to this library and to the reference binary.
"""
import os

import numpy as np

DT = "0.314159265359"

BASE = {
    "AspectRatio": "0.05",
    "Sigma0": "6.3662e-4",
    "SigmaSlope": "0.5",
    "FlaringIndex": "0.0",
    "ThicknessSmoothing": "0.6",
    "Transport": "FARGO",
    "InnerBoundary": "RIGID",
    "Disk": "YES",
    "OmegaFrame": "0.0",
    "Frame": "FIXED",
    "IndirectTerm": "YES",
    "RadialSpacing": "LOGARITHM",
    "Ntot": "200",
    "Ninterm": "10",
    "DT": DT,
    "SelfGravity": "NO",
    "Adiabatic": "NO",
    "AdiabaticIndex": "1.4",
    "Cooling": "NO",
}


def c1():
    p = dict(BASE, Nrad="128", Nsec="384", Rmin="0.4", Rmax="2.5", Viscosity="1e-5",
             ForcedCircular="YES")
    planets = [("Jupiter", 1.0, 1e-3, "NO", "NO")]
    return p, planets


def c2():
    p = dict(BASE, Nrad="256", Nsec="768", Rmin="0.4", Rmax="3.0", AlphaViscosity="1e-3",
             Adiabatic="YES", ForcedCircular="NO", Ntot="500")
    planets = [("Planet1", 1.0, 1e-3, "YES", "YES"), ("Planet2", 1.6, 3e-4, "YES", "YES")]
    return p, planets


def c3():
    p = dict(BASE, Nrad="512", Nsec="1024", Rmin="0.3", Rmax="4.0", Viscosity="1e-5",
             SigmaSlope="1.0", Sigma0="2.1507e-3", ThicknessSmoothing="0.3", SelfGravity="YES",
             ForcedCircular="YES", Ntot="300")
    planets = [("Planet", 1.0, 5e-4, "NO", "NO")]
    return p, planets


def c5():
    p = dict(BASE, Nrad="2048", Nsec="6144", Rmin="0.3", Rmax="5.0", AlphaViscosity="1e-3",
             Adiabatic="YES", SelfGravity="YES", ForcedCircular="NO")
    planets = [("P1", 1.0, 1e-3, "YES", "YES"), ("P2", 1.5, 3e-4, "YES", "YES"),
               ("P3", 2.3, 1e-4, "YES", "YES")]
    return p, planets


def c4(n=64, seed=42):
    """64 isothermal disks of uneven size and physics (seeded draws)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nrad = int(rng.choice([128, 192, 256, 384, 512]))
        q = float(np.exp(rng.uniform(np.log(1e-5), np.log(3e-3))))
        alpha = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
        h = float(rng.uniform(0.03, 0.08))
        slope = float(rng.uniform(0.0, 1.5))
        p = dict(BASE, Nrad=str(nrad), Nsec=str(3 * nrad), Rmin="0.4", Rmax="2.5",
                 AlphaViscosity="%.9g" % alpha, AspectRatio="%.9g" % h, SigmaSlope="%.9g" % slope,
                 ForcedCircular="YES", Ntot="1000")
        out.append((p, [("Planet", 1.0, q, "NO", "NO")]))
    return out


def small(kind="iso", nrad=32, nsec=96):
    """Reduced grids of each physics path for the parity tests."""
    if kind == "iso":
        p, pl = c1()
    elif kind == "adi":
        p, pl = c2()
    elif kind == "sg":
        p, pl = c3()
    elif kind == "adisg":
        p, pl = c5()
    else:
        raise ValueError(kind)
    p = dict(p, Nrad=str(nrad), Nsec=str(nsec))
    return p, pl


def write_cfg(path, planets):
    with open(path, "w") as f:
        f.write("# Planet Name \tDistance\tMass\tAccretion\tFeels Disk\tFeels Others\n")
        for name, dist, mass, fd, fo in planets:
            f.write("%s\t\t%.17g\t\t%.17g\t0.0\t%s\t\t%s\n" % (name, dist, mass, fd, fo))


def write_par(path, params, cfg_path, outdir):
    with open(path, "w") as f:
        for k, v in params.items():
            f.write("%s\t\t%s\n" % (k, v))
        f.write("PlanetConfig\t\t%s\n" % cfg_path)
        f.write("OutputDir\t\t%s\n" % outdir)


def materialise(params, planets, directory, name="run", relative=False):
    """Write <name>.par / <name>.cfg and an output directory; return the paths.

    relative=True writes the paths inside the .par relative to `directory`
    (run the program from there): the reference copies PlanetConfig and
    OutputDir-derived names into 100-character buffers (Main.cu:104,283;
    SourceEuler.cu:106-110), so long absolute paths get truncated."""
    os.makedirs(directory, exist_ok=True)
    cfg = os.path.join(directory, name + ".cfg")
    par = os.path.join(directory, name + ".par")
    out = os.path.join(directory, name + "_out") + "/"
    os.makedirs(out, exist_ok=True)
    write_cfg(cfg, planets)
    if relative:
        write_par(par, params, name + ".cfg", name + "_out/")
    else:
        write_par(par, params, cfg, out)
    return par, cfg, out
