"""Golden parse output of the reference: runs the reference binary built by
oracle/ref/Makefile.ref in parse-only verbose mode (`-vn`, Main.cu:114-119,
224-227: ReadVariables then TellEverything, no GPU work) on the .par files
under tests/golden/pars/ and stores its stdout next to them as *.vn.txt.

    python tests/golden/make_vn_golden.py
"""
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "fargo_ref")

if __name__ == "__main__":
    for par in sorted(glob.glob(os.path.join(HERE, "pars", "*.par"))):
        out = subprocess.run([EXE, "-vn", os.path.basename(par)], cwd=os.path.dirname(par),
                             stdout=subprocess.PIPE, stderr=subprocess.STDOUT).stdout
        with open(par[:-4] + ".vn.txt", "wb") as f:
            f.write(out)
        print(os.path.basename(par), len(out))
