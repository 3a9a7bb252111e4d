"""Build the in-tree CUDA library (sm_100a) and the drop-in driver binary.

    python cudaprotoplanetarydisksfloat_b200/build.py

Outputs, next to this file:
    libfargo_b200.so   the C ABI of include/fargo_b200.h
    fargo_b200         drop-in command-line driver (same flags / .par / outputs)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfargo_b200.so")
EXE = os.path.join(HERE, "fargo_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           "-diag-suppress", "177", "-I" + os.path.join(ROOT, "include")]

LIB_SOURCES = ["kernels_step.cu", "kernels_dispatch.cu", "fargo_api.cu", "sg.cu", "noalloc.cu", "host_params.cpp",
               "host_setup.cpp"]
# the step kernels a second time, without contraction of a*b+c into fused
# multiply-adds: the accurate precision mode's kernel set
VARIANTS = [("kernels_step.cu", "kernels_step_nofma.cu.o", ["-DFARGO_NOFMA", "-fmad=false"])]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    hdrs = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(ROOT, "include", "fargo_b200.h"))
    nv = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    jobs = [(s, os.path.basename(s) + ".o", []) for s in srcs]
    jobs += [(os.path.join(CSRC, s), o, f) for s, o, f in VARIANTS]
    for s, oname, extra in jobs:
        o = os.path.join(objdir, oname)
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            lang = [] if s.endswith(".cu") else ["-x", "cu"]
            cmd = [nv] + NVFLAGS + extra + ARCH + lang + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        if verbose and out:
            sys.stdout.write(out.decode())
    if force or _newer(LIB, objs):
        cmd = [nv] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcufft", "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    drv = os.path.join(CSRC, "driver", "fargo_main.cpp")
    if os.path.exists(drv) and (force or _newer(EXE, [drv, LIB] + hdrs)):
        cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), drv, "-o", EXE,
               "-L" + HERE, "-lfargo_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
