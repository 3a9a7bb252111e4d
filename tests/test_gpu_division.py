"""The divisions of csrc/fast_div.cuh against CUDA's IEEE division.

The CFL kernel divides by three per-ring constants (Rsup - Rinf, dxtheta and
their minimum) through their correctly rounded reciprocals: q0 = RN(x r),
e = x - q0 d (one fused multiply-add), q = RN(q0 + e r).  The quotient must
equal the IEEE division bit for bit, or the dt of a substep (hence the
substep count and every FARGO shift) could move away from the reference's.

The rounding of x/d depends only on the significands of x and d while
nothing overflows or underflows, so two checks cover it:
- every denominator of the benchmark grids (C1-C5 and the sweep's five grid
  sizes) as the CFL kernel forms it, against all 2^23 numerator significands;
- every denominator significand against every numerator significand:
  2^46 pairs, the whole binary32 normal range.
Both run on the GPU with the product's own device function."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from cudaprotoplanetarydisksfloat_b200 import configs, grid_radii
from tests.helpers import make

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cudaprotoplanetarydisksfloat_b200", "csrc")

SRC = r'''
#include <cuda_runtime.h>
#include "fast_div.cuh"

// x runs over the 2^23 significands of [1, 2); d over the given values.
__global__ void k_check(const float* ds, int nd, unsigned long long* bad, unsigned* first) {
  const int di = blockIdx.y;
  if (di >= nd) return;
  const float d = ds[di];
  const float r = (float)(1.0 / (double)d);
  if (threadIdx.x == 0 && blockIdx.x == 0 && r != __frcp_rn(d)) atomicAdd(bad + 1, 1ull);
  for (unsigned m = blockIdx.x * blockDim.x + threadIdx.x; m < (1u << 23); m += gridDim.x * blockDim.x) {
    const float x = __uint_as_float(0x3f800000u | m);
    const float a = __fdiv_rn(x, d), b = div_by_recip(x, d, r);
    if (__float_as_uint(a) != __float_as_uint(b)) {
      if (atomicAdd(bad, 1ull) == 0ull) {
        first[0] = __float_as_uint(x);
        first[1] = __float_as_uint(d);
      }
    }
  }
}

// every denominator significand d in [1, 2) from lo to hi (exclusive)
__global__ void k_check_all(unsigned lo, unsigned hi, unsigned long long* bad, unsigned* first) {
  const unsigned md = lo + blockIdx.y * 65535u + blockIdx.z;
  if (md >= hi) return;
  const float d = __uint_as_float(0x3f800000u | md);
  const float r = (float)(1.0 / (double)d);
  for (unsigned m = blockIdx.x * blockDim.x + threadIdx.x; m < (1u << 23); m += gridDim.x * blockDim.x) {
    const float x = __uint_as_float(0x3f800000u | m);
    const float a = __fdiv_rn(x, d), b = div_by_recip(x, d, r);
    if (__float_as_uint(a) != __float_as_uint(b)) {
      if (atomicAdd(bad, 1ull) == 0ull) {
        first[0] = __float_as_uint(x);
        first[1] = __float_as_uint(d);
      }
    }
  }
}

// div_refined against the IEEE division: x over the 2^23 significands of
// [1, 2), d over the given values; counts quotients that differ and those
// more than one ulp away.
__global__ void k_check_refined(const float* ds, int nd, unsigned long long* bad) {
  const int di = blockIdx.y;
  if (di >= nd) return;
  const float d = ds[di];
  unsigned long long n1 = 0, n2 = 0;
  for (unsigned m = blockIdx.x * blockDim.x + threadIdx.x; m < (1u << 23); m += gridDim.x * blockDim.x) {
    const float x = __uint_as_float(0x3f800000u | m);
    const int a = (int)__float_as_uint(__fdiv_rn(x, d)), b = (int)__float_as_uint(div_refined(x, d));
    if (a != b) n1++;
    if (a - b > 1 || b - a > 1) n2++;
  }
  if (n1) atomicAdd(bad, n1);
  if (n2) atomicAdd(bad + 1, n2);
}

extern "C" int check_refined(const float* hd, int nd, unsigned long long* bad_out) {
  float* d = nullptr;
  unsigned long long* bad = nullptr;
  if (cudaMalloc(&d, sizeof(float) * nd) || cudaMalloc(&bad, 16)) return 1;
  cudaMemcpy(d, hd, sizeof(float) * nd, cudaMemcpyHostToDevice);
  cudaMemset(bad, 0, 16);
  for (int o = 0; o < nd; o += 65535) {
    const int n = nd - o < 65535 ? nd - o : 65535;
    k_check_refined<<<dim3(64, n), 256>>>(d + o, n, bad);
  }
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(bad_out, bad, 16, cudaMemcpyDeviceToHost);
  cudaFree(d);
  cudaFree(bad);
  return e != cudaSuccess;
}

extern "C" int check_values(const float* hd, int nd, unsigned long long* bad_out, unsigned* first_out) {
  float* d = nullptr;
  unsigned long long* bad = nullptr;
  unsigned* first = nullptr;
  if (cudaMalloc(&d, sizeof(float) * nd) || cudaMalloc(&bad, 16) || cudaMalloc(&first, 8)) return 1;
  cudaMemcpy(d, hd, sizeof(float) * nd, cudaMemcpyHostToDevice);
  cudaMemset(bad, 0, 16);
  cudaMemset(first, 0, 8);
  for (int o = 0; o < nd; o += 65535) {
    const int n = nd - o < 65535 ? nd - o : 65535;
    k_check<<<dim3(64, n), 256>>>(d + o, n, bad, first);
  }
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(bad_out, bad, 16, cudaMemcpyDeviceToHost);
  cudaMemcpy(first_out, first, 8, cudaMemcpyDeviceToHost);
  cudaFree(d);
  cudaFree(bad);
  cudaFree(first);
  return e != cudaSuccess;
}

extern "C" int check_all(unsigned long long* bad_out, unsigned* first_out) {
  unsigned long long* bad = nullptr;
  unsigned* first = nullptr;
  if (cudaMalloc(&bad, 16) || cudaMalloc(&first, 8)) return 1;
  cudaMemset(bad, 0, 16);
  cudaMemset(first, 0, 8);
  const unsigned step = 1u << 15;  // denominators per launch (~0.15 s each)
  for (unsigned lo = 0; lo < (1u << 23); lo += step) {
    k_check_all<<<dim3(32, 1, step), 256>>>(lo, lo + step, bad, first);
    if (cudaDeviceSynchronize() != cudaSuccess) return 2;
  }
  cudaMemcpy(bad_out, bad, 16, cudaMemcpyDeviceToHost);
  cudaMemcpy(first_out, first, 8, cudaMemcpyDeviceToHost);
  cudaFree(bad);
  cudaFree(first);
  return 0;
}
'''


@pytest.fixture(scope="module")
def divlib(gpu, tmp_path_factory):
    d = tmp_path_factory.mktemp("div")
    cu = d / "divcheck.cu"
    cu.write_text(SRC)
    so = d / "divcheck.so"
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    subprocess.check_call([nvcc, "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-I" + CSRC, "-shared",
                           "-Xcompiler", "-fPIC", "-o", str(so), str(cu)])
    lib = C.CDLL(str(so))
    lib.check_values.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.check_all.argtypes = [C.c_void_p, C.c_void_p]
    lib.check_refined.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    return lib


def _cfl_divisors(P):
    """Rsup - Rinf, dxtheta and their minimum per ring, as the library forms
    them (FP64 host formulas rounded to float, then the float subtraction)."""
    R = grid_radii(P)
    rinf = R[:-1].astype(np.float32)
    rsup = R[1:].astype(np.float32)
    rmed = (2.0 / 3.0 * (R[1:] ** 3 - R[:-1] ** 3) / (R[1:] ** 2 - R[:-1] ** 2)).astype(np.float32)
    dxr = rsup - rinf
    dxt = (2.0 * np.pi / np.float64(np.float32(P.NSEC)) * rmed.astype(np.float64)).astype(np.float32)
    return np.concatenate([dxr, dxt, np.minimum(dxr, dxt)])


def _run(lib, fn, *args):
    bad = np.zeros(2, np.uint64)
    first = np.zeros(2, np.uint32)
    st = fn(*args, bad.ctypes.data, first.ctypes.data)
    assert st == 0
    x, d = first.view(np.float32)
    return int(bad[0]), int(bad[1]), (x, d)


def test_markstein_division_benchmark_denominators(divlib):
    grids = [configs.c1(), configs.c2(), configs.c3(), configs.c5()]
    seen = set()
    for p, pl in configs.c4(64, seed=42):
        if p["Nrad"] not in seen:
            seen.add(p["Nrad"])
            grids.append((p, pl))
    ds = np.unique(np.concatenate([_cfl_divisors(make(p, pl, "div")[0]) for p, pl in grids]))
    nbad, nrcp, first = _run(divlib, divlib.check_values, ds.ctypes.data, len(ds))
    assert nrcp == 0, "a reciprocal is not the correctly rounded one"
    assert nbad == 0, ("quotient differs from the IEEE division", first)


def test_markstein_division_all_significand_pairs(divlib):
    nbad, _, first = _run(divlib, divlib.check_all)
    assert nbad == 0, ("quotient differs from the IEEE division", first)


def test_refined_division_within_one_ulp(divlib):
    """div_refined (the per-cell quotients by density sums): against the IEEE
    division for every numerator significand and 4096 denominators spread
    over 2^-40 .. 2^40, no quotient more than one ulp away and fewer than
    1e-5 of them different at all."""
    rng = np.random.default_rng(7)
    ds = (rng.uniform(1.0, 2.0, 4096) * np.exp2(rng.integers(-40, 41, 4096))).astype(np.float32)
    bad = np.zeros(2, np.uint64)
    assert divlib.check_refined(ds.ctypes.data, len(ds), bad.ctypes.data) == 0
    total = len(ds) * (1 << 23)
    print("\ndiv_refined: %d of %d quotients differ from IEEE (%.2e), %d by more than one ulp"
          % (int(bad[0]), total, int(bad[0]) / total, int(bad[1])))
    assert int(bad[1]) == 0
    assert int(bad[0]) < 1e-5 * total
