// fast_div.cuh -- divisions without CUDA's IEEE division sequence.
//
// div_by_recip: division by a per-ring constant whose reciprocal is known.
//
// Markstein's method (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; the
// correction step of Theorem 8.10 in Muller et al., Handbook of
// Floating-Point Arithmetic): with r = RN(1/d), the correctly rounded
// reciprocal, q0 = RN(x r) and the residual e = x - q0 d, exact in one fused
// multiply-add, q = RN(q0 + e r) is RN(x/d): the IEEE quotient, bit for bit.
// It is checked exhaustively on the GPU against CUDA's IEEE division for
// every pair of significands of the benchmark grids' denominators and for a
// sample of all others (tests/test_gpu_division.py).  Valid for normal x, d
// and quotients (no underflow or overflow on the way); x = 0 gives 0.
#pragma once

__device__ __forceinline__ float div_by_recip(float x, float d, float r) {
  const float q0 = __fmul_rn(x, r);
  const float e = __fmaf_rn(-q0, d, x);
  return __fmaf_rn(e, r, q0);
}

// x / y for per-cell operands: the hardware's approximate reciprocal
// (rcp.approx, relative error below 2^-22), then the same residual
// correction: q0 = RN(x r), e = x - q0 y exact in one fused multiply-add,
// q = RN(q0 + e r).  The correction leaves q0's error times r's, so q is the
// IEEE quotient except when x/y lies within ~2^-22 ulp of a rounding
// boundary, and one ulp from it then (tests/test_gpu_division.py counts
// both).  For normal y and quotient; four instructions against the IEEE
// sequence's ~ten with its special-case branch.
__device__ __forceinline__ float rcp_approx(float y) {
  float r;
  asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(y));
  return r;
}
__device__ __forceinline__ float div_refined(float x, float y) {
  const float r = rcp_approx(y);
  const float q0 = __fmul_rn(x, r);
  return __fmaf_rn(__fmaf_rn(-q0, y, x), r, q0);
}
