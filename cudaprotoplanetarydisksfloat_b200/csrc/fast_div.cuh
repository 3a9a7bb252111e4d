// fast_div.cuh -- division by a per-ring constant whose reciprocal is known.
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
