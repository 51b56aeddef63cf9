// exact_div.cuh -- correctly rounded FP64 quotients from a reciprocal
// computed once per divisor.
//
// The FP64 kernels keep the reference's operation order, divisions included.
// The kinetic collision divides the 15 populations of a cell by the same
// tau_h, (h - E p) / tau_h, so the Poisson kernels compute y = RN(1/tau_h)
// once per cell (an IEEE division) and obtain every RN(a / tau_h) from it
// with remainder corrections (P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990, the final
// steps of FMA-based division; J.-M. Muller et al., Handbook of
// Floating-Point Arithmetic, chapter on division with an FMA):
//   q0 = RN(a y)                        within 1.5 ulp of a/b (y = RN(1/b))
//   q1 = RN(q0 + RN(a - b q0) y)        faithful
//   q2 = RN(q1 + (a - b q1) y)          = RN(a/b): with q1 faithful the
//                                        remainder a - b q1 is exact
// Numerators outside [2^-900, 2^900] in magnitude (zero, subnormal, huge,
// non-finite), where the remainders may underflow or overflow, take the IEEE
// division.  Divisors must be normal and finite.  lbm_selftest_division
// (selftest.cu) checks the result against CUDA's IEEE division.
#pragma once

#include <cuda_runtime.h>

namespace lbm {

__device__ __forceinline__ double div_rn(double a, double b, double y)
{
    const double m = fabs(a);
    if (!(m >= 0x1p-900 && m <= 0x1p+900)) return a / b;
    double q = a * y;
    double r = __fma_rn(-q, b, a);
    q = __fma_rn(r, y, q);
    r = __fma_rn(-q, b, a);
    return __fma_rn(r, y, q);
}

}  // namespace lbm
