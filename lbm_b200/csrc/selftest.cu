// selftest.cu -- lbm_selftest_division: the FP64 kernels' correctly rounded
// division from a reciprocal (exact_div.cuh) against CUDA's IEEE division on
// pseudo-random operands of the kinds the kernels use.
#include <cuda_runtime.h>

#include "../../include/lbm_b200.h"
#include "exact_div.cuh"

namespace {

__device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    // splitmix64 finaliser (S. Vigna), used as a counter-based generator
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// A normal double with a random significand, an exponent in [emin, emax] and,
// if `sign`, a random sign.
__device__ __forceinline__ double random_double(unsigned long long r, int emin, int emax, bool sign)
{
    const unsigned long long mant = r & ((1ULL << 52) - 1);
    const int e = emin + static_cast<int>((r >> 52) % static_cast<unsigned long long>(emax - emin + 1));
    const unsigned long long bits = (sign && (r >> 63) ? (1ULL << 63) : 0ULL) |
                                    (static_cast<unsigned long long>(e + 1023) << 52) | mant;
    return __longlong_as_double(static_cast<long long>(bits));
}

__global__ void division_selftest_kernel(unsigned long long n, unsigned long long seed,
                                         unsigned long long* __restrict__ mismatches)
{
    unsigned long long bad = 0;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long r1 = mix64(seed ^ (2 * i)), r2 = mix64(seed ^ (2 * i + 1));
        const double a = random_double(r1, -320, 320, true);
        double b;
        switch (r2 & 7) {
        case 0: b = 10.0; break;
        case 1: b = 5.0; break;
        case 2: b = 6.0; break;
        case 3: b = random_double(r2, -1, 0, false); break;        // relaxation times in [0.5, 2)
        case 4: b = random_double(r2, -10, 10, false); break;      // densities
        default: b = random_double(r2, -200, 200, true); break;   // any normal divisor
        }
        const double y = 1.0 / b;
        const double q = lbm::div_rn(a, b, y);
        const double ref = __ddiv_rn(a, b);
        if (__double_as_longlong(q) != __double_as_longlong(ref)) ++bad;
    }
    if (bad) atomicAdd(mismatches, bad);
}

}  // namespace

extern "C" lbm_status lbm_selftest_division(uint64_t samples, uint64_t seed, uint64_t* mismatches)
{
    if (!mismatches) return LBM_ERR_BAD_ARG;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, sizeof(unsigned long long)) != cudaSuccess) return LBM_ERR_OOM;
    cudaMemset(d, 0, sizeof(unsigned long long));
    division_selftest_kernel<<<148 * 8, 256>>>(samples, seed, d);
    unsigned long long h = 0;
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(d);
    if (!ok) return LBM_ERR_CUDA;
    *mismatches = h;
    return LBM_OK;
}
