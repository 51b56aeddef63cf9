// field_stats.cu -- device reduction of the per-field statistics of the
// reference's collectDiagnostics (CPU/Inamuro.cpp:412-507) and
// updateFieldStatistics / finalizeFieldStatistics (:1050-1092).
//
// Two passes, both in a fixed order (results are run-to-run identical):
//   stats_partial_kernel  block b reduces cells [4096 b, 4096 (b+1)): each of
//                         its 256 threads visits 16 cells (stride 256, so
//                         every warp load is coalesced), then a fixed
//                         shuffle/shared-memory tree
//   stats_final_kernel    one block folds the per-block partials
// The partials live in caller-provided global scratch (7 doubles per block).
#include <cuda_runtime.h>
#include <math_constants.h>


#include "../../include/lbm_b200.h"
#include "field_stats.cuh"

namespace lbm {
namespace {

enum { T_SUM = 0, T_CNT, T_NAN, T_INF, T_MIN, T_MAX, T_AMAX };

// Value sources of the partial pass: a field, or the velocity magnitude
// sqrt(u*u + v*v + w*w) of three fields (the reference's vel_mag, in FP64).
template <class T>
struct FieldSrc {
    const T* f;
    __device__ __forceinline__ double operator()(long long i) const { return static_cast<double>(f[i]); }
};

template <class T>
struct VelMagSrc {
    const T *u, *v, *w;
    __device__ __forceinline__ double operator()(long long i) const
    {
        const double a = static_cast<double>(u[i]), b = static_cast<double>(v[i]), c = static_cast<double>(w[i]);
        return sqrt(a * a + b * b + c * c);
    }
};

template <class Src>
__global__ void __launch_bounds__(256)
stats_partial_kernel(Src src, long long n, double* __restrict__ part, long long nblocks)
{
    double v[kStatsTerms] = {0.0, 0.0, 0.0, 0.0, CUDART_INF, -CUDART_INF, 0.0};
    const long long base = (long long)blockIdx.x * kStatsCellsPerBlock + threadIdx.x;
#pragma unroll 4
    for (int k = 0; k < kStatsCellsPerBlock / 256; ++k) {
        const long long i = base + 256LL * k;
        if (i < n) {
            const double x = src(i);
            if (isnan(x)) {
                v[T_NAN] += 1.0;
            } else if (isinf(x)) {
                v[T_INF] += 1.0;
            } else {
                v[T_SUM] += x;
                v[T_CNT] += 1.0;
                v[T_MIN] = fmin(v[T_MIN], x);
                v[T_MAX] = fmax(v[T_MAX], x);
                v[T_AMAX] = fmax(v[T_AMAX], fabs(x));
            }
        }
    }
    __shared__ double red[8][kStatsTerms];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < kStatsTerms; ++t) {
        double s = v[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double other = __shfl_xor_sync(0xffffffffu, s, o);
            s = (t == T_MIN) ? fmin(s, other) : (t >= T_MAX) ? fmax(s, other) : s + other;
        }
        if (lane == 0) red[warp][t] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < kStatsTerms; ++t) {
            const double ident = (t == T_MIN) ? CUDART_INF : (t == T_MAX) ? -CUDART_INF : 0.0;
            double s = lane < 8 ? red[lane][t] : ident;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double other = __shfl_xor_sync(0xffffffffu, s, o);
                s = (t == T_MIN) ? fmin(s, other) : (t >= T_MAX) ? fmax(s, other) : s + other;
            }
            if (lane == 0) part[(long long)t * nblocks + blockIdx.x] = s;
        }
    }
}

__global__ void __launch_bounds__(1024)
stats_final_kernel(const double* __restrict__ part, long long nblocks, lbm_field_stats* __restrict__ out)
{
    __shared__ double sm[1024];
    double r[kStatsTerms];
    for (int t = 0; t < kStatsTerms; ++t) {
        const double ident = (t == T_MIN) ? CUDART_INF : (t == T_MAX) ? -CUDART_INF : 0.0;
        double acc = ident;
        for (long long i = threadIdx.x; i < nblocks; i += blockDim.x) {
            const double x = part[(long long)t * nblocks + i];
            acc = (t == T_MIN) ? fmin(acc, x) : (t >= T_MAX) ? fmax(acc, x) : acc + x;
        }
        sm[threadIdx.x] = acc;
        __syncthreads();
        for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
            if (threadIdx.x < stride) {
                const double a = sm[threadIdx.x], b = sm[threadIdx.x + stride];
                sm[threadIdx.x] = (t == T_MIN) ? fmin(a, b) : (t >= T_MAX) ? fmax(a, b) : a + b;
            }
            __syncthreads();
        }
        r[t] = sm[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        lbm_field_stats s;
        const unsigned long long valid = static_cast<unsigned long long>(r[T_CNT]);
        s.valid_count = valid;
        s.nan_count = static_cast<unsigned long long>(r[T_NAN]);
        s.inf_count = static_cast<unsigned long long>(r[T_INF]);
        s.sum = r[T_SUM];
        if (valid == 0) {
            s.min = s.max = s.mean = s.abs_max = CUDART_NAN;
        } else {
            s.min = r[T_MIN];
            s.max = r[T_MAX];
            s.abs_max = r[T_AMAX];
            s.mean = r[T_SUM] / static_cast<double>(valid);
        }
        *out = s;
    }
}

}  // namespace

template <class T>
cudaError_t field_stats(cudaStream_t st, const T* f, long long n, double* partials,
                        lbm_field_stats* dev_out)
{
    const long long nb = stats_blocks(n);
    if (nb <= 0 || nb > 0x7fffffffLL) return cudaErrorInvalidValue;
    stats_partial_kernel<<<static_cast<unsigned>(nb), 256, 0, st>>>(FieldSrc<T>{f}, n, partials, nb);
    stats_final_kernel<<<1, 1024, 0, st>>>(partials, nb, dev_out);
    return cudaGetLastError();
}

template <class T>
cudaError_t velmag_stats(cudaStream_t st, const T* u, const T* v, const T* w, long long n, double* partials,
                         lbm_field_stats* dev_out)
{
    const long long nb = stats_blocks(n);
    if (nb <= 0 || nb > 0x7fffffffLL) return cudaErrorInvalidValue;
    stats_partial_kernel<<<static_cast<unsigned>(nb), 256, 0, st>>>(VelMagSrc<T>{u, v, w}, n, partials, nb);
    stats_final_kernel<<<1, 1024, 0, st>>>(partials, nb, dev_out);
    return cudaGetLastError();
}

template cudaError_t field_stats<double>(cudaStream_t, const double*, long long, double*, lbm_field_stats*);
template cudaError_t field_stats<float>(cudaStream_t, const float*, long long, double*, lbm_field_stats*);
template cudaError_t velmag_stats<double>(cudaStream_t, const double*, const double*, const double*, long long,
                                          double*, lbm_field_stats*);
template cudaError_t velmag_stats<float>(cudaStream_t, const float*, const float*, const float*, long long, double*,
                                         lbm_field_stats*);

}  // namespace lbm

// ---- lbm_field_statistics_noalloc ----------------------------------------
// The same two passes with their scratch in a statically sized device array,
// for callers that cannot allocate device memory (include/lbm_b200.h).
namespace {

constexpr long long kNoAllocMaxBlocks = 8192;   // x 4096 cells = LBM_NOALLOC_MAX_CELLS
static_assert(kNoAllocMaxBlocks * lbm::kStatsCellsPerBlock == (long long)LBM_NOALLOC_MAX_CELLS,
              "header limit and scratch capacity disagree");

struct NoAllocScratch {
    double partials[lbm::kStatsTerms * kNoAllocMaxBlocks];
    lbm_field_stats result;
};

// One instance per device that loads the library, reserved until exit.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

}  // namespace

// In host code `g_noalloc_scratch` names a host-side shadow, not device
// memory.  Its device address is looked up on every call, with the caller's
// device current: the lookup allocates nothing, and a cached address would go
// stale if the caller reset the device (a new primary context reloads the
// module at another address).
extern "C" lbm_status lbm_field_statistics_noalloc(const double* field, uint64_t n_cells, void* stream,
                                                   lbm_field_stats* out)
{
    if (!field || !out || n_cells == 0 || n_cells > LBM_NOALLOC_MAX_CELLS) return LBM_ERR_BAD_ARG;
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) return LBM_ERR_CUDA;
    NoAllocScratch* scratch = static_cast<NoAllocScratch*>(addr);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (lbm::field_stats<double>(st, field, static_cast<long long>(n_cells), scratch->partials,
                                 &scratch->result) != cudaSuccess)
        return LBM_ERR_CUDA;
    if (cudaMemcpyAsync(out, &scratch->result, sizeof(lbm_field_stats), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return LBM_ERR_CUDA;
    return LBM_OK;
}
