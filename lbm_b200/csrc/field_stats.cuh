// field_stats.cuh -- launch interface of the field-statistics reduction
// (field_stats.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/lbm_b200.h"

namespace lbm {

constexpr int kStatsTerms = 7;                 // sum, count, nan, inf, min, max, abs max
constexpr long long kStatsCellsPerBlock = 4096; // 256 threads x 16 cells

// Blocks of the partial pass for n cells; the scratch holds
// kStatsTerms * stats_blocks(n) doubles.
inline long long stats_blocks(long long n) { return (n + kStatsCellsPerBlock - 1) / kStatsCellsPerBlock; }

// Enqueues both passes on `st`; the result lands in *dev_out (device memory).
template <class T>
cudaError_t field_stats(cudaStream_t st, const T* f, long long n, double* partials,
                        lbm_field_stats* dev_out);

// The same for the velocity magnitude sqrt(u*u + v*v + w*w).
template <class T>
cudaError_t velmag_stats(cudaStream_t st, const T* u, const T* v, const T* w, long long n, double* partials,
                         lbm_field_stats* dev_out);

}  // namespace lbm
