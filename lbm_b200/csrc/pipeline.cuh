// pipeline.cuh -- shared-memory producer/consumer pipelines inside one CTA:
// mbarrier arrive and bounded waits (mbarrier.try_wait.parity), used by the
// warp-specialized two-sweep passes.  A wait gives up after kPipeSpin polls
// (seconds) and the kernel records SITE_PIPELINE in the box's DevState, so a
// broken pipeline ends its launch with an error the host reads instead of
// hanging the GPU.
#pragma once

#include <cuda_runtime.h>

#include "lbm_solver.cuh"

namespace lbm {
namespace {

constexpr long long kPipeSpin = 1LL << 24;

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
// Arrival with release semantics (the caller's shared-memory writes become
// visible to the threads that complete a wait on this phase).
__device__ __forceinline__ void mbar_arrive(unsigned long long* b)
{
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(b))
                 : "memory");
}
// Waits (acquire) for the phase of the given parity to complete; false after
// kPipeSpin polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity)
{
    for (long long i = 0; i < kPipeSpin; ++i) {
        unsigned done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(smem_u32(b)), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void pipeline_fail(DevState* ds)
{
    if (atomicCAS(&ds->error, 0, static_cast<int>(LBM_ERR_CUDA)) == 0) ds->error_site = SITE_PIPELINE;
}

}  // namespace
}  // namespace lbm
