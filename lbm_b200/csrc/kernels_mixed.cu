// kernels_mixed.cu -- mixed-precision box (placeholder until the FP32
// kernels land): every entry reports that the precision is unavailable.
#include "lbm_mixed.cuh"

namespace lbm {

lbm_status mixed_alloc(MixedBuffers&, const Geom&, const Launch&) { return LBM_ERR_BAD_ARG; }
lbm_status mixed_alloc_dual(MixedBuffers&, const Geom&) { return LBM_ERR_BAD_ARG; }
void mixed_free(MixedBuffers&) {}
lbm_status mixed_load(cudaStream_t, MixedBuffers&, const Geom&, const Phys&, const double* const[6],
                      cudaMemcpyKind)
{
    return LBM_ERR_BAD_ARG;
}
lbm_status mixed_download(cudaStream_t, MixedBuffers&, const Geom&, int, double*) { return LBM_ERR_BAD_ARG; }
lbm_status mixed_prologue(cudaStream_t, MixedBuffers&, const Launch&, const Geom&, const Phys&, bool,
                          int, bool, DevState*, cudaEvent_t*)
{
    return LBM_ERR_BAD_ARG;
}
int mixed_segment(cudaStream_t, MixedBuffers&, const Launch&, const Geom&, int start_parity, int,
                  bool, DevState*)
{
    return start_parity;
}
void mixed_correct(cudaStream_t, MixedBuffers&, const Launch&, const Geom&) {}
const void* mixed_field_ptr(const MixedBuffers&, int) { return nullptr; }

}  // namespace lbm
