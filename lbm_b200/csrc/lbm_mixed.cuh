// lbm_mixed.cuh -- the mixed-precision box: FP32 populations stored as
// deviations from rest-state values, FP32 stencils, FP64 reductions,
// convergence test and pressure accumulation (kernels_mixed.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/lbm_b200.h"
#include "lbm_solver.cuh"

namespace lbm {

struct MixedBuffers {
    float* f[2] = {nullptr, nullptr};   // moving populations q >= 1 (slot q = 0 unused)
    double* f0 = nullptr;               // rest population f_0 - f_rest,0 in FP64 (updated in place)
    float* g[2] = {nullptr, nullptr};
    float* h[2] = {nullptr, nullptr};
    float* hc = nullptr;
    float *phi = nullptr, *rho = nullptr, *u = nullptr, *v = nullptr, *w = nullptr;
    float* s = nullptr;
    double *p = nullptr, *p_prev = nullptr, *p_chk = nullptr;
    float *dux = nullptr, *dvy = nullptr, *dwz = nullptr;
    double *part_src = nullptr, *part_prep = nullptr, *part_a = nullptr, *part_b = nullptr,
           *part_c = nullptr, *part_mass = nullptr;
    double* scratch = nullptr;   // FP64 staging for loads/downloads (n doubles)
    // Iterative refinement of the Poisson solve (LBM_POISSON_REFINE): the FP64
    // post-collision populations (two buffers) and the FP32 residual.
    double* hd[2] = {nullptr, nullptr};
    float* rr = nullptr;
    int fuse_zlen = 0;           // >0: plain sweeps run two per pass, z runs of this length
    int collide_zlen = 0;        // >0: z-marching collide, z runs of this length
    bool allocated = false;
};

lbm_status mixed_alloc(MixedBuffers& mb, const Geom& g, const Launch& L);
lbm_status mixed_alloc_dual(MixedBuffers& mb, const Geom& g);
void mixed_free(MixedBuffers& mb);
lbm_status mixed_load(cudaStream_t st, MixedBuffers& mb, const Geom& g, const Phys& P,
                      const double* const src[6], cudaMemcpyKind kind);
lbm_status mixed_download(cudaStream_t st, MixedBuffers& mb, const Geom& g, int which, double* host);
// Launches collide, moments, source prep and the Poisson initial collision.
// ev (may be null) receives events 1 and 2 after collide and moments.
lbm_status mixed_prologue(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g,
                          const Phys& P, bool first, int fcur, bool h_loaded, DevState* ds,
                          cudaEvent_t* ev);
// Enqueues one Poisson segment (captured into a graph by the caller); returns
// the parity of the h buffer that holds the state afterwards.
int mixed_segment(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g,
                  int start_parity, int n_normal, bool dual, DevState* ds);
void mixed_correct(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g);
// Iterative refinement of the kinetic Poisson solve: allocates hd and rr (all
// or nothing); refine_init starts hd[0] from the prologue's p (or the loaded
// h); refine_segment enqueues one segment (an FP64 residual, n_normal - 1 FP32
// correction sweeps, FP64 checks A and B) and returns the hd buffer it ends
// in; refine_finish copies hd[parity] into the FP32 h[parity].
lbm_status mixed_alloc_refine(MixedBuffers& mb, const Geom& g);
void mixed_refine_init(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g, bool h_loaded);
int mixed_refine_segment(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g, int start_parity,
                         int n_normal, DevState* ds);
void mixed_refine_finish(cudaStream_t st, MixedBuffers& mb, const Geom& g, int parity);
// Saved state of a mixed box (the post-collision populations of buffer fcur,
// the rest population, the five FP32 macro fields and p): its size in bytes,
// and the copies in each direction.  Enqueued on st.
size_t mixed_state_bytes(const Geom& g);
lbm_status mixed_save_state(cudaStream_t st, const MixedBuffers& mb, const Geom& g, int fcur, void* dst);
lbm_status mixed_restore_state(cudaStream_t st, MixedBuffers& mb, const Geom& g, int fcur, const void* src);
// FP64 copies of the six macro fields and (h15 not null) of h buffer hbuf.
lbm_status mixed_export(cudaStream_t st, const MixedBuffers& mb, const Geom& g, int hbuf, double* macro6,
                        double* h15);
// Device pointer of a field: float for phi..w, double for p.
const void* mixed_field_ptr(const MixedBuffers& mb, int which);

}  // namespace lbm
