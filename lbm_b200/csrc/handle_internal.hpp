// handle_internal.hpp -- library-internal access to an FP64 box's device
// state, for drivers built on lbm_handle (the adjoint runs of
// adjoint_run.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include "../../include/lbm_b200.h"
#include "lbm_solver.cuh"

namespace lbm {

// Device pointers of the current state of an FP64 box: the post-collision
// populations the next step pulls (f, g), the macro fields and the h the last
// Poisson solve ended with (h_last).
struct Fp64View {
    Geom geom;
    Phys phys;
    Launch L;
    cudaStream_t stream;
    double* f;
    double* gpop;
    double* macro[6];   // phi, rho, u, v, w, p
    double* h_last;
};

// LBM_ERR_BAD_ARG for a mixed-precision handle.
lbm_status fp64_view(lbm_handle* h, Fp64View* out);

// ---- precision-independent state access (FP64 or mixed box) -----------------
// Geometry, physics, launch shape and stream of a box of either precision.
struct BoxInfo {
    Geom geom;
    Phys phys;
    Launch L;
    cudaStream_t stream;
    lbm_precision precision;
};
lbm_status box_info(lbm_handle* h, BoxInfo* out);
// Bytes of one saved state: what the next step reads (post-collision
// populations in the box's own storage, the macro fields, p).  FP64 box:
// 288 B per cell; mixed box: 156 B per cell (FP32 populations and fields,
// FP64 rest population and p).
size_t box_state_bytes(const lbm_handle* h);
// Copies the current state into dst (device memory, box_state_bytes), or
// makes a saved state current (a restored box is past its first step: its
// next Poisson solve starts from h = E p).  Enqueued on the box's stream.
lbm_status box_save_state(lbm_handle* h, void* dst);
lbm_status box_restore_state(lbm_handle* h, const void* src);
// FP64 copies of the six macro fields (macro6: 6 n doubles, phi rho u v w p)
// and, when h15 is not null, of the h the last Poisson solve ended with
// (15 n doubles, q-major); the mixed box converts its FP32 fields.
lbm_status box_export(lbm_handle* h, double* macro6, double* h15);

// Makes (f, g, macro fields) the box's current state between two steps of a
// run that is past its first step: the next step pulls f and g and starts its
// Poisson solve from h = E p, as every step after the first does.
lbm_status fp64_restore(lbm_handle* h, const double* f, const double* gpop, const double* const macro[6]);

}  // namespace lbm
