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

// Makes (f, g, macro fields) the box's current state between two steps of a
// run that is past its first step: the next step pulls f and g and starts its
// Poisson solve from h = E p, as every step after the first does.
lbm_status fp64_restore(lbm_handle* h, const double* f, const double* gpop, const double* const macro[6]);

}  // namespace lbm
