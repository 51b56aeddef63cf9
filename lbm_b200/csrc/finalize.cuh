// finalize.cuh -- the one-block reductions that turn fixed-slot block partial
// sums into the solver state (source mean, gauge target and shift, relative
// change, dual residual, mass) on the device.  Shared by the single-box
// finalize kernel and the per-instance finalize of the batched boxes.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "lbm_solver.cuh"

namespace lbm {
namespace {

__device__ __forceinline__ double relative(double num, double den)
{
    if (den > 0.0) return num / den;
    return num == 0.0 ? 0.0 : CUDART_INF;
}

// Sums T columns of a partials array (column t at part[t * stride], `count`
// entries) in a fixed order: thread i adds entries i, i + blockDim, ...
// sequentially, then a fixed tree (blockDim a power of two <= 1024).
template <int T>
__device__ void reduce_partials(const double* __restrict__ part, long long stride, long long count,
                                double (&out)[T])
{
    __shared__ double sm[1024];
    for (int t = 0; t < T; ++t) {
        double acc = 0.0;
        for (long long i = threadIdx.x; i < count; i += blockDim.x) acc += part[t * stride + i];
        sm[threadIdx.x] = acc;
        __syncthreads();
        for (int half = blockDim.x / 2; half > 0; half >>= 1) {
            if (threadIdx.x < half) sm[threadIdx.x] += sm[threadIdx.x + half];
            __syncthreads();
        }
        out[t] = sm[0];
        __syncthreads();
    }
}

__device__ __forceinline__ void set_error(DevState* ds, int site)
{
    if (ds->error == 0) {
        ds->error = 2;  // LBM_ERR_NONFINITE
        ds->error_site = site;
    }
}

// One finalisation step of kind `kind` (FinKind) for the box whose state is
// *ds; part/part2: its partial sums (part2: the dual-residual C terms).  All
// threads of the block call it.
__device__ void finalize_body(int kind, DevState* __restrict__ ds, const double* __restrict__ part,
                              long long stride, long long count, const double* __restrict__ part2,
                              long long stride2, long long count2)
{
    const double n = ds->n_cells;
    if (kind == FIN_SOURCE) {
        double r[3];
        reduce_partials<3>(part, stride, count, r);
        if (threadIdx.x == 0) {
            ds->div_sum = r[0];
            ds->div_abs_sum = r[1];
            ds->div_mean = r[0] / n;
            if (r[2] != 0.0 || !isfinite(r[0]) || !isfinite(r[1])) set_error(ds, SITE_SOURCE);
        }
    } else if (kind == FIN_PREP) {
        double r[3];
        reduce_partials<3>(part, stride, count, r);
        if (threadIdx.x == 0) {
            ds->proj_sum = r[0];
            if (r[1] != 0.0 || !isfinite(r[0])) set_error(ds, SITE_PROJECTED);
            ds->target = r[2] / n;
            if (!isfinite(r[2])) set_error(ds, SITE_GAUGE_TARGET);
            ds->max_shift = 0.0;
            ds->iterations = 0;
            ds->converged = 0;
        }
    } else if (kind == FIN_SIGMA) {
        double r[1];
        reduce_partials<1>(part, stride, count, r);
        if (threadIdx.x == 0) {
            const double shift = r[0] / n - ds->target;
            if (!isfinite(shift)) set_error(ds, SITE_GAUGE_SHIFT);
            ds->sigma = shift;
            if (fabs(shift) > ds->max_shift) ds->max_shift = fabs(shift);
        }
    } else if (kind == FIN_CHECK) {
        double rb[5];
        reduce_partials<5>(part, stride, count, rb);
        double rc[3] = {0.0, 0.0, 0.0};
        if (ds->dual) reduce_partials<3>(part2, stride2, count2, rc);
        if (threadIdx.x == 0) {
            bool fp_ok = true;
            if (ds->dual) {
                const double t[6] = {rc[0], rc[1], rc[2], rb[2], rb[3], rb[4]};
                for (int i = 0; i < 6; ++i) {
                    ds->fp_terms[i] = t[i];
                    if (!isfinite(t[i])) set_error(ds, SITE_FIXED_POINT);
                }
                ds->fp_h_scale = fmax(t[1], t[2]);
                ds->fp_h_rel = relative(t[0], ds->fp_h_scale);
                ds->fp_p_scale = fmax(t[4], t[5]);
                ds->fp_p_rel = relative(t[3], ds->fp_p_scale);
                ds->fp_rel = fmax(ds->fp_h_rel, ds->fp_p_rel);
                if (!isfinite(ds->fp_rel)) set_error(ds, SITE_FIXED_POINT);
                ds->fp_evaluated = 1;
                ds->fp_converged = ds->fp_rel < ds->tolerance;
                // dual == 2 is the shadow mode: reported, not part of the exit
                fp_ok = (ds->dual == 1) ? ds->fp_converged : true;
            }
            ds->l1_delta = rb[0];
            ds->l1_norm = rb[1];
            if (!isfinite(rb[0]) || !isfinite(rb[1])) set_error(ds, SITE_RESIDUAL);
            ds->rel = relative(rb[0], rb[1]);
            if (!isfinite(ds->rel)) set_error(ds, SITE_RESIDUAL);
            ds->pressure_converged = ds->rel < ds->tolerance;
            ds->converged = ds->pressure_converged && fp_ok;
            ds->iterations += (unsigned long long)ds->check_interval;
        }
    } else if (kind == FIN_MASS) {
        double r[1];
        reduce_partials<1>(part, stride, count, r);
        if (threadIdx.x == 0) ds->mass = r[0];
    } else if (kind == FIN_BLOCK) {
        double r[1];
        reduce_partials<1>(part, stride, count, r);
        if (threadIdx.x == 0) ds->block_frac = ds->l1_delta > 0.0 ? r[0] / ds->l1_delta : 0.0;
    } else if (kind == FIN_RHS) {
        double r[3];
        reduce_partials<3>(part, stride, count, r);
        if (threadIdx.x == 0) {
            ds->rhs_mean = r[0] / r[2];
            ds->rhs_chk = r[1] / r[2];
            if (!isfinite(r[0]) || !isfinite(r[1])) set_error(ds, SITE_PROJECTED);
        }
    }
}

}  // namespace
}  // namespace lbm
