// lbm_solver.cuh -- structures shared by the host orchestration (lbm_capi.cu)
// and the kernels (kernels_fp64.cu, kernels_mixed.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/lbm_b200.h"
#include "lbm_device.cuh"

namespace lbm {

// Physical constants of one box, with the derived constants the reference
// computes at run time folded here in the same IEEE operations.
struct Phys {
    double rho_L, rho_G;
    double mu_G;
    double mu_slope;      // (mu_L - mu_G) / (rho_L - rho_G)      CPU/Inamuro.cpp:137
    double tauf, taug;
    double k_f, k_g;
    double T, a, b;
    double fei_L, fei_G;
    double fei_avg;       // (fei_L + fei_G) / 2.0                CPU/Inamuro.cpp:296
    double dfei;          // fei_L - fei_G
    double half_drho;     // (rho_L - rho_G) / 2.0                CPU/Inamuro.cpp:326
    double visc;          // 1.5 * (taug - 0.5) * 2.0             CPU/Inamuro.cpp:217
    double inv_tauf, inv_taug;
    int tauf_pow2, taug_pow2;   // 1: tau is a power of two, x/tau == x*(1/tau) exactly
};

// Device-resident solver state: the scalars the reference computes on the
// host between kernel launches (GPU/InamuroCUDA.cu:1868-2159) live here, so a
// whole Poisson segment runs without a host round trip.
struct DevState {
    // source projection and gauge (per step)
    double div_sum, div_abs_sum, div_mean;
    double proj_sum;
    double target;              // pressure gauge target (mean p at solve start)
    // last check
    double sigma;               // gauge shift
    double max_shift;
    double l1_delta, l1_norm, rel;
    double fp_terms[6];
    double fp_h_scale, fp_h_rel, fp_p_scale, fp_p_rel, fp_rel;
    double mass;
    unsigned long long iterations;   // sweeps counted up to the last check
    int converged, pressure_converged, fp_converged, fp_evaluated;
    int error;                  // lbm_status code, 0 = ok
    int error_site;             // which check raised it
    int check_interval;
    int dual;
    double tolerance;
    double n_cells;             // (double)lx * ly * lz
    double rhs_mean;            // scalar red-black form: weighted mean of f = scale rho s (per step)
    double rhs_chk;             // ... and of chi f, chi = (-1)^(x+y+z)
    double block_frac;          // spatial diagnostics: sum |4^3 block sums of the change| / l1_delta
};

enum ErrorSite {
    SITE_NONE = 0,
    SITE_SOURCE = 1,        // "Poisson source contains NaN/Inf"
    SITE_PROJECTED = 2,     // "projected Poisson source contains NaN/Inf"
    SITE_GAUGE_TARGET = 3,  // "pressure mean is NaN/Inf"
    SITE_GAUGE_SHIFT = 4,   // "pressure gauge shift is NaN/Inf"
    SITE_FIXED_POINT = 5,   // "kinetic fixed-point residual contains NaN/Inf"
    SITE_RESIDUAL = 6       // "Poisson pressure/residual contains NaN/Inf"
};

// Launch shape: 2-D tiles of (bx, by) cells in an xy plane, one grid z-slice
// per lattice plane.
// The Poisson check kernels (A, B, C) use the same tiles but let one CTA
// cover runs of `zrun` planes (cgrid, cnblocks partial sums).
constexpr int kCheckZrun = 8;

struct Launch {
    dim3 grid, block;
    long long nblocks;
    dim3 cgrid;
    long long cnblocks;
    int zrun;
};

inline Launch make_launch(int lx, int ly, int lz, int bx, int by)
{
    Launch L;
    L.block = dim3(bx, by, 1);
    L.grid = dim3((lx + bx - 1) / bx, (ly + by - 1) / by, lz);
    L.nblocks = (long long)L.grid.x * L.grid.y * L.grid.z;
    L.zrun = kCheckZrun;
    L.cgrid = dim3(L.grid.x, L.grid.y, (lz + kCheckZrun - 1) / kCheckZrun);
    L.cnblocks = (long long)L.cgrid.x * L.cgrid.y * L.cgrid.z;
    return L;
}

// Buffers of one FP64 box.  Populations are q-major SoA: a[q*n + cell].
struct Fp64Buffers {
    double* f[2];       // post-collision f* ping-pong
    double* g[2];
    double* h[2];       // post-collision h* ping-pong (and h0 after a load)
    double* hc;         // gauged h at a check (dual residual only)
    double *phi, *rho, *u, *v, *w;
    double *p, *p_prev, *p_chk;
    double *dux, *dvy, *dwz, *s;
    double *part_src, *part_prep, *part_a, *part_b, *part_c, *part_mass;
};

// Kernel launchers (kernels_fp64.cu).
namespace fp64 {
// Collide: the z-marching form when zlen > 0 (collide_zm_prepare returned 1
// for the box), else one CTA per plane tile.  Returns the number of source
// partial-sum blocks written to part.
int collide_zm_prepare(const Geom& g);
long long collide(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P, bool first, int zlen,
                  const double* fin, double* fout, const double* gin, double* gout,
                  const double* phi, const double* rho, const double* u, const double* v,
                  const double* w, double* dux, double* dvy, double* dwz, double* part);
void moments(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P,
             const double* f, const double* gpop, double* phi, double* rho, double* u,
             double* v, double* w, double* part_mass);
void prep(cudaStream_t st, const Launch& L, const Geom& g, const DevState* ds,
          const double* dux, const double* dvy, const double* dwz, const double* p,
          double* s, double* part);
void poisson_init(cudaStream_t st, const Launch& L, const Geom& g, bool h_loaded,
                  const double* hload, double* hout, const double* p, const double* rho,
                  const double* s, bool source_aware = false,
                  double sa_scale = 1.0);
void sweep(cudaStream_t st, const Launch& L, const Geom& g, const double* hin, double* hout,
           const double* rho, const double* s);
// Two sweeps per launch (temporal blocking).  sweep2_prepare returns 1 when
// the box admits it (lx % 32 == 0, ly % 4 == 0) and the kernel is set up.
int sweep2_prepare(const Geom& g);
void sweep2(cudaStream_t st, const Geom& g, int zlen, const double* hin, double* hout,
            const double* rho, const double* s);
void sweep_check_a(cudaStream_t st, const Launch& L, const Geom& g, const double* hin,
                   double* hout, double* p_chk, double* part);
void sweep_check_b(cudaStream_t st, const Launch& L, const Geom& g, bool dual, const double* hin, double* hout,
                   double* hc, const double* p_chk, double* p_prev, double* p,
                   const double* rho, const double* s, const DevState* ds, double* part);
void sweep_check_c(cudaStream_t st, const Launch& L, const Geom& g, const double* hin,
                   double* hout, const double* hc, const double* rho, const double* s,
                   const DevState* ds, double* part);
void correct(cudaStream_t st, const Launch& L, const Geom& g, double* u, double* v, double* w,
             const double* p, const double* rho);
// Scalar Poisson forms: a Jacobi sweep of the reference's scalar form, a
// red-black SOR sweep (two launches) of the same equation, the partial sums
// of its right-hand side (FIN_RHS) and of p (FIN_SIGMA), and the check
// (gauge, relative change; FIN_CHECK layout).
void scalar_jacobi(cudaStream_t st, const Launch& L, const Geom& g, const double* pin, double* pout,
                   const double* rho, const double* s, double scale);
// Variable-coefficient form: one red-black SOR sweep of div((1/rho) grad p) = s
// (two launches) and the operator residual terms of a check (3 columns).
void rb_varcoef(cudaStream_t st, const Launch& L, const Geom& g, double* p, const double* rho, const double* s,
                double omega, const DevState* ds);
void varcoef_residual(cudaStream_t st, const Launch& L, const Geom& g, const double* p, const double* rho,
                      const double* s, const DevState* ds, double* part);
void rb_sor(cudaStream_t st, const Launch& L, const Geom& g, double* p, const double* rho, const double* s,
            double scale, double omega, const DevState* ds);
void scalar_rhs_sum(cudaStream_t st, const Launch& L, const Geom& g, const double* rho, const double* s,
                    double scale, double* part);
void p_sum(cudaStream_t st, const Launch& L, const Geom& g, const double* p, double* part);
void scalar_check(cudaStream_t st, const Launch& L, const Geom& g, const double* pin, double* p, double* p_prev,
                  const DevState* ds, double* part);
// The reference's one-pass form on the pre-collision h: start state, sweep
// (relaxation scale, fixed-point relaxation), Anderson-m1 (store, dot
// partials over kAndersonBlocks blocks, apply), the check (gauge of p and h,
// relative change, results into the parity-0 buffers) and the two-grid
// correction (4^3 block sums of the change, correction).
constexpr int kAndersonBlocks = 296;
void onepass_init(cudaStream_t st, const Launch& L, const Geom& g, bool h_loaded, const double* hload, double* hh,
                  const double* p, const double* rho, const double* s, bool source_aware, double sa_scale);
void onepass_sweep(cudaStream_t st, const Launch& L, const Geom& g, const double* hin, double* hout, const double* pin,
                   double* pout, const double* rho, const double* s, double relax, double omega);
void anderson_store(cudaStream_t st, const Geom& g, const double* hold, const double* himg, double* prev_r,
                    double* prev_img);
void anderson_dot(cudaStream_t st, const Geom& g, const double* hold, const double* himg, const double* prev_r,
                  double* part);
void anderson_apply(cudaStream_t st, const Launch& L, const Geom& g, const double* hold, double* himg, double* prev_r,
                    double* prev_img, double* pimg, double alpha);
void onepass_check(cudaStream_t st, const Launch& L, const Geom& g, const double* hin, double* hout, const double* pin,
                   double* p, double* p_prev, const DevState* ds, double* part);
int twogrid_blocks(const Geom& g, int* bxn, int* byn, int* bzn);
void twogrid_sums(cudaStream_t st, const Geom& g, const double* p, const double* p_prev, const DevState* ds,
                  double* bsum);
void twogrid_correct(cudaStream_t st, const Launch& L, const Geom& g, double* hh, double* p, double* p_prev,
                     const double* bsum, double strength, const DevState* ds);
// Partial sums (kAndersonBlocks blocks) of |bsum| over the 4^3 blocks (FIN_BLOCK).
void block_abs_sum(cudaStream_t st, const Geom& g, const double* bsum, double* part);
}  // namespace fp64

// BiCGSTAB on the kinetic fixed point (krylov.cu).  Work vectors of 15 n
// doubles; part/host: at least 3 * max(L.nblocks, kKrylovBlocks) doubles
// (host pinned).  kKrylovBlocks: grid of the vector updates (8 per SM).
constexpr int kKrylovBlocks = 1184;
struct KrylovBuffers {
    double *r, *r0, *p, *v, *s, *t;
    double* part;
    double* host;
    double *w1, *w2, *bm;   // polynomial form (degree > 1): powers of the operator, right-hand side
};
struct KrylovResult {
    uint64_t matvecs = 0;      // applications of (I - K): two per iteration plus the initial residual
    uint64_t iterations = 0;
    uint64_t restarts = 0;     // restarts from the true residual (near-breakdown, every 200 iterations)
    double rel_residual = 0.0; // ||b - (I - K) h|| / ||b|| at exit (the recurrence's)
    double gauge_shift = 0.0;
};
namespace krylov {
// h: initial guess in, solution out (post-collision populations); p, p_prev:
// the solution's p gauged to `target`.  Stops at ||r|| < tol ||b||;
// LBM_ERR_POISSON_BUDGET past max_matvecs applications (0: no cap),
// LBM_ERR_NONFINITE on a breakdown or a non-finite residual.
// degree > 1: BiCGSTAB on the polynomially preconditioned system
// (I - K^m) h = (I + K + ... + K^(m-1)) b, m = degree (kb.w1, w2, bm needed).
lbm_status solve(cudaStream_t st, const Launch& L, const Geom& g, const KrylovBuffers& kb, double* h, const double* rho,
                 const double* s, double* p, double* p_prev, double target, double tol, uint64_t max_matvecs,
                 int degree, KrylovResult* res);
// The adjoint Poisson problem y = M^T (pull from x + c_q of y) + lam_p
// (periodic boxes) by the same method: y initial guess in, solution out.
lbm_status solve_adjoint(cudaStream_t st, const Launch& L, const Geom& g, const KrylovBuffers& kb, double* y,
                         const double* rho, const double* lp, double tol, uint64_t max_matvecs, KrylovResult* res);
}  // namespace krylov

// Finalisation kernels (kernels_fp64.cu): reduce block partials in a fixed
// order and update DevState.
enum FinKind { FIN_SOURCE = 0, FIN_PREP = 1, FIN_SIGMA = 2, FIN_CHECK = 3, FIN_MASS = 4, FIN_RHS = 5, FIN_BLOCK = 6 };
void finalize(cudaStream_t st, FinKind kind, DevState* ds, const double* part,
              long long nblocks, const double* part2, long long nblocks2,
              const double* part3, long long nblocks3);

}  // namespace lbm
