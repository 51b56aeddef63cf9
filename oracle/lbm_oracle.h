/*
 * lbm_oracle.h -- FP64 CPU restatement of the Inamuro two-phase D3Q15 step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA library is compared
 * against; nothing in the product (lbm_b200/) links, loads or calls it.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * It restates, step for step and with the same floating-point operation order,
 * the reference solver in UniBoy222/LBM:
 *   CPU/common.hpp:3-45            D3Q15 tables
 *   CPU/Inamuro.hpp:213-314        firstord / secondord stencils
 *   CPU/Inamuro.cpp:134-250        collision (f, g equilibria + BGK + viscous term)
 *   CPU/Inamuro.cpp:252-287        periodic streaming
 *   CPU/Inamuro.cpp:589-623        x slip bounce-back
 *   CPU/Inamuro.cpp:294-346        moments (phi, rho(phi), u*)
 *   CPU/Inamuro.cpp:624-793        pressure Poisson solve (collision_p, getp, gauge, getError)
 *   CPU/Inamuro.cpp:794-840        velocity correction, h reset
 *   CPU/Inamuro.cpp:843-847        EOS
 *   GPU/InamuroCUDA.cu:1987-2057   kinetic fixed-point (dual) residual
 *   DUAL_RESIDUAL_CONTRACT.md      dual-residual definition
 *
 * Pinned: with dual=0, check_interval=100, tol=1e-3 it reproduces the compiled
 * reference CPU solver bit for bit (tests/golden, generated by oracle/_ref).
 *
 * Layout: every field is a flat array of N = lx*ly*lz doubles with x fastest,
 * cell = (z*ly + y)*lx + x (no z ghost layers).  Populations are q-major:
 * f[q*N + cell].
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int lx, ly, lz;
    double rho_L, rho_G;
    double mu_L, mu_G;
    double tauf, taug;
    double k_f, k_g;
    double T, a, b;
    double fei_L, fei_G;
    /* Poisson stopping rule */
    int check_interval;      /* reference: 100 */
    double tol;              /* reference: 1e-3 */
    int dual;                /* 1: also require the kinetic fixed-point residual < tol */
    uint64_t max_sweeps;     /* 0 = unbounded (reference contract); else error when hit */
    int periodic_x;          /* 1: periodic x (no slip walls) -- not a reference mode */
    int poisson_form;        /* 0: kinetic (production); 1: the reference's scalar Jacobi form;
                                2: the reference's one-pass form */
    double scalar_source_scale;  /* scalar form: --scalar-source-scale (reference default 2.0) */
    /* the reference's accelerators (GPU/main.cpp flags); a zero-initialised
       block means: relaxations 1 (0 is read as 1), all off */
    double pressure_relax_scale;     /* one-pass: --pressure-relax-scale */
    double fixed_point_relax;        /* one-pass: --poisson-fixed-point-relax */
    int anderson_m1;                 /* one-pass: --poisson-anderson-m1 */
    double anderson_beta_max;        /* --poisson-anderson-beta-max */
    int two_grid;                    /* one-pass: --poisson-two-grid-correction */
    double two_grid_strength;        /* --poisson-two-grid-strength */
    int source_aware_init;           /* kinetic and one-pass: --source-aware-hh-init */
    double source_aware_scale;       /* --source-aware-hh-scale */
} orc_params;

typedef struct {
    uint64_t sweeps;             /* Poisson sweeps taken this step */
    double relative_error;       /* last relative-change value */
    double pressure_l1_delta;
    double pressure_l1_norm;
    double fp_h_l1, fp_h_scale, fp_h_rel;
    double fp_p_l1, fp_p_scale, fp_p_rel;
    double fp_rel;
    double divergence_mean;      /* mean of u_x+v_y+w_z before projection */
    double gauge_target;
    double gauge_max_shift;
    double mass;                 /* sum of phi after the step (x-outer order) */
} orc_step_info;

enum {
    ORC_OK = 0,
    ORC_ERR_NONFINITE = 2,
    ORC_ERR_BUDGET = 3,
    ORC_ERR_ARG = 4,
    ORC_ERR_OOM = 5
};

typedef struct orc_state orc_state;

/* Fields are N doubles each, x fastest.  p may be NULL (zeros). */
orc_state* orc_create(const orc_params* prm,
                      const double* phi, const double* rho,
                      const double* u, const double* v, const double* w,
                      const double* p);
void orc_destroy(orc_state* s);

/* One full time step.  replay_sweeps > 0 forces exactly that many sweeps
 * (checks, gauges and p_prev updates still run every check_interval; the exit
 * test is ignored).  Returns ORC_OK or an error code. */
int orc_step(orc_state* s, uint64_t replay_sweeps, orc_step_info* info);

/* Copies out phi, rho, u, v, w, p (any pointer may be NULL). */
void orc_get_fields(const orc_state* s, double* phi, double* rho,
                    double* u, double* v, double* w, double* p);
/* Copies out f, g, h (15*N each, q-major; any may be NULL). */
void orc_get_populations(const orc_state* s, double* f, double* g, double* h);
/* Copies out the 19 derivative fields of the last collision, in the order
 * fei_x fei_y fei_z rho_x rho_y rho_z u_x u_y u_z v_x v_y v_z w_x w_y w_z
 * fei_lap u_lap v_lap w_lap (u_x after the Poisson mean projection). */
void orc_get_derivatives(const orc_state* s, double* out19);

/* Initial condition of GPU/Inamuro.cpp:491-566 on an N-cell box.  Writes phi,
 * rho, w (u, v untouched).  Fields must be pre-filled with the background
 * (phi = fei_min, rho = rho_G, w = 0). */
void orc_init_droplets(int lx, int ly, int lz, double DD,
                       double fei_max, double fei_min,
                       double rho_L, double rho_G,
                       int single_droplet, int tanh_profile,
                       double init_velocity, double interface_width,
                       double cx_in, double cy_in, double cz_in,
                       double separation, double offset_x,
                       double* phi, double* rho, double* w);

#ifdef __cplusplus
}
#endif
#endif
