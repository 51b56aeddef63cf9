/*
 * lbm_b200.h -- C ABI of the B200 (sm_100a) Inamuro two-phase D3Q15 droplet
 * time step.
 *
 * The reference (UniBoy222/LBM) exposes this path only as the C++ class
 * InamuroCUDA (GPU/InamuroCUDA.hpp:16-248) built on a CPU-side Inamuro object
 * (GPU/Inamuro.hpp:11-140).  This header is the flat boundary under the C++
 * drop-in class of include/InamuroCUDA.hpp: plain pointers and sizes,
 * integer status codes, no exceptions and no C++ or torch types.  Each entry
 * point names the reference interface it replaces.
 *
 * Field layout (host and device): a field is lx*ly*lz doubles, x fastest,
 * cell = (z*ly + y)*lx + x.  The "ghosted" variants use the reference's device
 * layout with one z ghost plane on each side: lx*ly*(lz+2) doubles,
 * ((z+1)*ly + y)*lx + x (GPU/InamuroCUDA.cu:1438, 1675-1696).
 *
 * A handle owns its device buffers and one CUDA stream; it is used by one host
 * thread at a time.  Every call is synchronous with respect to the host unless
 * stated otherwise.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Bumped whenever a struct layout or a signature of this header changes;
   callers compare it with lbm_abi_version() of the loaded library. */
#define LBM_B200_ABI_VERSION 6

typedef enum {
    LBM_OK = 0,
    LBM_ERR_CUDA = 1,            /* CUDA runtime error (reference: CUDA_CHECK -> runtime_error, .cu:12-18) */
    LBM_ERR_NONFINITE = 2,       /* NaN/Inf in source, gauge or residual (reference .cu:1888-2125 throws) */
    LBM_ERR_POISSON_BUDGET = 3,  /* sweep cap reached without convergence */
    LBM_ERR_BAD_ARG = 4,         /* invalid argument (reference: std::invalid_argument) */
    LBM_ERR_OOM = 5,             /* device allocation failed */
    LBM_ERR_IO = 6,              /* params file missing or unreadable */
    LBM_ERR_NO_DEVICE = 7,       /* no CUDA device or not sm_100 */
    LBM_ERR_OVERFLOW = 8         /* counter overflow (reference .cu:21-45) */
} lbm_status;

typedef enum {
    LBM_PRECISION_FP64 = 0,      /* plain FP64, reference operation order: the drop-in */
    LBM_PRECISION_MIXED = 1      /* FP32 populations as deviations + FP64 reductions.  Its
                                    plain Poisson sweeps stall at a relative change near 1e-7:
                                    for tighter tolerances select LBM_POISSON_REFINE, or the
                                    loop runs to max_sweeps (forever with no cap, as the
                                    reference's loop would) */
} lbm_precision;

typedef enum {
    LBM_FIELD_PHI = 0, LBM_FIELD_RHO = 1, LBM_FIELD_U = 2,
    LBM_FIELD_V = 3, LBM_FIELD_W = 4, LBM_FIELD_P = 5
} lbm_field;

/* params.in contents (CPU/Inamuro.cpp:38-53 positional lines, GPU/Inamuro.cpp:56-103
 * key=value init tokens; struct of GPU/Inamuro.hpp:36-76). */
typedef struct {
    int lx, ly, lz;              /* line 1 */
    int period;                  /* line 2 (read, unused by the step) */
    int t_max;                   /* line 3 */
    int nwri;                    /* line 4 */
    double rho_L, rho_G;         /* line 5 */
    double tauf, taug;           /* line 6 */
    double mu_L, mu_G;           /* line 7 */
    double k_f, k_g;             /* line 8 */
    double T;                    /* line 9 */
    double a;                    /* line 10 */
    double b;                    /* line 11 */
    double fei_max, fei_min;     /* line 12 */
    double fei_L, fei_G;         /* line 13 */
    double DD;                   /* line 14 */
    /* GPU-tree initial-condition tokens (defaults of GPU/Inamuro.hpp:56-64) */
    int init_single_droplet;     /* init_mode=single_droplet (else two_droplets) */
    int init_tanh;               /* init_profile=tanh (else sharp) */
    double init_velocity;
    double interface_width;
    double init_center_x, init_center_y, init_center_z;
    double init_separation;
    double init_offset_x;
    /* Not a reference mode: 1 makes x periodic instead of the reference's slip
     * walls (params.in token boundary_x=periodic); default 0 (slip walls). */
    int periodic_x;
} lbm_params;

/* Poisson stopping rule (InamuroCUDA::setPoissonConvergence /
 * setPoissonIterationLimit / setUsePoissonDualResidual, GPU/InamuroCUDA.hpp:83-86). */
typedef struct {
    int check_interval;          /* sweeps between checks; reference contract 100 */
    double tolerance;            /* relative-change (and dual) tolerance; contract 1e-3 */
    int dual_residual;           /* 0: relative change only; 1: also require the kinetic
                                    fixed-point residual < tol (--poisson-dual-residual);
                                    2: evaluate and report it without changing the exit
                                    (--poisson-fixed-point-shadow) */
    uint64_t max_sweeps;         /* 0 = unbounded (contract); else the iteration limit */
    int fail_on_limit;           /* 0: at the limit stop and finish the step unconverged, as
                                    the reference's poisson_iteration_limit does (.cu:2336-2339);
                                    1: return LBM_ERR_POISSON_BUDGET instead */
} lbm_poisson_cfg;

/* Per-step diagnostics (InamuroCUDA::PoissonStepDiagnostics, GPU/InamuroCUDA.hpp:19-43,
 * plus the step's mass and device time). */
typedef struct {
    uint64_t iterations;
    double relative_error;
    double pressure_l1_delta;
    double pressure_l1_norm;
    double fixed_point_h_l1;
    double fixed_point_h_scale;
    double fixed_point_h_relative;
    double fixed_point_p_l1;
    double fixed_point_p_scale;
    double fixed_point_p_relative;
    double fixed_point_relative;
    double source_mean;              /* -mean(div)/3, as the reference reports it */
    double source_abs_mean;
    double projected_source_mean;
    double pressure_gauge_target;
    double pressure_gauge_max_shift;
    double mass;                     /* sum of phi over the box after the step */
    int fixed_point_evaluated;
    int pressure_converged;
    int fixed_point_converged;
    int dual_residual_enabled;
    int converged;
    int reserved;
    double device_ms;                /* device time of the step (CUDA events) */
} lbm_step_stats;

/* Accumulated device time per kernel class since the last reset (CUDA events
 * on the handle's stream; replaces printPerformanceMetrics' per-phase timers,
 * GPU/InamuroCUDA.cu:2377-2437). */
typedef struct {
    double collide_ms;       /* fused stencils + collide + stream of f, g */
    double moments_ms;       /* pull + bounce + phi, rho, u* */
    double prep_ms;          /* source projection + gauge target */
    double poisson_ms;       /* all Poisson segments (sweeps + checks) */
    double correct_ms;       /* velocity correction */
    uint64_t steps;
    uint64_t sweeps;         /* Poisson sweeps summed over steps */
    uint64_t sweep_kernels;  /* sweep-kernel launches (incl. the extra one per check) */
    uint64_t kernel_launches;/* all kernels launched by the library (graph nodes included) */
    uint64_t fused_sweeps;   /* sweeps run inside two-sweep (temporally blocked) launches */
} lbm_timing;

/* Statistics of one field over the box (Inamuro::FieldStatistics,
 * CPU/Inamuro.hpp:91-99, filled as collectDiagnostics does,
 * CPU/Inamuro.cpp:412-507, 1050-1092): NaN and +-Inf values are counted and
 * left out; min, max, mean and abs_max are over the finite values (NaN when
 * there are none).  sum is the sum of the finite values (the mass for phi). */
typedef struct {
    double min, max, mean, abs_max;
    uint64_t nan_count, inf_count;
    double sum;
    uint64_t valid_count;
} lbm_field_stats;

/* All step statistics at once (Inamuro::collectDiagnostics,
 * CPU/Inamuro.cpp:412-507, the DiagnosticsSnapshot of CPU/Inamuro.hpp), in
 * its field order: rho, phi (fei), u, v, w, velocity magnitude
 * sqrt(u*u + v*v + w*w), p. */
typedef struct {
    lbm_field_stats rho, fei, u, v, w, velocity_magnitude, p;
} lbm_diagnostics;

/* One Poisson convergence check (the row InamuroCUDA::writePoissonDiagnostic
 * appends to the diagnostics CSV, GPU/InamuroCUDA.cu:2634-2682). */
typedef struct {
    uint64_t step;                   /* 1-based time step of the handle */
    uint64_t iteration;              /* sweep count at the check */
    double pressure_l1_delta;
    double pressure_l1_norm;
    double relative_error;
    double fixed_point_h_l1, fixed_point_h_scale, fixed_point_h_relative;
    double fixed_point_p_l1, fixed_point_p_scale, fixed_point_p_relative;
    double fixed_point_relative;     /* NaN when not evaluated */
    int fixed_point_evaluated;
    int pressure_converged;
    int fixed_point_converged;
    int dual_residual_enabled;
    int converged;
    int reserved;
    double block_low_frequency_fraction;   /* spatial diagnostics: sum_b |sum_{cells of b} (p - p_prev)|
                                              / sum |p - p_prev| over 4^3 blocks b; NaN when off */
    int spatial_block_size;                /* 4 when block sums are taken (spatial diagnostics or
                                              two-grid correction), else 0 */
    int spatial_block_count;
} lbm_check_record;

typedef void (*lbm_check_callback)(void* user, const lbm_check_record* record);

typedef struct lbm_handle lbm_handle;

/* ---- params and initial condition (host only, no GPU needed) ---- */

/* Reference defaults (GPU/Inamuro.hpp:36-76, box 48x96x128). */
void lbm_params_default(lbm_params* out);

/* Parses params.in: 14 positional lines (CPU/Inamuro.cpp:38-53), then both the
 * whitespace-token init keys (GPU/Inamuro.cpp:56-103) and the line-wise
 * key=value output keys (ignored here; CPU/InamuroSolver.cpp:143-218).
 * Replaces Inamuro::Parameters::Parameters(const std::string&). */
lbm_status lbm_params_load(const char* path, lbm_params* out);

/* Droplet initial condition of Inamuro::initializeDroplets (GPU/Inamuro.cpp:491-566)
 * written into physical-layout host fields (each lx*ly*lz doubles): phi, rho,
 * u, v, w, p.  Replaces Inamuro::initializeArrays + initializeDroplets. */
lbm_status lbm_init_droplets(const lbm_params* prm, double* phi, double* rho,
                             double* u, double* v, double* w, double* p);

/* ---- solver handle ---- */

/* Allocates the device state for one box on `device` (replaces the
 * InamuroCUDA(const Inamuro&) constructor's allocateDeviceMemory,
 * GPU/InamuroCUDA.cu:1429-1461, 1536-1607).  Fields start at the background
 * state; load them with lbm_load_fields*.  Poisson config starts at the
 * reference contract {100, 1e-3, dual=0, unbounded}. */
lbm_status lbm_create(const lbm_params* prm, lbm_precision precision, int device,
                      lbm_handle** out);
void lbm_destroy(lbm_handle* h);

/* Host -> device upload of the macro fields; resets the step counter so the
 * next step is a "first step" (f, g set to equilibrium).  p may be NULL (zero).
 * Replaces InamuroCUDA::initFromCPU (GPU/InamuroCUDA.cu:1628-1673). */
lbm_status lbm_load_fields(lbm_handle* h, const double* phi, const double* rho,
                           const double* u, const double* v, const double* w,
                           const double* p);
/* Same with ghosted (lx*ly*(lz+2)) arrays; the ghost planes are kept and given
 * back unchanged by lbm_download_ghosted, as the reference does. */
lbm_status lbm_load_fields_ghosted(lbm_handle* h, const double* phi, const double* rho,
                                   const double* u, const double* v, const double* w,
                                   const double* p);
/* Device -> device upload (pointers to device memory on the handle's device). */
lbm_status lbm_load_fields_device(lbm_handle* h, const double* phi, const double* rho,
                                  const double* u, const double* v, const double* w,
                                  const double* p);

/* InamuroCUDA::setPoissonConvergence / setPoissonIterationLimit /
 * setUsePoissonDualResidual (GPU/InamuroCUDA.cu:2573-2608). */
lbm_status lbm_set_poisson(lbm_handle* h, const lbm_poisson_cfg* cfg);
lbm_status lbm_get_poisson(const lbm_handle* h, lbm_poisson_cfg* cfg);

/* Poisson form.  LBM_POISSON_KINETIC is the reference's production solve (its
 * split form; its fused form and fused boundary do the same arithmetic, so
 * they are this form too).  The scalar forms are the reference's
 * non-production scalar option (InamuroCUDA::setUseScalarPoisson,
 * GPU/InamuroCUDA.cu:864-901, 2207-2218): the 14-neighbour stencil
 * lap p = (sum_nb p - 14 p)/5 solved for lap p = source_scale rho s, with the
 * same gauge and relative-change exit; its result differs from the kinetic
 * form's (another equation).  LBM_POISSON_SCALAR_JACOBI sweeps as the
 * kernel of the reference's option states (its own loop overwrites p from
 * the unchanged h after every sweep, GPU/InamuroCUDA.cu:2307-2329, so its
 * option leaves p at its start value); LBM_POISSON_SCALAR_RB solves the same
 * equation by red-black SOR with the right-hand side's constant and
 * checkerboard components removed (the components the Jacobi sweeps never
 * take up at their even check counts; projected with weight 1/2 on the
 * slip-wall planes), reaching the Jacobi sweeps' gauged limit in far fewer
 * sweeps.
 * Scalar forms: FP64 only, no dual residual; red-black needs even ly, lz
 * (and lx with periodic_x).  source_scale: the reference's
 * --scalar-source-scale (default 2.0); omega: SOR relaxation in (0, 2), 0 =
 * the optimum for the box's slowest mode. */
typedef enum {
    LBM_POISSON_KINETIC = 0,
    LBM_POISSON_SCALAR_JACOBI = 1,
    LBM_POISSON_SCALAR_RB = 2,
    LBM_POISSON_ONEPASS = 3,     /* the reference's one-pass form (setUseOnePassPoisson,
                                    GPU/InamuroCUDA.cu:780-844): the kinetic map on the
                                    pre-collision h with the accelerators of lbm_poisson_accel */
    LBM_POISSON_KRYLOV = 4,      /* not a reference form: the kinetic form's fixed point solved by
                                    BiCGSTAB, stopping at ||b - (I - K) h|| < tolerance ||b|| (the
                                    lbm_poisson_cfg tolerance; max_sweeps caps the applications of
                                    the kinetic map).  Same fixed point as the kinetic form (with
                                    the slip walls, the gauged one: the walls' overwrite makes
                                    the system inconsistent, and the solve runs on the bordered
                                    system with the sweeps' drift and the gauge); FP64,
                                    no dual residual, no two-grid or
                                    spatial diagnostics, no lbm_step_replay (it has no sweep count
                                    to replay).  A NaN/Inf source or start iterate returns
                                    LBM_ERR_NONFINITE; twenty restarts in a row that do not lower
                                    the true residual (a tolerance below the rounding floor)
                                    stop the solve with LBM_ERR_POISSON_BUDGET */
    LBM_POISSON_VARCOEF_RB = 5,  /* not a reference form: div((1/rho) grad p) = s, the continuum
                                    limit of the kinetic form (diffusivity 1/(3 rho), source
                                    -s/3), on the D3Q15 neighbours with arithmetic face means
                                    of 1/rho (x mirrored at the slip walls), solved by red-black
                                    SOR (omega as for LBM_POISSON_SCALAR_RB).  Each check gauges
                                    p, takes the relative change and the operator residual
                                    ||A p - s|| / max(||s||, ||A p||) (reported in the
                                    fixed-point fields of lbm_step_stats); the exit needs both
                                    below the tolerance.  Another discretisation than the
                                    kinetic form's: its p differs at the interface.  FP64, even
                                    ly, lz (and lx with periodic_x), no lbm_poisson_cfg dual
                                    residual, no accelerators */
    LBM_POISSON_REFINE = 6       /* not a reference form: the kinetic form on the mixed box by
                                    iterative refinement.  The post-collision h is kept in FP64
                                    (a further 300 B/cell); each check interval runs as one FP64
                                    residual r = K h + b - h, check_interval - 2 FP32 correction
                                    sweeps e <- K e + r and the FP64 check (gauge, relative
                                    change) on h + e: in exact arithmetic the kinetic form's
                                    sweeps and exit, but the FP32 rounding falls on the
                                    correction only, so tight tolerances converge to the FP64
                                    fixed point (the plain mixed sweeps stall near 1e-7).
                                    Mixed precision only; no dual residual, no accelerators */
} lbm_poisson_form;
lbm_status lbm_set_poisson_form(lbm_handle* h, lbm_poisson_form form, double source_scale, double omega);
/* Current form, source scale and the relaxation in use (the computed optimum
 * when 0 was set); any pointer may be NULL. */
lbm_status lbm_get_poisson_form(const lbm_handle* h, lbm_poisson_form* form, double* source_scale, double* omega);

/* The reference's Poisson accelerators (InamuroCUDA setters,
 * GPU/InamuroCUDA.hpp:67-88; CLI flags of GPU/main.cpp:156-171), FP64.
 * pressure_relax_scale, fixed_point_relax and Anderson-m1 need the one-pass
 * form (LBM_ERR_BAD_ARG at the next step otherwise); two-grid correction,
 * source-aware h init and spatial diagnostics apply to the kinetic and
 * one-pass forms.  None combines with the dual residual (the reference
 * refuses that too).  Defaults: 1, 1, off, 1, off, 0.5, off, 1, off, 0. */
typedef struct {
    double pressure_relax_scale;   /* --pressure-relax-scale: scales (h - E p) / tau_h */
    double fixed_point_relax;      /* --poisson-fixed-point-relax: h = h_old + omega (T(h) - h_old) */
    int anderson_m1;               /* --poisson-anderson-m1 */
    double anderson_beta_max;      /* --poisson-anderson-beta-max: alpha clamped to [-b, 1 + b] */
    int two_grid;                  /* --poisson-two-grid-correction */
    double two_grid_strength;      /* --poisson-two-grid-strength */
    int source_aware_init;         /* --source-aware-hh-init */
    double source_aware_scale;     /* --source-aware-hh-scale */
    int spatial_diagnostics;       /* --poisson-spatial-diagnostics: block_low_frequency_fraction of
                                      every check record */
    int krylov_degree;             /* not a reference setting: LBM_POISSON_KRYLOV's polynomial
                                      preconditioner, BiCGSTAB on (I - K^m) h =
                                      (I + K + ... + K^(m-1)) b with m = krylov_degree (0 or 1: the
                                      plain system; at most 16).  Same solution, fewer iterations
                                      for m applications of K each; the tolerance then applies to
                                      the preconditioned residual */
} lbm_poisson_accel;
lbm_status lbm_set_poisson_accel(lbm_handle* h, const lbm_poisson_accel* a);
lbm_status lbm_get_poisson_accel(const lbm_handle* h, lbm_poisson_accel* out);

/* Advances n_steps time steps (InamuroCUDA::performTimeStepGPU,
 * GPU/InamuroCUDA.cu:2372-2442).  `stats` (may be NULL) receives n_steps
 * entries.  On error the state is left as of the failing step. */
lbm_status lbm_step(lbm_handle* h, int n_steps, lbm_step_stats* stats);

/* Like lbm_step, but every step runs exactly sweeps[i] Poisson sweeps (a
 * multiple of the check interval); checks, gauges and p_prev updates still run
 * at every check.  Used to compare two precisions on identical sweep counts. */
lbm_status lbm_step_replay(lbm_handle* h, int n_steps, const uint64_t* sweeps,
                           lbm_step_stats* stats);

/* Calls cb(user, record) on the host after every Poisson convergence check
 * (NULL cb disables).  Replaces InamuroCUDA::setPoissonDiagnosticsPath's
 * per-check CSV rows (GPU/InamuroCUDA.cu:2610-2682): the caller formats them.
 * While a callback is set the Poisson loop returns to the host after every
 * check; without one the checks run back to back on the device (a CUDA graph
 * with a conditional WHILE node, at most 64 checks per launch), with the same
 * results and sweep counts. */
lbm_status lbm_set_check_callback(lbm_handle* h, lbm_check_callback cb, void* user);

/* Device -> host download of one field (physical layout). */
lbm_status lbm_download(lbm_handle* h, lbm_field which, double* host);
/* Ghosted layout, ghost planes as loaded (InamuroCUDA::downloadFieldsToCPU,
 * GPU/InamuroCUDA.cu:1675-1701). */
lbm_status lbm_download_ghosted(lbm_handle* h, lbm_field which, double* host_ghosted);
/* h populations in the reference's AoS layout cell*15+q, 15*lx*ly*lz doubles
 * (InamuroCUDA::downloadHH, GPU/InamuroCUDA.cu:1703-1707).  Between steps
 * h = E_q p, as after update_hh. */
lbm_status lbm_download_h(lbm_handle* h, double* host);
/* Device pointer of a field (physical layout, FP64 handles only, valid until
 * the next call on the handle).  For device-resident consumers. */
lbm_status lbm_field_device_ptr(lbm_handle* h, lbm_field which, const double** dev);

/* Device reduction of one field's statistics (Inamuro::collectDiagnostics /
 * updateFieldStatistics / finalizeFieldStatistics, CPU/Inamuro.cpp:412-507,
 * 1050-1092; the reference computes them on the host after a download).
 * Fixed-order reduction: repeated calls give identical results. */
lbm_status lbm_field_statistics(lbm_handle* h, lbm_field which, lbm_field_stats* out);

/* Largest field lbm_field_statistics_noalloc accepts: 8192 partial blocks of
 * 4096 cells each, the capacity of its static device scratch (8192 x 7 doubles,
 * 458,752 bytes, plus one result record; every GPU that loads the library keeps
 * that much reserved until the process exits). */
#define LBM_NOALLOC_MAX_CELLS 33554432ULL

/* Inamuro::collectDiagnostics on the device: the statistics of every field
 * and of the velocity magnitude in one call (fixed-order reductions; the
 * mean of a field may differ from the reference's serial sum in the last
 * bits).  The step_diagnostics.csv columns of CPU/InamuroSolver.cpp:276-334. */
lbm_status lbm_diagnostics_snapshot(lbm_handle* h, lbm_diagnostics* out);

/* Same statistics as lbm_field_statistics for a caller-owned device field of
 * n_cells doubles, without allocating anything.  It has no counterpart in the
 * reference.  It is for callers that must not allocate device memory: a host
 * application that hands the GPU's memory to its own pool at start-up (an
 * extra cudaMalloc would fail or fragment that pool), a time-critical loop
 * that cannot afford cudaMalloc/cudaFree (they may synchronize the whole
 * device), or a plugin that is given device pointers but no allocator.
 *   - field: device pointer on the calling thread's current device;
 *     stream: a cudaStream_t (NULL = the legacy default stream); the call
 *     returns after the result has been copied into *out.
 *   - The scratch is a static array inside the library, shared by every call
 *     on a device and keeping the last call's contents; nothing in it needs to
 *     start at zero (each block writes its own slot before the final pass reads
 *     it).  Calls whose GPU work overlaps (other threads or streams) race on
 *     it: serialise them.
 *   - Every call looks up the array's device address with the calling
 *     thread's current device (the lookup allocates nothing), so a device
 *     reset between calls is followed.  The first call on a device may also
 *     load the library's device code there (CUDA's lazy module loading);
 *     make that first call before any stream capture.
 *   - Returns LBM_ERR_BAD_ARG for a null pointer, n_cells == 0 or
 *     n_cells > LBM_NOALLOC_MAX_CELLS, LBM_ERR_CUDA on a CUDA failure. */
lbm_status lbm_field_statistics_noalloc(const double* field, uint64_t n_cells, void* stream,
                                        lbm_field_stats* out);

/* InamuroCUDA::synchronize (GPU/InamuroCUDA.cu:1709-1712). */
lbm_status lbm_synchronize(lbm_handle* h);

lbm_status lbm_get_timing(const lbm_handle* h, lbm_timing* out);
lbm_status lbm_reset_timing(lbm_handle* h);
/* Enables per-kernel-class CUDA-event timing (default on). */
lbm_status lbm_set_timing(lbm_handle* h, int enabled);

/* Text of the last error on this handle ("" if none); valid until the next call.
 * With h == NULL: why the calling thread's last lbm_create failed. */
const char* lbm_last_error(const lbm_handle* h);
const char* lbm_status_string(lbm_status s);
int lbm_abi_version(void);

/* Self-check of the FP64 kernels' division (a correctly rounded a/b from a
 * reciprocal computed once per divisor, exact_div.cuh) against the IEEE
 * division on the current device: `samples` pseudo-random operand pairs of
 * the kinds the kernels divide (stencil constants, relaxation times,
 * densities, arbitrary normals); *mismatches = pairs whose bits differ. */
lbm_status lbm_selftest_division(uint64_t samples, uint64_t seed, uint64_t* mismatches);

/* ---- batched boxes ------------------------------------------------------
 * Many independent droplet boxes of different sizes and physics advanced
 * together on one GPU, mixed precision (FP32 populations, FP64 pressure sums,
 * reductions and exit tests, as LBM_PRECISION_MIXED).  The reference has no
 * batched form; each instance follows the single-box step exactly (same
 * kernels' cell arithmetic, same Poisson exit per instance), and every phase
 * of a step is one launch over all instances: a persistent grid walks a work
 * list of (instance, xy tile, z run) items.  Each instance leaves the Poisson
 * loop at its own check; its items are skipped for the rest of the step.
 * x boundary per instance as in the single box (slip walls, or periodic with
 * lbm_params.periodic_x); the dual residual is not available
 * (dual_residual must be 0). */
typedef struct lbm_batch lbm_batch;

/* Launch shape of the batched kernels (what lbm_batch_tune chooses). */
typedef struct {
    int tile_x, tile_y;      /* cells per CTA tile in x and y (tile_x * tile_y = 256) */
    int zrun;                /* z planes per work item */
    int ctas_per_sm;         /* persistent grid: ctas_per_sm CTAs per SM */
    int sweep2_zrun;         /* > 0: plain sweeps run two per launch (temporal blocking,
                                16 x 8 tiles) on z runs of this length; 0: one per launch */
    int reserved;
    double sweep_ms;         /* measured time per sweep of the chosen form (lbm_batch_tune), else 0 */
} lbm_batch_tuning;

/* One box per params[i] (its own lx, ly, lz and physics). */
lbm_status lbm_batch_create(const lbm_params* params, int n_instances, int device, lbm_batch** out);
void lbm_batch_destroy(lbm_batch* b);
int lbm_batch_size(const lbm_batch* b);
/* Initial macro fields of instance inst, physical layout (lbm_load_fields);
 * NULL fields load as zero (p, u, v, w) or the gas state (phi, rho).  The
 * next step restarts EVERY instance from its current macro fields
 * (equilibrium populations, first Poisson solve from h = 0), as constructing
 * the reference's class from a CPU object does: load all instances, then step. */
lbm_status lbm_batch_load_fields(lbm_batch* b, int inst, const double* phi, const double* rho, const double* u,
                                 const double* v, const double* w, const double* p);
/* Poisson settings for every instance (lbm_set_poisson; dual_residual must be 0). */
lbm_status lbm_batch_set_poisson(lbm_batch* b, const lbm_poisson_cfg* cfg);
/* n_steps steps of every instance; stats (may be NULL): n_steps * n_instances
 * entries, step-major (stats[s * n_instances + i]). */
lbm_status lbm_batch_step(lbm_batch* b, int n_steps, lbm_step_stats* stats);
/* The same with a fixed sweep count per step and instance (multiples of the
 * check interval), sweeps[s * n_instances + i]. */
lbm_status lbm_batch_step_replay(lbm_batch* b, int n_steps, const uint64_t* sweeps, lbm_step_stats* stats);
/* A field of instance inst in the physical layout (lbm_download). */
lbm_status lbm_batch_download(lbm_batch* b, int inst, lbm_field which, double* host);
/* Autotuner: times the batched sweep over the candidate tiles (32x8, 16x16,
 * 8x32), z runs (1, 2, 4, 8) and persistent grids (2, 4, 8 CTAs per SM), then
 * the two-sweep pass on z runs of 8, 16 and 32, on the loaded state, and keeps
 * the fastest per sweep (the Poisson state is rebuilt at the next step, so
 * tuning changes no result).  chosen may be NULL. */
lbm_status lbm_batch_tune(lbm_batch* b, lbm_batch_tuning* chosen);
lbm_status lbm_batch_set_tuning(lbm_batch* b, const lbm_batch_tuning* t);
lbm_status lbm_batch_get_tuning(const lbm_batch* b, lbm_batch_tuning* out);
/* Device time per kernel class summed over instances' launches (lbm_timing;
 * sweeps = sweeps summed over steps and instances, sweep_kernels = batched
 * sweep launches). */
lbm_status lbm_batch_get_timing(const lbm_batch* b, lbm_timing* out);
lbm_status lbm_batch_reset_timing(lbm_batch* b);
/* Text of the last error on this batch ("" if none); with b == NULL: why the
 * calling thread's last lbm_batch_create failed. */
const char* lbm_batch_last_error(const lbm_batch* b);

/* ---- adjoints of the explicit FP64 kernels --------------------------------
 * Forward/backward pairs over caller-owned DEVICE buffers of one box
 * (cell = (z*ly + y)*lx + x, populations q-major: a[q*n + cell]); each call
 * synchronises the device.  The reference computes no derivatives: these give
 * the building blocks of a gradient through its step.  A forward call is the
 * FP64 kernel of the solver (bitwise the same values); the matching backward
 * call takes the adjoint (dJ/d output) of every output and returns the adjoint
 * of every input at the same state, i.e. the transposed Jacobian applied to
 * it.  Both x boundaries are differentiated: with the reference's slip walls
 * (lbm_params.periodic_x = 0) the backward calls transpose the walls'
 * overwrite of the pulled populations and the mirrored x neighbours of the
 * stencils and of the correction.
 *
 * Collide (CPU/Inamuro.cpp:134-250): pull of the previous post-collision
 * populations fin/gin, then the f and g collisions with the stencils of phi,
 * rho, u, v, w; outputs fout, gout and the velocity derivatives u_x, v_y,
 * w_z (the Poisson source).  The map is affine in fin and gin, so the backward
 * call does not read them (they may be NULL there). */
lbm_status lbm_collide_forward(const lbm_params* p, const double* fin, const double* gin, const double* phi,
                               const double* rho, const double* u, const double* v, const double* w, double* fout,
                               double* gout, double* dux, double* dvy, double* dwz);
lbm_status lbm_collide_backward(const lbm_params* p, const double* fin, const double* gin, const double* phi,
                                const double* rho, const double* u, const double* v, const double* w,
                                const double* lam_fout, const double* lam_gout, const double* lam_dux,
                                const double* lam_dvy, const double* lam_dwz, double* lam_fin, double* lam_gin,
                                double* lam_phi, double* lam_rho, double* lam_u, double* lam_v, double* lam_w);
/* Moments (CPU/Inamuro.cpp:294-346): pull of f*, g*, then phi, rho(phi)
 * (sine interpolation between fei_G and fei_L), u*, v*, w*. */
lbm_status lbm_moments_forward(const lbm_params* p, const double* f, const double* g, double* phi, double* rho,
                               double* u, double* v, double* w);
lbm_status lbm_moments_backward(const lbm_params* p, const double* phi, const double* lam_phi,
                                const double* lam_rho, const double* lam_u, const double* lam_v, const double* lam_w,
                                double* lam_f, double* lam_g);
/* Velocity correction (CPU/Inamuro.cpp:794-823), in place:
 * u -= (p(x+1) - p(x-1)) / (2 rho), likewise v, w.  The adjoints of u*, v*,
 * w* equal those of u, v, w; backward returns those of p and rho. */
lbm_status lbm_correct_forward(const lbm_params* p, double* u, double* v, double* w, const double* press,
                               const double* rho);
lbm_status lbm_correct_backward(const lbm_params* p, const double* press, const double* rho, const double* lam_u,
                                const double* lam_v, const double* lam_w, double* lam_p, double* lam_rho);

/* ---- adjoint runs: gradients through whole FP64 time steps ------------------
 * A forward run of n steps of one FP64 box (slip walls or periodic x, as
 * lbm_params.periodic_x says) from loaded macro fields, then its reverse
 * pass: given the adjoint of the final fields (dJ/d phi_T, ... for an
 * objective J of them), the gradient of J
 * with respect to the loaded fields and to k_f (kappa_f).  The Poisson solve
 * is differentiated implicitly: each step's reverse pass solves one adjoint
 * problem of the solve's fixed point (the transposed kinetic sweep, iterated
 * to the tolerance of lbm_adjoint_cfg) instead of unrolling its sweeps, so
 * the gradient is that of the converged solve.  The forward run keeps the
 * state every checkpoint_interval steps; the reverse pass recomputes each
 * interval from its checkpoint (replaying the forward's sweep counts, so the
 * recomputed states are bitwise the forward's) and walks it backwards.
 * Device memory: about 288 B/cell per checkpoint (156 with the mixed forward box) plus 168 B/cell per step of
 * one interval (uniform) or of one step (binomial) plus about 1 kB/cell of
 * adjoint buffers.  The reference has no derivatives. */
typedef struct lbm_adjoint lbm_adjoint;

typedef struct {
    int checkpoint_interval;   /* steps between stored states (>= 1) */
    int check_interval;        /* adjoint Poisson: sweeps between convergence checks (>= 1) */
    double tolerance;          /* adjoint Poisson: stop when sum|pi - pi_prev| / sum|pi| < tolerance,
                                  pi = sum_q of the adjoint iterate, compared across checks */
    uint64_t max_sweeps;       /* adjoint Poisson: cap per step; 0 = none.  Reaching it returns
                                  LBM_ERR_POISSON_BUDGET */
    int binomial_checkpoints;  /* 0: uniform checkpoints every checkpoint_interval steps.  > 0:
                                  binomial checkpointing (Griewank's revolve schedule) with at most
                                  this many stored states besides the loaded one; the forward run
                                  then keeps no states, and the reverse pass keeps one step's */
    int krylov;                /* 1: solve each step's adjoint Poisson problem by BiCGSTAB (the
                                  transposed kinetic operator, as LBM_POISSON_KRYLOV does forward)
                                  to a relative residual of krylov_tolerance, instead of the
                                  transposed sweeps and their check of tolerance; a NaN/Inf
                                  adjoint right-hand side returns LBM_ERR_NONFINITE, restarts
                                  without progress LBM_ERR_POISSON_BUDGET as in the forward form */
    double krylov_tolerance;   /* 0: 1e-10 */
    int precision;             /* 0: the forward box is FP64.  1: the forward box is the mixed box
                                  (FP32 populations and fields, FP64 rest population, pressure and
                                  reductions); its checkpoints take 156 B/cell instead of 288, and
                                  the reverse pass differentiates the FP64 step at the mixed
                                  forward's states (fields converted to FP64), so the gradient
                                  carries the mixed forward's error (not bitwise reproducible
                                  against an FP64 forward) */
} lbm_adjoint_cfg;

typedef struct {
    double grad_kappa_f;       /* dJ/dk_f */
    uint64_t forward_steps;    /* steps of the forward run */
    uint64_t forward_sweeps;   /* Poisson sweeps of the forward run */
    uint64_t recompute_steps;  /* steps recomputed from checkpoints by the reverse pass */
    uint64_t adjoint_sweeps;   /* transposed Poisson sweeps of the reverse pass */
    double forward_ms;         /* wall time of lbm_adjoint_forward */
    double backward_ms;        /* wall time of lbm_adjoint_backward (recomputation included) */
} lbm_adjoint_stats;

lbm_status lbm_adjoint_create(const lbm_params* p, int device, const lbm_adjoint_cfg* cfg, lbm_adjoint** out);
void lbm_adjoint_destroy(lbm_adjoint* a);
/* Poisson settings of the forward run (lbm_set_poisson). */
lbm_status lbm_adjoint_set_poisson(lbm_adjoint* a, const lbm_poisson_cfg* cfg);
/* Loads the initial macro fields (host, physical layout; p may be NULL = 0)
 * and runs n_steps steps, keeping checkpoints.  sweeps: NULL for the Poisson
 * exits of the settings, else a fixed sweep count per step (lbm_step_replay). */
lbm_status lbm_adjoint_forward(lbm_adjoint* a, const double* phi, const double* rho, const double* u,
                               const double* v, const double* w, const double* p, int n_steps,
                               const uint64_t* sweeps);
/* Sweep count of each forward step (n_steps entries). */
lbm_status lbm_adjoint_sweeps(const lbm_adjoint* a, uint64_t* out);
/* A field of the forward run's final state (host, physical layout). */
lbm_status lbm_adjoint_download(const lbm_adjoint* a, lbm_field which, double* host);
/* Reverse pass.  lam_*: dJ/d(final field), host, NULL = 0.  grad_*: dJ/d(loaded
 * field), host, NULL = not wanted.  stats may be NULL. */
lbm_status lbm_adjoint_backward(lbm_adjoint* a, const double* lam_phi, const double* lam_rho, const double* lam_u,
                                const double* lam_v, const double* lam_w, const double* lam_p, double* grad_phi,
                                double* grad_rho, double* grad_u, double* grad_v, double* grad_w, double* grad_p,
                                lbm_adjoint_stats* stats);
/* Text of the last error on this object ("" if none); with a == NULL: why the
 * calling thread's last lbm_adjoint_create failed. */
const char* lbm_adjoint_last_error(const lbm_adjoint* a);
/* The binomial schedule of a reverse pass over n_steps steps with at most
 * `checkpoints` stored states, run dry (no device work): the forward steps it
 * recomputes and the most states it holds at once.  For sizing runs. */
lbm_status lbm_adjoint_schedule(int n_steps, int checkpoints, uint64_t* recompute_steps, int* peak_checkpoints);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
