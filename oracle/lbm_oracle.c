/*
 * lbm_oracle.c -- FP64 CPU restatement of the Inamuro two-phase D3Q15 step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  See lbm_oracle.h for the list of
 * reference functions restated here.  Every floating-point expression keeps the
 * operand order of the reference so that, compiled without FP contraction
 * (-ffp-contract=off, no -ffast-math), results are bitwise those of the
 * reference CPU build.  Per-cell loops may run in parallel (OpenMP): each cell
 * is independent, so the result does not depend on the thread count.  Global
 * sums keep the reference's serial x-outer / z-inner order.
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define Q 15

/* D3Q15 velocity set and weights: CPU/common.hpp:3-45 */
static const int EX[Q] = {0, 1, 0, 0, -1, 0, 0, 1, -1, 1, 1, -1, 1, -1, -1};
static const int EY[Q] = {0, 0, 1, 0, 0, -1, 0, 1, 1, -1, 1, -1, -1, 1, -1};
static const int EZ[Q] = {0, 0, 0, 1, 0, 0, -1, 1, 1, 1, -1, -1, -1, -1, 1};
static const double UC[Q] = {0.0, 1.0, 0.0, 0.0, -1.0, 0.0, 0.0,
                             1.0, -1.0, 1.0, 1.0, -1.0, 1.0, -1.0, -1.0};
static const double VC[Q] = {0.0, 0.0, 1.0, 0.0, 0.0, -1.0, 0.0,
                             1.0, 1.0, -1.0, 1.0, -1.0, -1.0, 1.0, -1.0};
static const double WC[Q] = {0.0, 0.0, 0.0, 1.0, 0.0, 0.0, -1.0,
                             1.0, 1.0, 1.0, -1.0, -1.0, -1.0, -1.0, 1.0};
static const double EI[Q] = {2.0 / 9.0,
                             1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                             1.0 / 72.0, 1.0 / 72.0, 1.0 / 72.0, 1.0 / 72.0,
                             1.0 / 72.0, 1.0 / 72.0, 1.0 / 72.0, 1.0 / 72.0};
static const double HI[Q] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
                             0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
static const double FI[Q] = {-7.0 / 3.0,
                             1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0,
                             1.0 / 24.0, 1.0 / 24.0, 1.0 / 24.0, 1.0 / 24.0,
                             1.0 / 24.0, 1.0 / 24.0, 1.0 / 24.0, 1.0 / 24.0};
/* x slip pairs (incoming, outgoing): CPU/Inamuro.cpp:592-593 */
static const int BPOS[5] = {1, 7, 9, 10, 12};
static const int BNEG[5] = {4, 8, 14, 13, 11};

enum { D_FX, D_FY, D_FZ, D_RX, D_RY, D_RZ, D_UX, D_UY, D_UZ, D_VX, D_VY, D_VZ,
       D_WX, D_WY, D_WZ, D_FLAP, D_ULAP, D_VLAP, D_WLAP, D_COUNT };

struct orc_state {
    orc_params P;
    long N;
    int first_step;
    double *f, *g, *h, *tmp, *img;        /* 15N each */
    double *phi, *rho, *u, *v, *w, *p, *p_prev, *pf;
    double *d[D_COUNT];
};

static inline long idx(const orc_state* s, int x, int y, int z)
{
    return ((long)z * s->P.ly + y) * s->P.lx + x;
}

/* Neighbour index for the stencils: x mirrored (lx-2 / 1), y and z periodic.
 * CPU/Inamuro.hpp:230-248. */
static inline long stencil_nb(const orc_state* s, int x, int y, int z, int k)
{
    int xp = x + EX[k], yp = y + EY[k], zp = z + EZ[k];
    const int lx = s->P.lx, ly = s->P.ly, lz = s->P.lz;
    if (s->P.periodic_x) {
        if (xp >= lx) xp = 0;
        if (xp < 0) xp = lx - 1;
    } else {
        if (xp >= lx) xp = lx - 2;
        if (xp < 0) xp = 1;
    }
    if (yp >= ly) yp = 0;
    if (yp < 0) yp = ly - 1;
    if (zp >= lz) zp = 0;
    if (zp < 0) zp = lz - 1;
    return idx(s, xp, yp, zp);
}

/* firstord: CPU/Inamuro.hpp:213-266 */
static void firstord(orc_state* s, const double* var, double* vx, double* vy, double* vz)
{
    const int lx = s->P.lx, ly = s->P.ly, lz = s->P.lz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < lz; ++z)
        for (int y = 0; y < ly; ++y)
            for (int x = 0; x < lx; ++x) {
                double ax = 0.0, ay = 0.0, az = 0.0;
                for (int k = 1; k < Q; ++k) {
                    const double val = var[stencil_nb(s, x, y, z, k)];
                    ax += val * UC[k];
                    ay += val * VC[k];
                    az += val * WC[k];
                }
                const long c = idx(s, x, y, z);
                vx[c] = ax / 10.0;
                vy[c] = ay / 10.0;
                vz[c] = az / 10.0;
            }
}

/* secondord: CPU/Inamuro.hpp:268-314 */
static void secondord(orc_state* s, const double* var, double* lap)
{
    const int lx = s->P.lx, ly = s->P.ly, lz = s->P.lz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < lz; ++z)
        for (int y = 0; y < ly; ++y)
            for (int x = 0; x < lx; ++x) {
                double acc = 0.0;
                for (int k = 1; k < Q; ++k) acc += var[stencil_nb(s, x, y, z, k)];
                const long c = idx(s, x, y, z);
                lap[c] = (acc - 14.0 * var[c]) / 5.0;
            }
}

/* collision: CPU/Inamuro.cpp:134-250 (EOS :843-847) */
static void collision(orc_state* s)
{
    const orc_params* P = &s->P;
    const double tmp1 = (P->mu_L - P->mu_G) / (P->rho_L - P->rho_G);
    double** d = s->d;
    firstord(s, s->u, d[D_UX], d[D_UY], d[D_UZ]);
    firstord(s, s->v, d[D_VX], d[D_VY], d[D_VZ]);
    firstord(s, s->w, d[D_WX], d[D_WY], d[D_WZ]);
    firstord(s, s->rho, d[D_RX], d[D_RY], d[D_RZ]);
    firstord(s, s->phi, d[D_FX], d[D_FY], d[D_FZ]);
    secondord(s, s->u, d[D_ULAP]);
    secondord(s, s->v, d[D_VLAP]);
    secondord(s, s->w, d[D_WLAP]);
    secondord(s, s->phi, d[D_FLAP]);

    const long N = s->N;
    const int first = s->first_step;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < N; ++c) {
        const double rho = s->rho[c], fei = s->phi[c];
        const double uu = s->u[c], vv = s->v[c], ww = s->w[c];
        const double fx = d[D_FX][c], fy = d[D_FY][c], fz = d[D_FZ][c];
        const double rx = d[D_RX][c], ry = d[D_RY][c], rz = d[D_RZ][c];
        const double u_x = d[D_UX][c], u_y = d[D_UY][c], u_z = d[D_UZ][c];
        const double v_x = d[D_VX][c], v_y = d[D_VY][c], v_z = d[D_VZ][c];
        const double w_x = d[D_WX][c], w_y = d[D_WY][c], w_z = d[D_WZ][c];
        const double mu = (rho - P->rho_G) * tmp1 + P->mu_G;
        const double sum_fei = fx * fx + fy * fy + fz * fz;
        const double sum_rho = rx * rx + ry * ry + rz * rz;
        const double fei2sum = d[D_FLAP][c];
        const double usq = uu * uu + vv * vv + ww * ww;
        const double p0 = fei * P->T / (1.0 - P->b * fei) - P->a * fei * fei;
        for (int i = 0; i < Q; ++i) {
            const double un = UC[i] * uu + VC[i] * vv + WC[i] * ww;
            const double fei_ei = UC[i] * fx + VC[i] * fy + WC[i] * fz;
            const double rho_ei = UC[i] * rx + VC[i] * ry + WC[i] * rz;
            const double ci_sq = UC[i] * UC[i] + VC[i] * VC[i] + WC[i] * WC[i];
            const double Gfei = 4.5 * (fei_ei * fei_ei) - 1.5 * sum_fei * ci_sq;
            const double Grho = 4.5 * (rho_ei * rho_ei) - 1.5 * sum_rho * ci_sq;
            const double fequ = HI[i] * fei +
                                FI[i] * (p0 - P->k_f * fei * fei2sum - P->k_f * sum_fei / 6.0) +
                                3.0 * EI[i] * fei * un +
                                EI[i] * P->k_f * Gfei;
            const double velPart = 1.0 + 3.0 * un - 1.5 * usq + 4.5 * un * un +
                                   1.5 * (P->taug - 0.5) * 2.0 *
                                       (UC[i] * UC[i] * u_x + UC[i] * VC[i] * u_y + UC[i] * WC[i] * u_z +
                                        VC[i] * UC[i] * v_x + VC[i] * VC[i] * v_y + VC[i] * WC[i] * v_z +
                                        WC[i] * UC[i] * w_x + WC[i] * VC[i] * w_y + WC[i] * WC[i] * w_z);
            const double gequ = EI[i] * velPart +
                                EI[i] * P->k_g / rho * Grho -
                                2.0 / 3.0 * FI[i] * P->k_g / rho * sum_rho;
            const long id = (long)i * N + c;
            if (first) {
                s->f[id] = fequ;
                s->g[id] = gequ;
            } else {
                s->f[id] = s->f[id] - (s->f[id] - fequ) / P->tauf;
                s->g[id] = s->g[id] - (s->g[id] - gequ) / P->taug +
                           3.0 * EI[i] / rho * mu *
                               (UC[i] * d[D_ULAP][c] + VC[i] * d[D_VLAP][c] + WC[i] * d[D_WLAP][c]);
            }
        }
    }
    s->first_step = 0;
}

/* Periodic streaming f_q(x) <- f_q(x - c_q): CPU/Inamuro.cpp:252-287 (push
 * form there; the copy is the same).  Result lands in s->tmp, then swapped. */
static void stream(orc_state* s, double** dist)
{
    const int lx = s->P.lx, ly = s->P.ly, lz = s->P.lz;
    const long N = s->N;
    double* in = *dist;
    double* out = s->tmp;
#pragma omp parallel for collapse(2) schedule(static)
    for (int q = 0; q < Q; ++q)
        for (int z = 0; z < lz; ++z)
            for (int y = 0; y < ly; ++y)
                for (int x = 0; x < lx; ++x) {
                    const int xs = (x - EX[q] + lx) % lx;
                    const int ys = (y - EY[q] + ly) % ly;
                    const int zs = (z - EZ[q] + lz) % lz;
                    out[(long)q * N + idx(s, x, y, z)] = in[(long)q * N + idx(s, xs, ys, zs)];
                }
    s->tmp = in;
    *dist = out;
}

/* slipBounceBack: CPU/Inamuro.cpp:589-623 */
static void bounce(orc_state* s, double* dist)
{
    if (s->P.periodic_x) return;
    const int lx = s->P.lx, ly = s->P.ly, lz = s->P.lz;
    const long N = s->N;
    for (int y = 0; y < ly; ++y)
        for (int z = 0; z < lz; ++z)
            for (int r = 0; r < 5; ++r) {
                const long c = idx(s, 0, y, z);
                dist[(long)BPOS[r] * N + c] = dist[(long)BNEG[r] * N + c];
            }
    for (int y = 0; y < ly; ++y)
        for (int z = 0; z < lz; ++z)
            for (int r = 0; r < 5; ++r) {
                const long c = idx(s, lx - 1, y, z);
                dist[(long)BNEG[r] * N + c] = dist[(long)BPOS[r] * N + c];
            }
}

/* getMacro: CPU/Inamuro.cpp:294-346 */
static void get_macro(orc_state* s)
{
    const orc_params* P = &s->P;
    const long N = s->N;
    const double fei_avg = (P->fei_L + P->fei_G) / 2.0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < N; ++c) {
        double fei_local = 0.0;
        for (int i = 0; i < Q; ++i) fei_local += s->f[(long)i * N + c];
        s->phi[c] = fei_local;
        double density;
        if (fei_local <= P->fei_G) {
            density = P->rho_G;
        } else if (fei_local >= P->fei_L) {
            density = P->rho_L;
        } else {
            const double arg = (fei_local - fei_avg) / (P->fei_L - P->fei_G) * M_PI;
            density = (P->rho_L - P->rho_G) / 2.0 * (sin(arg) + 1.0) + P->rho_G;
        }
        s->rho[c] = density;
        double uu = 0.0, vv = 0.0, ww = 0.0;
        for (int i = 1; i < Q; ++i) {
            const double gv = s->g[(long)i * N + c];
            uu += UC[i] * gv;
            vv += VC[i] * gv;
            ww += WC[i] * gv;
        }
        s->u[c] = uu;
        s->v[c] = vv;
        s->w[c] = ww;
    }
}

/* collision_p: CPU/Inamuro.cpp:755-778 (also the shadow map's collision,
 * GPU/InamuroCUDA.cu:503-537 with unit relaxation). */
static void collision_p(orc_state* s, double* hh)
{
    const long N = s->N;
    double* const* d = s->d;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < N; ++c) {
        const double tauh = 1.0 / s->rho[c] + 0.5;
        for (int k = 0; k < Q; ++k) {
            const double hequ = EI[k] * s->p[c];
            const long id = (long)k * N + c;
            hh[id] = hh[id] - (hh[id] - hequ) / tauh -
                     (EI[k] / 3.0) * (d[D_UX][c] + d[D_VY][c] + d[D_WZ][c]);
        }
    }
}

/* getp: CPU/Inamuro.cpp:779-793 */
static void sum_h(const orc_state* s, const double* hh, double* out)
{
    const long N = s->N;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < N; ++c) {
        double acc = 0.0;
        for (int i = 0; i < Q; ++i) acc += hh[(long)i * N + c];
        out[c] = acc;
    }
}

/* Serial sum over cells in the reference's x-outer / z-inner order. */
static double sum_xouter(const orc_state* s, const double* a)
{
    double acc = 0.0;
    for (int x = 0; x < s->P.lx; ++x)
        for (int y = 0; y < s->P.ly; ++y)
            for (int z = 0; z < s->P.lz; ++z) acc += a[idx(s, x, y, z)];
    return acc;
}

static double relative(double num, double den)
{
    if (den > 0.0) return num / den;
    return num == 0.0 ? 0.0 : INFINITY;
}

/* Kinetic fixed-point residual F(h,p) = BS[C(h,p)]:
 * GPU/InamuroCUDA.cu:1987-2057, 1114-1171; DUAL_RESIDUAL_CONTRACT.md:24-37. */
static int dual_residual(orc_state* s, double g, orc_step_info* info)
{
    const long N = s->N;
    memcpy(s->img, s->h, sizeof(double) * Q * N);
    collision_p(s, s->img);
    double* img = s->img;
    stream(s, &img);           /* result in img, old img buffer becomes tmp */
    s->img = img;
    bounce(s, s->img);
    sum_h(s, s->h, s->pf);
    double t[6] = {0, 0, 0, 0, 0, 0};
    for (int x = 0; x < s->P.lx; ++x)
        for (int y = 0; y < s->P.ly; ++y)
            for (int z = 0; z < s->P.lz; ++z) {
                const long c = idx(s, x, y, z);
                for (int q = 0; q < Q; ++q) {
                    const double hv = s->h[(long)q * N + c];
                    const double iv = s->img[(long)q * N + c];
                    const double ge = EI[q] * g;
                    t[0] += fabs(hv - iv);
                    t[1] += fabs(hv - ge);
                    t[2] += fabs(iv - ge);
                }
                t[3] += fabs(s->p[c] - s->pf[c]);
                t[4] += fabs(s->p[c] - g);
                t[5] += fabs(s->pf[c] - g);
            }
    for (int i = 0; i < 6; ++i)
        if (!isfinite(t[i])) return ORC_ERR_NONFINITE;
    info->fp_h_l1 = t[0];
    info->fp_h_scale = t[1] > t[2] ? t[1] : t[2];
    info->fp_h_rel = relative(t[0], info->fp_h_scale);
    info->fp_p_l1 = t[3];
    info->fp_p_scale = t[4] > t[5] ? t[4] : t[5];
    info->fp_p_rel = relative(t[3], info->fp_p_scale);
    info->fp_rel = info->fp_h_rel > info->fp_p_rel ? info->fp_h_rel : info->fp_p_rel;
    if (!isfinite(info->fp_rel)) return ORC_ERR_NONFINITE;
    return ORC_OK;
}

/* The reference's scalar Poisson form (GPU only there): Jacobi sweeps of
 * scalarPressureJacobiKernel, GPU/InamuroCUDA.cu:864-901 (x neighbours
 * mirrored at the slip walls, pressure_bounce_direction :846-862), with the
 * gauge and relative-change check of check_residual (:1977-2140) every
 * check_interval sweeps.  u_x is already projected.  x-outer sums. */
static int poisson_scalar(orc_state* s, uint64_t replay, orc_step_info* info, double target)
{
    const orc_params* P = &s->P;
    const int lx = P->lx, ly = P->ly, lz = P->lz;
    const long N = s->N;
    const double cell_count = (double)lx * ly * lz;
    const double* ux = s->d[D_UX];
    const double* vy = s->d[D_VY];
    const double* wz = s->d[D_WZ];
    uint64_t iter = 0;
    for (;;) {
        ++iter;
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < lz; ++z)
            for (int y = 0; y < ly; ++y)
                for (int x = 0; x < lx; ++x) {
                    double nsum = 0.0;
                    for (int q = 1; q < Q; ++q) {
                        int xs = x - EX[q], ys = y - EY[q], zs = z - EZ[q];
                        if (!P->periodic_x && xs < 0) xs = 1;
                        else if (!P->periodic_x && xs >= lx) xs = lx - 2;
                        else if (xs < 0) xs += lx;
                        else if (xs >= lx) xs -= lx;
                        if (ys < 0) ys += ly; else if (ys >= ly) ys -= ly;
                        if (zs < 0) zs += lz; else if (zs >= lz) zs -= lz;
                        nsum += s->p[idx(s, xs, ys, zs)];
                    }
                    const long c = idx(s, x, y, z);
                    const double div_u = ux[c] + vy[c] + wz[c];
                    const double rhs = P->scalar_source_scale * s->rho[c] * div_u;
                    s->pf[c] = (nsum - 5.0 * rhs) / 14.0;
                }
        memcpy(s->p, s->pf, sizeof(double) * N);
        int converged = 0;
        if (iter % (uint64_t)P->check_interval == 0) {
            const double shift = sum_xouter(s, s->p) / cell_count - target;
            if (!isfinite(shift)) return ORC_ERR_NONFINITE;
            if (fabs(shift) > info->gauge_max_shift) info->gauge_max_shift = fabs(shift);
            for (long c = 0; c < N; ++c) s->p[c] -= shift;
            double err1 = 0.0, err2 = 0.0;
            for (int x = 0; x < lx; ++x)
                for (int y = 0; y < ly; ++y)
                    for (int z = 0; z < lz; ++z) {
                        const long c = idx(s, x, y, z);
                        err1 += fabs(s->p[c] - s->p_prev[c]);
                        err2 += fabs(s->p[c]);
                        s->p_prev[c] = s->p[c];
                    }
            if (!isfinite(err1) || !isfinite(err2)) return ORC_ERR_NONFINITE;
            info->pressure_l1_delta = err1;
            info->pressure_l1_norm = err2;
            info->relative_error = relative(err1, err2);
            converged = info->relative_error < P->tol;
        }
        if (replay) {
            if (iter == replay) break;
        } else if (converged) {
            break;
        }
        if (!replay && P->max_sweeps && iter >= P->max_sweeps) {
            info->sweeps = iter;
            return ORC_ERR_BUDGET;
        }
    }
    info->sweeps = iter;
    return ORC_OK;
}

/* sourceAwareHHInitKernel (GPU/InamuroCUDA.cu:903-929): the solve's start
 * h = E_q p - scale tau_h (E_q / 3) s, s the projected u_x + v_y + w_z. */
static void source_aware_init(orc_state* s)
{
    const long N = s->N;
    for (long c = 0; c < N; ++c) {
        const double tauh = 1.0 / s->rho[c] + 0.5;
        const double div = s->d[D_UX][c] + s->d[D_VY][c] + s->d[D_WZ][c];
        for (int q = 0; q < Q; ++q)
            s->h[(long)q * N + c] = EI[q] * s->p[c] - s->P.source_aware_scale * tauh * ((EI[q] / 3.0) * div);
    }
}

/* The reference's one-pass Poisson form with its accelerators (GPU only
 * there): collisionStreamBoundaryPressureKernel (GPU/InamuroCUDA.cu:780-844),
 * Anderson-m1 (:931-1013, 2230-2275), the check with the two-grid
 * correction (:1198-1255, 1284-1328, 2057-2156).  State: the pre-collision
 * h and p = sum_q h.  x-outer sums; Anderson's inner products cell-major. */
static int poisson_onepass(orc_state* s, uint64_t replay, orc_step_info* info, double target)
{
    const orc_params* P = &s->P;
    const int lx = P->lx, ly = P->ly, lz = P->lz;
    const long N = s->N;
    const double cell_count = (double)lx * ly * lz;
    const double relax = P->pressure_relax_scale != 0.0 ? P->pressure_relax_scale : 1.0;
    const double omega = P->fixed_point_relax != 0.0 ? P->fixed_point_relax : 1.0;
    double* prev_r = NULL;
    double* prev_img = NULL;
    if (P->anderson_m1) {
        prev_r = (double*)malloc(sizeof(double) * Q * N);
        prev_img = (double*)malloc(sizeof(double) * Q * N);
        if (!prev_r || !prev_img) {
            free(prev_r);
            free(prev_img);
            return ORC_ERR_OOM;
        }
    }
    const int bs = 4, bxn = (lx + bs - 1) / bs, byn = (ly + bs - 1) / bs, bzn = (lz + bs - 1) / bs;
    double* bsum = P->two_grid ? (double*)calloc((size_t)bxn * byn * bzn, sizeof(double)) : NULL;
    int has_history = 0, status = ORC_OK;
    uint64_t iter = 0;
    for (;;) {
        ++iter;
#pragma omp parallel for collapse(2) schedule(static)
        for (int z = 0; z < lz; ++z)
            for (int y = 0; y < ly; ++y)
                for (int x = 0; x < lx; ++x) {
                    double h[Q];
                    for (int q = 0; q < Q; ++q) {
                        int xs = x - EX[q], ys = y - EY[q], zs = z - EZ[q];
                        if (xs < 0) xs += lx; else if (xs >= lx) xs -= lx;
                        if (ys < 0) ys += ly; else if (ys >= ly) ys -= ly;
                        if (zs < 0) zs += lz; else if (zs >= lz) zs -= lz;
                        const long src = idx(s, xs, ys, zs);
                        const double tauh = 1.0 / s->rho[src] + 0.5;
                        const double hequ = EI[q] * s->p[src];
                        const double h_old = s->h[(long)q * N + src];
                        const double div = s->d[D_UX][src] + s->d[D_VY][src] + s->d[D_WZ][src];
                        h[q] = h_old - relax * (h_old - hequ) / tauh - (EI[q] / 3.0) * div;
                    }
                    if (!P->periodic_x && x == 0) {
                        h[1] = h[4]; h[7] = h[8]; h[9] = h[14]; h[10] = h[13]; h[12] = h[11];
                    } else if (!P->periodic_x && x == lx - 1) {
                        h[4] = h[1]; h[8] = h[7]; h[14] = h[9]; h[13] = h[10]; h[11] = h[12];
                    }
                    const long c = idx(s, x, y, z);
                    double psum = 0.0;
                    for (int q = 0; q < Q; ++q) {
                        const double h_old = s->h[(long)q * N + c];
                        const double hv = h_old + omega * (h[q] - h_old);
                        s->img[(long)q * N + c] = hv;
                        psum += hv;
                    }
                    s->pf[c] = psum;
                }
        if (P->anderson_m1) {
            if (!has_history) {
                for (long i = 0; i < (long)Q * N; ++i) {
                    prev_r[i] = s->img[i] - s->h[i];
                    prev_img[i] = s->img[i];
                }
                has_history = 1;
            } else {
                double num = 0.0, den = 0.0;
                for (long c = 0; c < N; ++c)
                    for (int q = 0; q < Q; ++q) {
                        const long i = (long)q * N + c;
                        const double r = s->img[i] - s->h[i];
                        const double dl = r - prev_r[i];
                        num += prev_r[i] * dl;
                        den += dl * dl;
                    }
                double alpha = 1.0;
                if (den > 1.0e-300) alpha = -num / den;
                if (!isfinite(alpha)) alpha = 1.0;
                const double lo = -P->anderson_beta_max, hi = 1.0 + P->anderson_beta_max;
                alpha = alpha < lo ? lo : (alpha > hi ? hi : alpha);
                for (long c = 0; c < N; ++c) {
                    double psum = 0.0;
                    for (int q = 0; q < Q; ++q) {
                        const long i = (long)q * N + c;
                        const double cur = s->img[i];
                        const double acc = (1.0 - alpha) * prev_img[i] + alpha * cur;
                        prev_r[i] = cur - s->h[i];
                        prev_img[i] = cur;
                        s->img[i] = acc;
                        psum += acc;
                    }
                    s->pf[c] = psum;
                }
            }
        }
        double* t = s->h;
        s->h = s->img;
        s->img = t;
        memcpy(s->p, s->pf, sizeof(double) * N);
        int converged = 0;
        if (iter % (uint64_t)P->check_interval == 0) {
            const double shift = sum_xouter(s, s->p) / cell_count - target;
            if (!isfinite(shift)) { status = ORC_ERR_NONFINITE; break; }
            if (fabs(shift) > info->gauge_max_shift) info->gauge_max_shift = fabs(shift);
            for (long c = 0; c < N; ++c) {
                s->p[c] -= shift;
                for (int q = 0; q < Q; ++q) s->h[(long)q * N + c] -= EI[q] * shift;
            }
            if (bsum) {
                memset(bsum, 0, sizeof(double) * bxn * byn * bzn);
                for (int z = 0; z < lz; ++z)
                    for (int y = 0; y < ly; ++y)
                        for (int x = 0; x < lx; ++x) {
                            const long c = idx(s, x, y, z);
                            bsum[((z / bs) * byn + y / bs) * bxn + x / bs] += s->p[c] - s->p_prev[c];
                        }
            }
            double err1 = 0.0, err2 = 0.0;
            for (int x = 0; x < lx; ++x)
                for (int y = 0; y < ly; ++y)
                    for (int z = 0; z < lz; ++z) {
                        const long c = idx(s, x, y, z);
                        err1 += fabs(s->p[c] - s->p_prev[c]);
                        err2 += fabs(s->p[c]);
                        s->p_prev[c] = s->p[c];
                    }
            if (!isfinite(err1) || !isfinite(err2)) { status = ORC_ERR_NONFINITE; break; }
            info->pressure_l1_delta = err1;
            info->pressure_l1_norm = err2;
            info->relative_error = relative(err1, err2);
            converged = info->relative_error < P->tol;
            if (bsum && !converged && err1 > 0.0) {
                for (int z = 0; z < lz; ++z)
                    for (int y = 0; y < ly; ++y)
                        for (int x = 0; x < lx; ++x) {
                            const int bx = x / bs, by = y / bs, bz = z / bs;
                            const int x1 = (bx + 1) * bs < lx ? (bx + 1) * bs : lx;
                            const int y1 = (by + 1) * bs < ly ? (by + 1) * bs : ly;
                            const int z1 = (bz + 1) * bs < lz ? (bz + 1) * bs : lz;
                            const int cells = (x1 - bx * bs) * (y1 - by * bs) * (z1 - bz * bs);
                            const double corr = P->two_grid_strength * bsum[(bz * byn + by) * bxn + bx] / (double)cells;
                            const long c = idx(s, x, y, z);
                            s->p[c] += corr;
                            s->p_prev[c] = s->p[c];
                            for (int q = 0; q < Q; ++q) s->h[(long)q * N + c] += EI[q] * corr;
                        }
            }
        }
        if (replay) {
            if (iter == replay) break;
        } else if (converged) {
            break;
        }
        if (!replay && P->max_sweeps && iter >= P->max_sweeps) {
            status = ORC_ERR_BUDGET;
            break;
        }
    }
    free(prev_r);
    free(prev_img);
    free(bsum);
    info->sweeps = iter;
    return status;
}

/* solvePressurePoisson: CPU/Inamuro.cpp:624-724 */
static int poisson(orc_state* s, uint64_t replay, orc_step_info* info)
{
    const orc_params* P = &s->P;
    const long N = s->N;
    const double cell_count = (double)P->lx * P->ly * P->lz;
    double* ux = s->d[D_UX];
    const double* vy = s->d[D_VY];
    const double* wz = s->d[D_WZ];
    double divergence_sum = 0.0, pressure_sum = 0.0;
    for (int x = 0; x < P->lx; ++x)
        for (int y = 0; y < P->ly; ++y)
            for (int z = 0; z < P->lz; ++z) {
                const long c = idx(s, x, y, z);
                divergence_sum += ux[c] + vy[c] + wz[c];
                pressure_sum += s->p[c];
            }
    const double divergence_mean = divergence_sum / cell_count;
    const double target = pressure_sum / cell_count;
    if (!isfinite(divergence_mean) || !isfinite(target)) return ORC_ERR_NONFINITE;
    for (long c = 0; c < N; ++c) ux[c] -= divergence_mean;
    info->divergence_mean = divergence_mean;
    info->gauge_target = target;
    info->gauge_max_shift = 0.0;
    if (P->poisson_form == 1) return poisson_scalar(s, replay, info, target);
    if (P->source_aware_init) source_aware_init(s);
    if (P->poisson_form == 2) return poisson_onepass(s, replay, info, target);

    uint64_t iter = 0;
    for (;;) {
        ++iter;
        collision_p(s, s->h);
        stream(s, &s->h);
        bounce(s, s->h);
        sum_h(s, s->h, s->p);
        int converged = 0;
        if (iter % (uint64_t)P->check_interval == 0) {
            const double shift = sum_xouter(s, s->p) / cell_count - target;
            if (!isfinite(shift)) return ORC_ERR_NONFINITE;
            if (fabs(shift) > info->gauge_max_shift) info->gauge_max_shift = fabs(shift);
#pragma omp parallel for schedule(static)
            for (long c = 0; c < N; ++c) {
                s->p[c] -= shift;
                for (int q = 0; q < Q; ++q) s->h[(long)q * N + c] -= EI[q] * shift;
            }
            int fp_ok = 1;
            if (P->dual) {
                const int st = dual_residual(s, target, info);
                if (st != ORC_OK) return st;
                fp_ok = info->fp_rel < P->tol;
            }
            /* two-grid correction (GPU/InamuroCUDA.cu:1198-1255, 1284-1328,
               2149-2156): 4^3 block sums of the change before p_prev moves */
            const int bs = 4, bxn = (P->lx + bs - 1) / bs, byn = (P->ly + bs - 1) / bs, bzn = (P->lz + bs - 1) / bs;
            double* bsum = NULL;
            if (P->two_grid) {
                bsum = (double*)calloc((size_t)bxn * byn * bzn, sizeof(double));
                if (!bsum) return ORC_ERR_OOM;
                for (int z = 0; z < P->lz; ++z)
                    for (int y = 0; y < P->ly; ++y)
                        for (int x = 0; x < P->lx; ++x) {
                            const long c = idx(s, x, y, z);
                            bsum[((z / bs) * byn + y / bs) * bxn + x / bs] += s->p[c] - s->p_prev[c];
                        }
            }
            /* getError: CPU/Inamuro.cpp:726-753 */
            double err1 = 0.0, err2 = 0.0;
            for (int x = 0; x < P->lx; ++x)
                for (int y = 0; y < P->ly; ++y)
                    for (int z = 0; z < P->lz; ++z) {
                        const long c = idx(s, x, y, z);
                        err1 += fabs(s->p[c] - s->p_prev[c]);
                        err2 += fabs(s->p[c]);
                        s->p_prev[c] = s->p[c];
                    }
            if (!isfinite(err1) || !isfinite(err2)) return ORC_ERR_NONFINITE;
            const double error = relative(err1, err2);
            info->pressure_l1_delta = err1;
            info->pressure_l1_norm = err2;
            info->relative_error = error;
            converged = (error < P->tol) && fp_ok;
            if (bsum && !converged && err1 > 0.0) {
                for (int z = 0; z < P->lz; ++z)
                    for (int y = 0; y < P->ly; ++y)
                        for (int x = 0; x < P->lx; ++x) {
                            const int bx = x / bs, by = y / bs, bz = z / bs;
                            const int x1 = (bx + 1) * bs < P->lx ? (bx + 1) * bs : P->lx;
                            const int y1 = (by + 1) * bs < P->ly ? (by + 1) * bs : P->ly;
                            const int z1 = (bz + 1) * bs < P->lz ? (bz + 1) * bs : P->lz;
                            const int cells = (x1 - bx * bs) * (y1 - by * bs) * (z1 - bz * bs);
                            const double corr = P->two_grid_strength * bsum[(bz * byn + by) * bxn + bx] / (double)cells;
                            const long c = idx(s, x, y, z);
                            s->p[c] += corr;
                            s->p_prev[c] = s->p[c];
                            for (int q = 0; q < Q; ++q) s->h[(long)q * N + c] += EI[q] * corr;
                        }
            }
            free(bsum);
        }
        if (replay) {
            if (iter == replay) break;
        } else if (converged) {
            break;
        }
        if (!replay && P->max_sweeps && iter >= P->max_sweeps) {
            info->sweeps = iter;
            return ORC_ERR_BUDGET;
        }
    }
    info->sweeps = iter;
    return ORC_OK;
}

/* correct_uvw + update_hh: CPU/Inamuro.cpp:794-840 */
static void correct_and_reset(orc_state* s)
{
    const int lx = s->P.lx, ly = s->P.ly, lz = s->P.lz;
    const long N = s->N;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < lz; ++z)
        for (int y = 0; y < ly; ++y)
            for (int x = 0; x < lx; ++x) {
                int x_e, x_w;
                if (s->P.periodic_x) {
                    x_e = (x == lx - 1) ? 0 : x + 1;
                    x_w = (x == 0) ? lx - 1 : x - 1;
                } else {
                    x_e = (x == lx - 1) ? lx - 2 : x + 1;
                    x_w = (x == 0) ? 1 : x - 1;
                }
                const int y_n = (y == ly - 1) ? 0 : y + 1;
                const int y_s = (y == 0) ? ly - 1 : y - 1;
                const int z_n = (z == lz - 1) ? 0 : z + 1;
                const int z_s = (z == 0) ? lz - 1 : z - 1;
                const long c = idx(s, x, y, z);
                const double inv_2rho = 1.0 / (2.0 * s->rho[c]);
                s->u[c] -= (s->p[idx(s, x_e, y, z)] - s->p[idx(s, x_w, y, z)]) * inv_2rho;
                s->v[c] -= (s->p[idx(s, x, y_n, z)] - s->p[idx(s, x, y_s, z)]) * inv_2rho;
                s->w[c] -= (s->p[idx(s, x, y, z_n)] - s->p[idx(s, x, y, z_s)]) * inv_2rho;
            }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < N; ++c)
        for (int i = 0; i < Q; ++i) s->h[(long)i * N + c] = s->p[c] * EI[i];
}

int orc_step(orc_state* s, uint64_t replay, orc_step_info* info)
{
    orc_step_info local;
    if (!info) info = &local;
    memset(info, 0, sizeof(*info));
    /* performTimeStep: CPU/Inamuro.cpp:347-363 */
    collision(s);
    stream(s, &s->f);
    stream(s, &s->g);
    bounce(s, s->f);
    bounce(s, s->g);
    get_macro(s);
    const int st = poisson(s, replay, info);
    if (st != ORC_OK) return st;
    correct_and_reset(s);
    info->mass = sum_xouter(s, s->phi);
    return ORC_OK;
}

orc_state* orc_create(const orc_params* prm,
                      const double* phi, const double* rho,
                      const double* u, const double* v, const double* w,
                      const double* p)
{
    if (!prm || prm->lx < 2 || prm->ly < 1 || prm->lz < 1 || prm->check_interval <= 0) return NULL;
    if (prm->poisson_form < 0 || prm->poisson_form > 2 || (prm->poisson_form != 0 && prm->dual)) return NULL;
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    if (!s) return NULL;
    s->P = *prm;
    s->N = (long)prm->lx * prm->ly * prm->lz;
    s->first_step = 1;
    const long N = s->N;
    double** pops[5] = {&s->f, &s->g, &s->h, &s->tmp, &s->img};
    for (int i = 0; i < 5; ++i) *pops[i] = (double*)calloc((size_t)Q * N, sizeof(double));
    double** scal[8] = {&s->phi, &s->rho, &s->u, &s->v, &s->w, &s->p, &s->p_prev, &s->pf};
    for (int i = 0; i < 8; ++i) *scal[i] = (double*)calloc((size_t)N, sizeof(double));
    for (int i = 0; i < D_COUNT; ++i) s->d[i] = (double*)calloc((size_t)N, sizeof(double));
    int ok = 1;
    for (int i = 0; i < 5; ++i) ok &= (*pops[i] != NULL);
    for (int i = 0; i < 8; ++i) ok &= (*scal[i] != NULL);
    for (int i = 0; i < D_COUNT; ++i) ok &= (s->d[i] != NULL);
    if (!ok) {
        orc_destroy(s);
        return NULL;
    }
    const size_t nb = sizeof(double) * (size_t)N;
    memcpy(s->phi, phi, nb);
    memcpy(s->rho, rho, nb);
    memcpy(s->u, u, nb);
    memcpy(s->v, v, nb);
    memcpy(s->w, w, nb);
    if (p) memcpy(s->p, p, nb);
    /* h starts at zero (CPU/Inamuro.cpp:516), p_prev at zero (:634). */
    return s;
}

void orc_destroy(orc_state* s)
{
    if (!s) return;
    free(s->f); free(s->g); free(s->h); free(s->tmp); free(s->img);
    free(s->phi); free(s->rho); free(s->u); free(s->v); free(s->w);
    free(s->p); free(s->p_prev); free(s->pf);
    for (int i = 0; i < D_COUNT; ++i) free(s->d[i]);
    free(s);
}

void orc_get_fields(const orc_state* s, double* phi, double* rho,
                    double* u, double* v, double* w, double* p)
{
    const size_t nb = sizeof(double) * (size_t)s->N;
    if (phi) memcpy(phi, s->phi, nb);
    if (rho) memcpy(rho, s->rho, nb);
    if (u) memcpy(u, s->u, nb);
    if (v) memcpy(v, s->v, nb);
    if (w) memcpy(w, s->w, nb);
    if (p) memcpy(p, s->p, nb);
}

void orc_get_populations(const orc_state* s, double* f, double* g, double* h)
{
    const size_t nb = sizeof(double) * (size_t)Q * (size_t)s->N;
    if (f) memcpy(f, s->f, nb);
    if (g) memcpy(g, s->g, nb);
    if (h) memcpy(h, s->h, nb);
}

void orc_get_derivatives(const orc_state* s, double* out19)
{
    for (int i = 0; i < D_COUNT; ++i)
        memcpy(out19 + (size_t)i * s->N, s->d[i], sizeof(double) * (size_t)s->N);
}

/* initializeDroplets: GPU/Inamuro.cpp:491-566 */
static void place_droplet(int lx, int ly, int lz, double radius, int use_tanh, double iw,
                          double fei_max, double fei_min, double rho_L, double rho_G,
                          double cx, double cy, double cz, double vz,
                          double* phi, double* rho, double* w)
{
    for (int x = 0; x < lx; ++x)
        for (int y = 0; y < ly; ++y)
            for (int z = 1; z < lz + 1; ++z) {
                const double dx = x - cx;
                const double dy = y - cy;
                const double dz = (z - 1) - cz;
                const double r = sqrt(dx * dx + dy * dy + dz * dz);
                double liquid_fraction = 0.0;
                if (use_tanh)
                    liquid_fraction = 0.5 * (1.0 - tanh((r - radius) / iw));
                else if (r < radius)
                    liquid_fraction = 1.0;
                if (liquid_fraction > 0.0) {
                    const long c = ((long)(z - 1) * ly + y) * lx + x;
                    const double local_fei = fei_min + liquid_fraction * (fei_max - fei_min);
                    if (local_fei > phi[c]) {
                        phi[c] = local_fei;
                        rho[c] = rho_G + liquid_fraction * (rho_L - rho_G);
                        w[c] = vz * liquid_fraction;
                    }
                }
            }
}

void orc_init_droplets(int lx, int ly, int lz, double DD,
                       double fei_max, double fei_min,
                       double rho_L, double rho_G,
                       int single_droplet, int tanh_profile,
                       double init_velocity, double interface_width,
                       double cx_in, double cy_in, double cz_in,
                       double separation_in, double offset_x,
                       double* phi, double* rho, double* w)
{
    const double radius = DD / 2.0;
    const double cy_default = ly / 2.0;
    const double cz_default = lz / 2.0;
    const double iw = (interface_width > 0.0) ? interface_width : 2.0;
    if (single_droplet) {
        const double cx = (cx_in >= 0.0) ? cx_in : lx / 2.0;
        const double cy = (cy_in >= 0.0) ? cy_in : cy_default;
        const double cz = (cz_in >= 0.0) ? cz_in : cz_default;
        place_droplet(lx, ly, lz, radius, tanh_profile, iw, fei_max, fei_min, rho_L, rho_G,
                      cx, cy, cz, init_velocity, phi, rho, w);
        return;
    }
    const double cx = (cx_in >= 0.0) ? cx_in : 0.0;
    const double cy = (cy_in >= 0.0) ? cy_in : cy_default;
    const double separation = (separation_in >= 0.0) ? separation_in : DD;
    const double cx1 = cx - 0.5 * offset_x;
    const double cx2 = cx + 0.5 * offset_x;
    const double cz1 = (cz_in >= 0.0) ? cz_in + separation : cz_default + separation;
    const double cz2 = (cz_in >= 0.0) ? cz_in - separation : cz_default - separation;
    place_droplet(lx, ly, lz, radius, tanh_profile, iw, fei_max, fei_min, rho_L, rho_G,
                  cx1, cy, cz1, -init_velocity, phi, rho, w);
    place_droplet(lx, ly, lz, radius, tanh_profile, iw, fei_max, fei_min, rho_L, rho_G,
                  cx2, cy, cz2, init_velocity, phi, rho, w);
}
