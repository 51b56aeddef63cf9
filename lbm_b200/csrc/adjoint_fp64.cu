// adjoint_fp64.cu -- hand-written adjoints (reverse-mode derivatives) of the
// explicit kernels of the FP64 step, each behind a forward/backward pair of
// the C ABI (lbm_collide_forward/backward, lbm_moments_forward/backward,
// lbm_correct_forward/backward).  The reference has no derivatives; these are
// the building blocks of a gradient through the time step.
//
// Given the adjoint (dJ/d output) of a kernel's outputs, a backward call
// returns the adjoint of its inputs at the same state, i.e. the transpose of
// the kernel's Jacobian applied to the output adjoint:
//   collide  (f*, g* of the previous step, phi, rho, u, v, w)
//              -> (f*, g*, u_x, v_y, w_z)          CPU/Inamuro.cpp:134-250
//   moments  (f*, g*) -> (phi, rho, u*, v*, w*)     CPU/Inamuro.cpp:294-346
//   correct  (u*, v*, w*, p, rho) -> (u, v, w)     CPU/Inamuro.cpp:794-823
// The pull stream is a permutation, so its transpose is a push; the stencils'
// transposes gather the per-cell stencil adjoints from x - c_k.  With the
// reference's x slip walls (CPU/Inamuro.cpp:589-623) the overwrite after the
// pull is transposed too (slip_T: a discarded incoming population gets 0, its
// mirror gains its adjoint), and so are the stencils' and the correction's
// mirrored x neighbours (x - 1 -> 1 at x = 0, x + 1 -> lx - 2 at x = lx - 1,
// CPU/Inamuro.hpp:230-248).  Derivatives are exact for the real-number map;
// they match centred finite differences of the FP64 forward kernels on both
// x boundaries (tests/test_gpu_adjoint.py).
#include <cuda_runtime.h>
#include <math_constants.h>

#include <string>
#include <type_traits>

#include "../../include/lbm_b200.h"
#include "adjoint.hpp"
#include "lbm_solver.cuh"
#include "phys_host.hpp"

namespace lbm {
namespace {

__device__ __forceinline__ bool cell_xyz(const Geom& g, int& x, int& y, int& z)
{
    x = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    z = blockIdx.z;
    return x < g.lx && y < g.ly;
}

// Periodic neighbour (x + dx, y + dy, z + dz), |d| <= 1.
__device__ __forceinline__ long long nb(const Geom& g, int x, int y, int z, int dx, int dy, int dz)
{
    x += dx;
    y += dy;
    z += dz;
    x = x < 0 ? x + g.lx : (x >= g.lx ? x - g.lx : x);
    y = y < 0 ? y + g.ly : (y >= g.ly ? y - g.ly : y);
    z = z < 0 ? z + g.lz : (z >= g.lz ? z - g.lz : z);
    return cell_of(g, x, y, z);
}

// Gradient (/10) and laplacian (/5) stencils of one field at a cell, x
// neighbours mirrored at the slip walls as in the forward collision.
__device__ __forceinline__ void grad_lap(const double* __restrict__ f, const Geom& g, int x, int y, int z,
                                         long long c, double& gx, double& gy, double& gz, double& lap)
{
    double ax = 0.0, ay = 0.0, az = 0.0, al = 0.0;
    const Mirror m(g, x, y, z);
    static_for<1, Q>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const double val = f[stencil_nb<k>(g, m, x, y, z)];
        ax += cx(k) * val;
        ay += cy(k) * val;
        az += cz(k) * val;
        al += val;
    });
    gx = ax / 10.0;
    gy = ay / 10.0;
    gz = az / 10.0;
    lap = (al - 14.0 * f[c]) / 5.0;
}

// Per-cell adjoints of the stencil values, SoA in the scratch array.
enum {
    A_FX, A_FY, A_FZ, A_FLAP, A_RX, A_RY, A_RZ,
    A_UX, A_UY, A_UZ, A_ULAP, A_VX, A_VY, A_VZ, A_VLAP, A_WX, A_WY, A_WZ, A_WLAP, A_N
};

// Collide, pass 1: local adjoints of one cell.  Writes the direct adjoints of
// the cell's own phi, rho, u, v, w (stencil contributions follow in pass 2),
// pushes the populations' adjoints to the cells they were pulled from, and
// stores the stencil adjoints.  kFirst: the first collision of a run, which
// writes the equilibria (no populations in, no viscous term); lfin and lgin
// (may be null) get zeros.  lkf (may be null): the cell's term of dJ/dk_f.
template <bool kFirst>
__global__ void __launch_bounds__(256)
collide_adjoint_local(Geom g, Phys P, const double* __restrict__ phi, const double* __restrict__ rho,
                      const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
                      const double* __restrict__ lf, const double* __restrict__ lg, const double* __restrict__ ldux,
                      const double* __restrict__ ldvy, const double* __restrict__ ldwz, double* __restrict__ lfin,
                      double* __restrict__ lgin, double* __restrict__ lphi, double* __restrict__ lrho_out,
                      double* __restrict__ lu, double* __restrict__ lv, double* __restrict__ lw,
                      double* __restrict__ scratch, double* __restrict__ lkf)
{
    int x, y, z;
    if (!cell_xyz(g, x, y, z)) return;
    const long long n = g.n;
    const long long c = cell_of(g, x, y, z);
    double f_x, f_y, f_z, f_lap, r_x, r_y, r_z, r_lap, u_x, u_y, u_z, u_lap, v_x, v_y, v_z, v_lap, w_x, w_y, w_z,
        w_lap;
    grad_lap(phi, g, x, y, z, c, f_x, f_y, f_z, f_lap);
    grad_lap(rho, g, x, y, z, c, r_x, r_y, r_z, r_lap);
    grad_lap(u, g, x, y, z, c, u_x, u_y, u_z, u_lap);
    grad_lap(v, g, x, y, z, c, v_x, v_y, v_z, v_lap);
    grad_lap(w, g, x, y, z, c, w_x, w_y, w_z, w_lap);
    (void)r_lap;
    const double fei = phi[c], lr = rho[c], uu = u[c], vv = v[c], ww = w[c];
    const double mu = (lr - P.rho_G) * P.mu_slope + P.mu_G;
    const double sum_fei = f_x * f_x + f_y * f_y + f_z * f_z;
    const double sum_rho = r_x * r_x + r_y * r_y + r_z * r_z;
    const double den = 1.0 - P.b * fei;
    const double dp0 = P.T / (den * den) - 2.0 * P.a * fei;   // d p0 / d phi

    double a_fei = 0, a_chem = 0, a_sumfei = 0, a_fx = 0, a_fy = 0, a_fz = 0, a_flap = 0;
    double a_uu = 0, a_vv = 0, a_ww = 0, a_usq = 0, a_lr = 0, a_sumrho = 0, a_rx = 0, a_ry = 0, a_rz = 0, a_mu = 0;
    double a_ux = ldux[c], a_uy = 0, a_uz = 0, a_vx = 0, a_vy = ldvy[c], a_vz = 0, a_wx = 0, a_wy = 0,
           a_wz = ldwz[c];
    double a_ulap = 0, a_vlap = 0, a_wlap = 0;
    double a_kf = 0;   // sum over q of E_q Gfei_q times the adjoint of f_eq_q (the k_f Gfei term)
    const double kf1 = 1.0 - 1.0 / P.tauf, kf2 = 1.0 / P.tauf;
    const double kg1 = 1.0 - 1.0 / P.taug, kg2 = 1.0 / P.taug;
    const Wrap wr(g, x, y, z);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int X = cx(q), Y = cy(q), Z = cz(q);
        constexpr double E = wE(q), F = wF(q), CS = csq(q);
        const long long src = pull_src<q>(g, wr, x, y, z);
        // ---- f: out = fv (1 - 1/tau_f) + feq / tau_f ----
        const double lF = lf[(long long)q * n + c];
        if (lfin)
            lfin[(long long)q * n + src] =
                kFirst ? 0.0 : slip_T<q>(g, x, [&](auto k) { return lf[decltype(k)::value * n + c]; }) * kf1;
        const double le = kFirst ? lF : lF * kf2;   // adjoint of f_eq
        if constexpr (q == 0) {
            a_fei += le;
            a_chem += F * le;
        } else {
            const double un = X * uu + Y * vv + Z * ww;
            const double fe = X * f_x + Y * f_y + Z * f_z;
            a_chem += F * le;
            a_fei += 3.0 * E * un * le;
            const double a_un = 3.0 * E * fei * le;
            a_uu += X * a_un;
            a_vv += Y * a_un;
            a_ww += Z * a_un;
            const double a_fe = E * P.k_f * 9.0 * fe * le;
            a_fx += X * a_fe;
            a_fy += Y * a_fe;
            a_fz += Z * a_fe;
            a_sumfei += -1.5 * CS * E * P.k_f * le;
            a_kf += E * (4.5 * fe * fe - 1.5 * CS * sum_fei) * le;
        }
        // ---- g: out = gv (1 - 1/tau_g) + geq / tau_g + 3 E mu lapdot / rho ----
        const double lG = lg[(long long)q * n + c];
        if (lgin)
            lgin[(long long)q * n + src] =
                kFirst ? 0.0 : slip_T<q>(g, x, [&](auto k) { return lg[decltype(k)::value * n + c]; }) * kg1;
        const double lq = kFirst ? lG : lG * kg2;   // adjoint of g_eq
        const double Cq = -2.0 / 3.0 * F * P.k_g;   // (2/3 F k_g / rho) sum_rho term coefficient
        a_sumrho += Cq / lr * lq;
        a_lr += -Cq * sum_rho / (lr * lr) * lq;
        if constexpr (q == 0) {
            a_usq += -1.5 * E * lq;
        } else {
            const double un = X * uu + Y * vv + Z * ww;
            const double re = X * r_x + Y * r_y + Z * r_z;
            const double a_un = E * (3.0 + 9.0 * un) * lq;
            a_uu += X * a_un;
            a_vv += Y * a_un;
            a_ww += Z * a_un;
            a_usq += -1.5 * E * lq;
            const double a_S = E * P.visc * lq;
            a_ux += X * X * a_S;
            a_uy += X * Y * a_S;
            a_uz += X * Z * a_S;
            a_vx += Y * X * a_S;
            a_vy += Y * Y * a_S;
            a_vz += Y * Z * a_S;
            a_wx += Z * X * a_S;
            a_wy += Z * Y * a_S;
            a_wz += Z * Z * a_S;
            const double Grho = 4.5 * re * re - 1.5 * CS * sum_rho;
            const double kq = E * P.k_g / lr;
            const double a_re = kq * 9.0 * re * lq;
            a_rx += X * a_re;
            a_ry += Y * a_re;
            a_rz += Z * a_re;
            a_sumrho += kq * (-1.5 * CS) * lq;
            a_lr += -E * P.k_g * Grho / (lr * lr) * lq;
            if constexpr (!kFirst) {
                // viscous term 3 E mu (c . lap u) / rho, on the output directly
                const double lapdot = X * u_lap + Y * v_lap + Z * w_lap;
                a_mu += 3.0 * E * lapdot / lr * lG;
                a_lr += -3.0 * E * mu * lapdot / (lr * lr) * lG;
                const double a_ld = 3.0 * E * mu / lr * lG;
                a_ulap += X * a_ld;
                a_vlap += Y * a_ld;
                a_wlap += Z * a_ld;
            }
        }
    });
    // chem = p0(phi) - k_f phi lap(phi) - k_f sum_fei / 6
    if (lkf) lkf[c] = a_chem * (-fei * f_lap - sum_fei / 6.0) + a_kf;
    a_fei += dp0 * a_chem - P.k_f * f_lap * a_chem;
    a_flap += -P.k_f * fei * a_chem;
    a_sumfei += -P.k_f / 6.0 * a_chem;
    a_fx += 2.0 * f_x * a_sumfei;
    a_fy += 2.0 * f_y * a_sumfei;
    a_fz += 2.0 * f_z * a_sumfei;
    a_rx += 2.0 * r_x * a_sumrho;
    a_ry += 2.0 * r_y * a_sumrho;
    a_rz += 2.0 * r_z * a_sumrho;
    a_uu += 2.0 * uu * a_usq;
    a_vv += 2.0 * vv * a_usq;
    a_ww += 2.0 * ww * a_usq;
    a_lr += P.mu_slope * a_mu;
    lphi[c] = a_fei;
    lrho_out[c] = a_lr;
    lu[c] = a_uu;
    lv[c] = a_vv;
    lw[c] = a_ww;
    const double vals[A_N] = {a_fx, a_fy, a_fz, a_flap, a_rx, a_ry, a_rz, a_ux, a_uy, a_uz, a_ulap,
                              a_vx, a_vy, a_vz, a_vlap, a_wx, a_wy, a_wz, a_wlap};
#pragma unroll
    for (int i = 0; i < A_N; ++i) scratch[(long long)i * n + c] = vals[i];
}

// Transpose of one field's stencils at cell t: the cells c = t - c_k read t as
// their neighbour k.  With the slip walls x does not wrap, and the wall cells
// read the mirrored neighbour: x = 0 reads x = 1 for c_x = -1, x = lx - 1
// reads x = lx - 2 for c_x = +1.
__device__ __forceinline__ double stencil_T(const Geom& g, int x, int y, int z, long long t,
                                            const double* __restrict__ agx, const double* __restrict__ agy,
                                            const double* __restrict__ agz, const double* __restrict__ alap)
{
    double s = 0.0, l = 0.0;
    static_for<1, Q>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        auto add = [&](long long c) {
            s += cx(k) * agx[c] + cy(k) * agy[c] + cz(k) * agz[c];
            if (alap) l += alap[c];
        };
        if (g.periodic_x) {
            add(nb(g, x, y, z, -cx(k), -cy(k), -cz(k)));
        } else {
            const int xc = x - cx(k);
            if (xc >= 0 && xc < g.lx) add(nb(g, xc, y, z, 0, -cy(k), -cz(k)));
            if constexpr (cx(k) == -1) {
                if (x == 1) add(nb(g, 0, y, z, 0, -cy(k), -cz(k)));
            } else if constexpr (cx(k) == 1) {
                if (x == g.lx - 2) add(nb(g, g.lx - 1, y, z, 0, -cy(k), -cz(k)));
            }
        }
    });
    double out = s / 10.0;
    if (alap) out += (l - 14.0 * alap[t]) / 5.0;
    return out;
}

// Collide, pass 2: add the stencils' transposes to the field adjoints.
__global__ void __launch_bounds__(256)
collide_adjoint_gather(Geom g, const double* __restrict__ scratch, double* __restrict__ lphi,
                       double* __restrict__ lrho, double* __restrict__ lu, double* __restrict__ lv,
                       double* __restrict__ lw)
{
    int x, y, z;
    if (!cell_xyz(g, x, y, z)) return;
    const long long n = g.n;
    const long long t = cell_of(g, x, y, z);
    auto S = [&](int i) { return scratch + (long long)i * n; };
    lphi[t] += stencil_T(g, x, y, z, t, S(A_FX), S(A_FY), S(A_FZ), S(A_FLAP));
    lrho[t] += stencil_T(g, x, y, z, t, S(A_RX), S(A_RY), S(A_RZ), nullptr);
    lu[t] += stencil_T(g, x, y, z, t, S(A_UX), S(A_UY), S(A_UZ), S(A_ULAP));
    lv[t] += stencil_T(g, x, y, z, t, S(A_VX), S(A_VY), S(A_VZ), S(A_VLAP));
    lw[t] += stencil_T(g, x, y, z, t, S(A_WX), S(A_WY), S(A_WZ), S(A_WLAP));
}

// Moments backward: phi = sum_q f*(x - c_q), rho = rho(phi) (the sine
// interpolation, CPU/Inamuro.cpp:315-327), u* = sum_q c_q g*(x - c_q), the
// pulled populations overwritten at the slip walls (slip_T).
// kAdd: add to lf, lg instead of overwriting them.
template <bool kAdd>
__global__ void __launch_bounds__(256)
moments_adjoint(Geom g, Phys P, const double* __restrict__ phi, const double* __restrict__ lphi,
                const double* __restrict__ lrho, const double* __restrict__ lu, const double* __restrict__ lv,
                const double* __restrict__ lw, double* __restrict__ lf, double* __restrict__ lg)
{
    int x, y, z;
    if (!cell_xyz(g, x, y, z)) return;
    const long long n = g.n;
    const long long c = cell_of(g, x, y, z);
    const double fei = phi[c];
    double drho = 0.0;
    if (fei > P.fei_G && fei < P.fei_L) {
        const double arg = (fei - P.fei_avg) / P.dfei * CUDART_PI;
        drho = P.half_drho * cos(arg) * CUDART_PI / P.dfei;
    }
    const double a_phi = lphi[c] + drho * lrho[c];
    const double au = lu[c], av = lv[c], aw = lw[c];
    const Wrap wr(g, x, y, z);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const long long src = pull_src<q>(g, wr, x, y, z);
        const double vf = slip_T<q>(g, x, [&](auto) { return a_phi; });
        const double vg = slip_T<q>(g, x, [&](auto k) {
            constexpr int j = decltype(k)::value;
            return cx(j) * au + cy(j) * av + cz(j) * aw;
        });
        if constexpr (kAdd) {
            lf[(long long)q * n + src] += vf;
            lg[(long long)q * n + src] += vg;
        } else {
            lf[(long long)q * n + src] = vf;
            lg[(long long)q * n + src] = vg;
        }
    });
}

// Correction backward: u = u* - (p(x+1) - p(x-1)) / (2 rho), likewise v, w.
// lu, lv, lw: adjoints of u, v, w (= those of u*, v*, w*); outputs the
// adjoints of p and rho (kAdd: added to lp, lrho).  With the slip walls the
// x neighbours are mirrored (CPU/Inamuro.cpp:794-823): a wall cell reads the
// same cell as both neighbours, so its x difference is identically zero and
// it contributes nothing, and x does not wrap.
template <bool kAdd>
__global__ void __launch_bounds__(256)
correct_adjoint(Geom g, const double* __restrict__ p, const double* __restrict__ rho,
                const double* __restrict__ lu, const double* __restrict__ lv, const double* __restrict__ lw,
                double* __restrict__ lp, double* __restrict__ lrho)
{
    int x, y, z;
    if (!cell_xyz(g, x, y, z)) return;
    const long long t = cell_of(g, x, y, z);
    const double* la[3] = {lu, lv, lw};
    const int d[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    const Mirror mr(g, x, y, z);
    double ap = 0.0, ar = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const long long cm = nb(g, x, y, z, -d[a][0], -d[a][1], -d[a][2]);   // reads t as its + neighbour
        const long long cp = nb(g, x, y, z, d[a][0], d[a][1], d[a][2]);      // reads t as its - neighbour
        if (a == 0 && !g.periodic_x) {
            // x: interior cells only (x = 1 .. lx-2), no wrap
            const double am = (x - 1 >= 1) ? -la[a][cm] / (2.0 * rho[cm]) : 0.0;
            const double bp = (x + 1 <= g.lx - 2) ? la[a][cp] / (2.0 * rho[cp]) : 0.0;
            ap += am + bp;
            const double grad = p[cell_of(g, mr.xp, y, z)] - p[cell_of(g, mr.xm, y, z)];
            ar += la[a][t] * grad / (2.0 * rho[t] * rho[t]);
            continue;
        }
        ap += -la[a][cm] / (2.0 * rho[cm]) + la[a][cp] / (2.0 * rho[cp]);
        const double grad = p[cp] - p[cm];
        ar += la[a][t] * grad / (2.0 * rho[t] * rho[t]);
    }
    if constexpr (kAdd) {
        lp[t] += ap;
        lrho[t] += ar;
    } else {
        lp[t] = ap;
        lrho[t] = ar;
    }
}

// ---- the implicit adjoint of the kinetic Poisson solve ---------------------
// The forward solve iterates h <- K h - E s / 3 to its fixed point, with
// K = M R: R the pull stream, M the per-cell relaxation
// hv -> hv - (hv - E sum(hv)) / tau_h, tau_h = 1/rho + 0.5
// (CPU/Inamuro.cpp:755-778), and p = sum_q (R h)_q.  With lam_p the adjoint
// of p (zero mean; its mean belongs to the gauge), the multiplier mu of the
// fixed-point equation solves mu = K^T mu + R^T 1 lam_p, K^T = R^T M^T:
// M^T m = (1 - 1/tau) m + (sum_k E_k m_k) / tau per cell, and R^T pulls
// from x + c_q where R pulls from x - c_q.  Iterated on y = M^T mu + lam_p:
//   y <- M^T (pull from x + c_q of y) + lam_p,   mu_q(x) = y_q(x + c_q),
// one sweep costs what a forward sweep does.  Then
//   dJ/ds   = -sum_q E_q mu_q / 3,
//   dJ/drho = -sum_q mu_q (hv_q - E_q p) / (tau^2 rho^2)   (hv = R h*).
// The constant mode (K^T 1 = 1) only shifts dJ/ds by a constant, which the
// source's mean projection and the periodic stencils' transposes remove.
//
// Slip walls: R becomes W R, W the overwrite of the incoming populations at
// x = 0 and lx-1 (not a permutation), and the pull from x + c_q becomes the
// transposed pull tpull (W^T, then the push).  K no longer conserves
// sum(h): (I - K) keeps the right null vector E (uniform p), but its left
// null vector l is not uniform, so the forward system is inconsistent and the
// sweeps drift along E by delta per sweep, which the gauge removes at each
// check.  The converged, gauged state solves the bordered system
//   (I - K) h + delta E = b,   mean(P h) = target,
// whose adjoint is (I - K)^T mu + nu P^T 1/N = P^T lam_p with E . mu = 0:
// nu = sum(lam_p) (the gauge's share, as above), and the transposed
// iteration keeps E . mu fixed (E^T K^T = E^T because K E = E) at its start
// value 0 (the start y = lam_p - mean has E . y = 0), so it converges to that
// solution without l itself.

// y_q(x) = lp(x) for every q.
__global__ void __launch_bounds__(256)
padj_init(Geom g, const double* __restrict__ lp, double* __restrict__ y)
{
    int x, yy, z;
    if (!cell_xyz(g, x, yy, z)) return;
    const long long c = cell_of(g, x, yy, z);
    const double v = lp[c];
#pragma unroll
    for (int q = 0; q < Q; ++q) y[(long long)q * g.n + c] = v;
}

// pi = sum_q y_q of a starting iterate (the reference of the first check).
__global__ void __launch_bounds__(256)
padj_pi(Geom g, const double* __restrict__ y, double* __restrict__ pi)
{
    int x, yy, z;
    if (!cell_xyz(g, x, yy, z)) return;
    const long long c = cell_of(g, x, yy, z);
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < Q; ++q) s += y[(long long)q * g.n + c];
    pi[c] = s;
}

// One transposed sweep.  kCheck: also the relative change of
// pi = sum_q y_q against the copy kept from the previous check (block
// partials of sum |pi - pi_prev| and sum |pi|), and the new copy.  The pull
// from x + c_q (tpull) uses the forward sweep's wrap table with the
// directions reversed; kOff32: 32-bit offsets (15 n < 2^31).
template <bool kCheck, bool kOff32>
__global__ void __launch_bounds__(256)
padj_sweep(Geom g, const double* __restrict__ yin, double* __restrict__ yout, const double* __restrict__ rho,
           const double* __restrict__ lp, double* __restrict__ pi_prev, double* __restrict__ part,
           long long nblocks)
{
    int x, yy, z;
    const bool active = cell_xyz(g, x, yy, z);
    double red[2] = {0.0, 0.0};
    if (active) {
        using I = typename std::conditional<kOff32, unsigned, long long>::type;
        const I n = static_cast<I>(g.n);
        const I c = static_cast<I>(cell_of(g, x, yy, z));
        const Wrap w(g, x, yy, z);
        double m[Q];
        double S = 0.0;
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            m[q] = tpull<q>(yin, n, g, w, x, yy, z);
            S += wE(q) * m[q];
        });
        const double tau = 1.0 / __ldg(rho + c) + 0.5;
        const double a = 1.0 - 1.0 / tau, b = S / tau, l = __ldg(lp + c);
        double pi = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double v = a * m[q] + b + l;
            yout[static_cast<I>(q) * n + c] = v;
            pi += v;
        }
        if constexpr (kCheck) {
            red[0] = fabs(pi - pi_prev[c]);
            red[1] = fabs(pi);
            pi_prev[c] = pi;
        }
    }
    if constexpr (kCheck) block_sum_store<2>(red, part, nblocks, block_linear());
}

// mu from the converged y; dJ/ds into ls, dJ/drho added to lrho.  h: the
// forward solve's converged (post-collision) h.
__global__ void __launch_bounds__(256)
padj_final(Geom g, const double* __restrict__ y, const double* __restrict__ h, const double* __restrict__ rho,
           double* __restrict__ ls, double* __restrict__ lrho)
{
    int x, yy, z;
    if (!cell_xyz(g, x, yy, z)) return;
    const long long n = g.n;
    const long long c = cell_of(g, x, yy, z);
    double mu[Q], hv[Q];
    double p = 0.0, smu = 0.0;
    const Wrap w(g, x, yy, z);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        mu[q] = tpull<q>(y, n, g, w, x, yy, z);
        hv[q] = h[(long long)q * n + nb(g, x, yy, z, -cx(q), -cy(q), -cz(q))];
        smu += wE(q) * mu[q];
    });
    bounce_regs(hv, g, x);
    static_for<0, Q>([&](auto qc) { p += hv[decltype(qc)::value]; });
    double t = 0.0;
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        t += mu[q] * (hv[q] - wE(q) * p);
    });
    const double r = rho[c];
    const double tau = 1.0 / r + 0.5;
    ls[c] = -smu / 3.0;
    lrho[c] += -t / (tau * tau * r * r);
}

// Source projection backward: s = (u_x - mean(u_x)) + v_y + w_z
// (CPU/Inamuro.cpp:652-668).
__global__ void __launch_bounds__(256)
prep_adjoint(Geom g, const double* __restrict__ ls, double mean_ls, double* __restrict__ ldux,
             double* __restrict__ ldvy, double* __restrict__ ldwz)
{
    int x, y, z;
    if (!cell_xyz(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    const double v = ls[c];
    ldux[c] = v - mean_ls;
    ldvy[c] = v;
    ldwz[c] = v;
}

// Block partial sums of a[0..n) on a fixed grid (deterministic order).
__global__ void __launch_bounds__(256)
sum_partials(const double* __restrict__ a, long long n, double* __restrict__ part)
{
    double v[1] = {0.0};
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) v[0] += a[i];
    block_sum_store<1>(v, part, gridDim.x, blockIdx.x);
}

__global__ void __launch_bounds__(256)
add_const(double* __restrict__ a, long long n, double alpha)
{
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) a[i] += alpha;
}

}  // namespace

namespace adj {

void collide_backward(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P, bool first,
                      const double* phi, const double* rho, const double* u, const double* v, const double* w,
                      const double* lf, const double* lg, const double* ldux, const double* ldvy,
                      const double* ldwz, double* lfin, double* lgin, double* lphi, double* lrho, double* lu,
                      double* lv, double* lw, double* scratch, double* lkf)
{
    if (first)
        collide_adjoint_local<true><<<L.grid, L.block, 0, st>>>(g, P, phi, rho, u, v, w, lf, lg, ldux, ldvy, ldwz,
                                                                lfin, lgin, lphi, lrho, lu, lv, lw, scratch, lkf);
    else
        collide_adjoint_local<false><<<L.grid, L.block, 0, st>>>(g, P, phi, rho, u, v, w, lf, lg, ldux, ldvy, ldwz,
                                                                 lfin, lgin, lphi, lrho, lu, lv, lw, scratch, lkf);
    collide_adjoint_gather<<<L.grid, L.block, 0, st>>>(g, scratch, lphi, lrho, lu, lv, lw);
}

void moments_backward_add(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P, const double* phi,
                          const double* lphi, const double* lrho, const double* lu, const double* lv,
                          const double* lw, double* lf, double* lg)
{
    moments_adjoint<true><<<L.grid, L.block, 0, st>>>(g, P, phi, lphi, lrho, lu, lv, lw, lf, lg);
}

void correct_backward_add(cudaStream_t st, const Launch& L, const Geom& g, const double* p, const double* rho,
                          const double* lu, const double* lv, const double* lw, double* lp, double* lrho)
{
    correct_adjoint<true><<<L.grid, L.block, 0, st>>>(g, p, rho, lu, lv, lw, lp, lrho);
}

void poisson_init(cudaStream_t st, const Launch& L, const Geom& g, const double* lp, double* y)
{
    padj_init<<<L.grid, L.block, 0, st>>>(g, lp, y);
}

void poisson_pi(cudaStream_t st, const Launch& L, const Geom& g, const double* y, double* pi)
{
    padj_pi<<<L.grid, L.block, 0, st>>>(g, y, pi);
}

void poisson_sweep(cudaStream_t st, const Launch& L, const Geom& g, bool check, const double* yin, double* yout,
                   const double* rho, const double* lp, double* pi_prev, double* part)
{
    const bool off32 = 15 * g.n < (1LL << 31);
    if (check) {
        if (off32) padj_sweep<true, true><<<L.grid, L.block, 0, st>>>(g, yin, yout, rho, lp, pi_prev, part, L.nblocks);
        else padj_sweep<true, false><<<L.grid, L.block, 0, st>>>(g, yin, yout, rho, lp, pi_prev, part, L.nblocks);
    } else {
        if (off32) padj_sweep<false, true><<<L.grid, L.block, 0, st>>>(g, yin, yout, rho, lp, pi_prev, part, L.nblocks);
        else padj_sweep<false, false><<<L.grid, L.block, 0, st>>>(g, yin, yout, rho, lp, pi_prev, part, L.nblocks);
    }
}

void poisson_final(cudaStream_t st, const Launch& L, const Geom& g, const double* y, const double* h,
                   const double* rho, double* ls, double* lrho)
{
    padj_final<<<L.grid, L.block, 0, st>>>(g, y, h, rho, ls, lrho);
}

void prep_backward(cudaStream_t st, const Launch& L, const Geom& g, const double* ls, double mean_ls,
                   double* ldux, double* ldvy, double* ldwz)
{
    prep_adjoint<<<L.grid, L.block, 0, st>>>(g, ls, mean_ls, ldux, ldvy, ldwz);
}

void sum_partials(cudaStream_t st, const double* a, long long n, double* part)
{
    lbm::sum_partials<<<kSumBlocks, 256, 0, st>>>(a, n, part);
}

void add_const(cudaStream_t st, double* a, long long n, double alpha)
{
    lbm::add_const<<<kSumBlocks, 256, 0, st>>>(a, n, alpha);
}

}  // namespace adj
}  // namespace lbm

using namespace lbm;

namespace {

struct Box {
    Geom g;
    Phys P;
    Launch L;
};

lbm_status make_box(const lbm_params* prm, Box& b)
{
    if (!prm || prm->lx < 2 || prm->ly < 1 || prm->lz < 1 || prm->lz > 65535) return LBM_ERR_BAD_ARG;
    b.g.lx = prm->lx;
    b.g.ly = prm->ly;
    b.g.lz = prm->lz;
    b.g.periodic_x = prm->periodic_x ? 1 : 0;
    b.g.n = static_cast<long long>(prm->lx) * prm->ly * prm->lz;
    b.P = make_phys(*prm);
    const int bx = prm->lx >= 32 ? 32 : 16;
    b.L = make_launch(prm->lx, prm->ly, prm->lz, bx, 256 / bx);
    return LBM_OK;
}

lbm_status finish(cudaError_t e)
{
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e == cudaSuccess ? LBM_OK : (e == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA);
}

}  // namespace

extern "C" {

lbm_status lbm_collide_forward(const lbm_params* prm, const double* fin, const double* gin, const double* phi,
                               const double* rho, const double* u, const double* v, const double* w, double* fout,
                               double* gout, double* dux, double* dvy, double* dwz)
{
    Box b;
    const lbm_status s = make_box(prm, b);
    if (s != LBM_OK) return s;
    if (!fin || !gin || !phi || !rho || !u || !v || !w || !fout || !gout || !dux || !dvy || !dwz) return LBM_ERR_BAD_ARG;
    double* part = nullptr;
    if (cudaMalloc(&part, 3 * b.L.nblocks * sizeof(double)) != cudaSuccess) return LBM_ERR_OOM;
    fp64::collide(0, b.L, b.g, b.P, false, 0, fin, fout, gin, gout, phi, rho, u, v, w, dux, dvy, dwz, part);
    const lbm_status r = finish(cudaSuccess);
    cudaFree(part);
    return r;
}

lbm_status lbm_collide_backward(const lbm_params* prm, const double* fin, const double* gin, const double* phi,
                                const double* rho, const double* u, const double* v, const double* w,
                                const double* lam_fout, const double* lam_gout, const double* lam_dux,
                                const double* lam_dvy, const double* lam_dwz, double* lam_fin, double* lam_gin,
                                double* lam_phi, double* lam_rho, double* lam_u, double* lam_v, double* lam_w)
{
    Box b;
    const lbm_status s = make_box(prm, b);
    if (s != LBM_OK) return s;
    if (!phi || !rho || !u || !v || !w || !lam_fout || !lam_gout || !lam_dux || !lam_dvy || !lam_dwz || !lam_fin ||
        !lam_gin || !lam_phi || !lam_rho || !lam_u || !lam_v || !lam_w)
        return LBM_ERR_BAD_ARG;
    (void)fin;   // the map is affine in the populations: their values do not enter the adjoint
    (void)gin;
    double* scratch = nullptr;
    if (cudaMalloc(&scratch, static_cast<size_t>(A_N) * b.g.n * sizeof(double)) != cudaSuccess) return LBM_ERR_OOM;
    collide_adjoint_local<false><<<b.L.grid, b.L.block>>>(b.g, b.P, phi, rho, u, v, w, lam_fout, lam_gout,
                                                          lam_dux, lam_dvy, lam_dwz, lam_fin, lam_gin, lam_phi,
                                                          lam_rho, lam_u, lam_v, lam_w, scratch, nullptr);
    collide_adjoint_gather<<<b.L.grid, b.L.block>>>(b.g, scratch, lam_phi, lam_rho, lam_u, lam_v, lam_w);
    const lbm_status r = finish(cudaSuccess);
    cudaFree(scratch);
    return r;
}

lbm_status lbm_moments_forward(const lbm_params* prm, const double* f, const double* g, double* phi, double* rho,
                               double* u, double* v, double* w)
{
    Box b;
    const lbm_status s = make_box(prm, b);
    if (s != LBM_OK) return s;
    if (!f || !g || !phi || !rho || !u || !v || !w) return LBM_ERR_BAD_ARG;
    double* part = nullptr;
    if (cudaMalloc(&part, b.L.nblocks * sizeof(double)) != cudaSuccess) return LBM_ERR_OOM;
    fp64::moments(0, b.L, b.g, b.P, f, g, phi, rho, u, v, w, part);
    const lbm_status r = finish(cudaSuccess);
    cudaFree(part);
    return r;
}

lbm_status lbm_moments_backward(const lbm_params* prm, const double* phi, const double* lam_phi,
                                const double* lam_rho, const double* lam_u, const double* lam_v, const double* lam_w,
                                double* lam_f, double* lam_g)
{
    Box b;
    const lbm_status s = make_box(prm, b);
    if (s != LBM_OK) return s;
    if (!phi || !lam_phi || !lam_rho || !lam_u || !lam_v || !lam_w || !lam_f || !lam_g) return LBM_ERR_BAD_ARG;
    moments_adjoint<false><<<b.L.grid, b.L.block>>>(b.g, b.P, phi, lam_phi, lam_rho, lam_u, lam_v, lam_w, lam_f, lam_g);
    return finish(cudaSuccess);
}

lbm_status lbm_correct_forward(const lbm_params* prm, double* u, double* v, double* w, const double* p,
                               const double* rho)
{
    Box b;
    const lbm_status s = make_box(prm, b);
    if (s != LBM_OK) return s;
    if (!u || !v || !w || !p || !rho) return LBM_ERR_BAD_ARG;
    fp64::correct(0, b.L, b.g, u, v, w, p, rho);
    return finish(cudaSuccess);
}

lbm_status lbm_correct_backward(const lbm_params* prm, const double* p, const double* rho, const double* lam_u,
                                const double* lam_v, const double* lam_w, double* lam_p, double* lam_rho)
{
    Box b;
    const lbm_status s = make_box(prm, b);
    if (s != LBM_OK) return s;
    if (!p || !rho || !lam_u || !lam_v || !lam_w || !lam_p || !lam_rho) return LBM_ERR_BAD_ARG;
    correct_adjoint<false><<<b.L.grid, b.L.block>>>(b.g, p, rho, lam_u, lam_v, lam_w, lam_p, lam_rho);
    return finish(cudaSuccess);
}

}  // extern "C"
