// mixed_cells.cuh -- per-cell building blocks of the mixed-precision box
// (FP32 populations stored as rest-state deviations, FP32 stencils, FP64
// pressure sums), shared by the single-box kernels (kernels_mixed.cu) and the
// batched kernels (batch_mixed.cu) so both evaluate every cell identically.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "collide_zm.cuh"
#include "lbm_mixed.cuh"

namespace lbm {
namespace {

template <int Q0 = 0>
__device__ __forceinline__ void pull_regs(float (&v)[Q], const float* __restrict__ src, const Geom& g,
                                          int x, int y, int z)
{
    const Wrap w(g, x, y, z);
    static_for<Q0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        v[q] = __ldg(src + (long long)q * g.n + pull_src<q>(g, w, x, y, z));
    });
}

template <bool kLap>
__device__ __forceinline__ void stencil(const float* __restrict__ f, const Geom& g, const Mirror& m,
                                        int x, int y, int z, long long c,
                                        float& gx, float& gy, float& gz, float& lap)
{
    float ax = 0.f, ay = 0.f, az = 0.f, al = 0.f;
    static_for<1, Q>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const float val = __ldg(f + stencil_nb<k>(g, m, x, y, z));
        ax = acc_signed<cx(k)>(ax, val);
        ay = acc_signed<cy(k)>(ay, val);
        az = acc_signed<cz(k)>(az, val);
        if constexpr (kLap) al += val;
    });
    gx = ax * 0.1f;
    gy = ay * 0.1f;
    gz = az * 0.1f;
    if constexpr (kLap) lap = (al - 14.f * __ldg(f + c)) * 0.2f;
}

struct MixPhys {
    float rho_G, mu_G, mu_slope, inv_tauf, inv_taug, k_f, k_g, T, a, b, visc;
    float fei_G, p0_G;          // gas rest state of f
};

// Per-cell constants of the mixed collision (CPU/Inamuro.cpp:134-250 in
// deviation form: f_rest and E_q cancel in f - (f - f_eq)/tau).
struct MixCell {
    float inv_rho, mu, sum_fei, sum_rho, usq, chem_dev, dphi, kg_rho;
};

// The constants the g collision uses.
__device__ __forceinline__ void mix_cell_g(const MixPhys& P, const CellDeriv<float>& d, MixCell& k)
{
    k.inv_rho = 1.f / d.lrho;
    k.mu = (d.lrho - P.rho_G) * P.mu_slope + P.mu_G;
    k.sum_rho = d.r_x * d.r_x + d.r_y * d.r_y + d.r_z * d.r_z;
    k.usq = d.uu * d.uu + d.vv * d.vv + d.ww * d.ww;
    k.kg_rho = P.k_g * k.inv_rho;
}

// The constants the f collision uses.
__device__ __forceinline__ void mix_cell_f(const MixPhys& P, const CellDeriv<float>& d, MixCell& k)
{
    k.sum_fei = d.f_x * d.f_x + d.f_y * d.f_y + d.f_z * d.f_z;
    const float p0 = d.fei * P.T / (1.f - P.b * d.fei) - P.a * d.fei * d.fei;
    k.chem_dev = (p0 - P.p0_G) - P.k_f * d.fei * d.f_lap - P.k_f * k.sum_fei * (1.f / 6.f);
    k.dphi = d.fei - P.fei_G;
}

// Post-collision f_q (deviation from f_rest,q); fin: the pulled, bounced f_q.
template <int q, bool kFirst>
__device__ __forceinline__ float mix_f_post(const MixPhys& P, const CellDeriv<float>& d, const MixCell& k,
                                            float fin)
{
    constexpr float E = float(wE(q)), F = float(wF(q));
    const float un = dotq<q>(d.uu, d.vv, d.ww);
    const float fe = dotq<q>(d.f_x, d.f_y, d.f_z);
    float feq;
    if constexpr (q == 0) {
        feq = k.dphi + F * k.chem_dev;
    } else {
        const float Gfei = 4.5f * fe * fe - 1.5f * float(csq(q)) * k.sum_fei;
        feq = F * k.chem_dev + 3.f * E * d.fei * un + E * P.k_f * Gfei;
    }
    if constexpr (kFirst) return feq;
    else return fin - (fin - feq) * P.inv_tauf;
}

// Post-collision g_q (deviation from E_q) with the viscous term.
template <int q, bool kFirst>
__device__ __forceinline__ float mix_g_post(const MixPhys& P, const CellDeriv<float>& d, const MixCell& k,
                                            float gin)
{
    constexpr float E = float(wE(q)), F = float(wF(q));
    const float un = dotq<q>(d.uu, d.vv, d.ww);
    float geq;
    if constexpr (q == 0) {
        geq = -1.5f * E * k.usq - (2.f / 3.f) * F * k.kg_rho * k.sum_rho;
    } else {
        const float S = cc_contract<q>(d);
        const float re = dotq<q>(d.r_x, d.r_y, d.r_z);
        const float Grho = 4.5f * re * re - 1.5f * float(csq(q)) * k.sum_rho;
        geq = E * (3.f * un - 1.5f * k.usq + 4.5f * un * un + P.visc * S) + E * k.kg_rho * Grho -
              (2.f / 3.f) * F * k.kg_rho * k.sum_rho;
    }
    if constexpr (kFirst) return geq;
    float out = gin - (gin - geq) * P.inv_taug;
    if constexpr (q != 0) out += 3.f * E * k.inv_rho * k.mu * dotq<q>(d.u_lap, d.v_lap, d.w_lap);
    return out;
}

// div = u_x + v_y + w_z into the source partial sums (sum, sum |.|, non-finite flag).
__device__ __forceinline__ float mix_div(const CellDeriv<float>& d, double (&red)[3])
{
    const float div = d.u_x + d.v_y + d.w_z;
    if (isfinite(div)) {
        red[0] += div;
        red[1] += fabs((double)div);
    } else {
        red[2] = 1.0;
    }
    return div;
}

// A cell's pressure as an unevaluated pair of floats, p = hi + lo.
struct P32 {
    float hi, lo;
};
__device__ __forceinline__ P32 p32_of(double pv)
{
    P32 r;
    r.hi = (float)pv;
    r.lo = (float)(pv - (double)r.hi);
    return r;
}

// Kinetic collision of one population, h - (h - E p) omega - (E/3) s, in an
// order that keeps FP32 rounding from biasing the solve.  The sweep is a
// contraction whose slow modes accumulate any error that repeats from sweep
// to sweep; in FP32 the plain expression has such an error, of order
// u |h| (u = 2^-24) and the same in every cell of a uniform region: E is not
// representable (E p rounds), and h - E s/3 rounds before the relaxation term
// is added.  Here the non-equilibrium part t = h - E p is formed with E and p
// each split into two floats (three FMAs: each rounding is of order u |t|,
// and t = 0 exactly at equilibrium), the collision's change -omega t - E s/3
// is formed from the small terms alone, and h gains it in one rounding, so a
// population at its fixed point stays there.  (Measured at 256^3 against the
// FP64 box, 3 steps x 1000 sweeps: p error 2.2e-5 with the plain expression.)
template <int q>
__device__ __forceinline__ float collide_h(float h, P32 p, float om, float sv)
{
    constexpr float E = float(wE(q));
    constexpr float El = float(wE(q) - double(float(wE(q))));   // E = E + El to FP64 precision
    constexpr float E3 = float(wE(q) / 3.0);
    float t = fmaf(-E, p.hi, h);
    t = fmaf(-E, p.lo, t);
    t = fmaf(-El, p.hi, t);
    return h + fmaf(-om, t, -(E3 * sv));
}

__device__ __forceinline__ void collide_h_store(const float (&hv)[Q], double pv, float om, float sv,
                                                float* __restrict__ hout, long long n, long long c)
{
    const P32 p32 = p32_of(pv);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hout[(long long)q * n + c] = collide_h<q>(hv[q], p32, om, sv);
    });
}

__device__ __forceinline__ double sum_q(const float (&hv)[Q])
{
    double acc = 0.0;
    static_for<0, Q>([&](auto qc) { acc += (double)hv[decltype(qc)::value]; });
    return acc;
}

// p = sum_q h of the plain sweeps (the check kernels sum in FP64).
#ifndef LBM_PSUM
#define LBM_PSUM 0
#endif
__device__ __forceinline__ P32 sum_q32(const float (&h)[Q])
{
#if LBM_PSUM == 0
    P32 r;
    r.lo = 0.f;
    r.hi = (((h[0] + h[1]) + (h[2] + h[3])) + ((h[4] + h[5]) + (h[6] + h[7]))) +
           (((h[8] + h[9]) + (h[10] + h[11])) + ((h[12] + h[13]) + h[14]));
    return r;
#elif LBM_PSUM == 1
    double acc = 0.0;
    static_for<0, Q>([&](auto qc) { acc += (double)h[decltype(qc)::value]; });
    return p32_of(acc);
#else
    float s = h[0], c = 0.f;
    static_for<1, Q>([&](auto qc) {
        const float x = h[decltype(qc)::value];
        const float tt = s + x;
        const float z = tt - s;
        c += (s - (tt - z)) + (x - z);
        s = tt;
    });
    P32 r;
    r.hi = s + c;
    r.lo = c - (r.hi - s);
    return r;
#endif
}

__device__ __forceinline__ void collide_h_store32(const float (&hv)[Q], P32 p32, float om, float sv,
                                                  float* __restrict__ hout, int n, int c)
{
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hout[q * n + c] = collide_h<q>(hv[q], p32, om, sv);
    });
}

// ---- per-cell bodies ------------------------------------------------------
// One cell (x, y, z) of box g; populations q-major with stride g.n.  The
// single-box kernels and the batched kernels call these, so a cell is
// evaluated the same way in both.  Reduction terms are added to red.

// phi - phi_G in FP64: the rest population f0 (FP64, it does not move) plus
// the pulled moving populations f_1..f_14 (FP32 deviations), in q order.  The
// moments and the next collision evaluate it from the same values in the same
// order, so both see the same phi.
__device__ __forceinline__ double phi_dev(double f0, const float (&fv)[Q])
{
    double acc = f0;
    static_for<1, Q>([&](auto qc) { acc += (double)fv[decltype(qc)::value]; });
    return acc;
}

// Post-collision f: the moving populations in FP32 (fout, q >= 1), the rest
// population in FP64 as what remains of phi once the stored moving
// populations are taken out.  The collision conserves phi (sum_q f_eq = phi),
// so this is f0's own BGK value; and since the stream moves the stored FP32
// values unchanged (a permutation under periodic boundaries), sum(phi) over
// the box is carried from step to step to FP64 rounding.
template <bool kFirst, class Idx>
__device__ __forceinline__ void store_f_post(const MixPhys& P, const CellDeriv<float>& d, const MixCell& k,
                                             const float (&fv)[Q], double f0_in, float* __restrict__ fout,
                                             double* __restrict__ f0, Idx n, Idx c)
{
    // before the first collision f0 holds phi - phi_G (the load), the moving
    // populations nothing
    const double dev = kFirst ? f0_in : phi_dev(f0_in, fv);
    double moved = 0.0;
    static_for<1, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        float in = 0.f;
        if constexpr (!kFirst) in = fv[q];
        const float out = mix_f_post<q, kFirst>(P, d, k, in);
        fout[q * n + c] = out;
        moved += (double)out;
    });
    f0[c] = dev - moved;
}

// Plane collide: stencils gathered from global memory (CPU/Inamuro.cpp:134-250).
template <bool kFirst>
__device__ __forceinline__ void mixc_collide(const Geom& g, const MixPhys& P, const float* __restrict__ fin,
                                             float* __restrict__ fout, double* __restrict__ f0,
                                             const float* __restrict__ gin,
                                             float* __restrict__ gout, const float* __restrict__ phi,
                                             const float* __restrict__ rho, const float* __restrict__ u,
                                             const float* __restrict__ v, const float* __restrict__ w,
                                             float* __restrict__ div_out, int x, int y, int z, double (&red)[3])
{
    const long long c = cell_of(g, x, y, z);
    const Mirror m(g, x, y, z);
    CellDeriv<float> d;
    float unused;
    stencil<true>(u, g, m, x, y, z, c, d.u_x, d.u_y, d.u_z, d.u_lap);
    stencil<true>(v, g, m, x, y, z, c, d.v_x, d.v_y, d.v_z, d.v_lap);
    stencil<true>(w, g, m, x, y, z, c, d.w_x, d.w_y, d.w_z, d.w_lap);
    stencil<false>(rho, g, m, x, y, z, c, d.r_x, d.r_y, d.r_z, unused);
    stencil<true>(phi, g, m, x, y, z, c, d.f_x, d.f_y, d.f_z, d.f_lap);
    (void)unused;
    d.lrho = __ldg(rho + c);
    d.fei = __ldg(phi + c);
    d.uu = __ldg(u + c);
    d.vv = __ldg(v + c);
    d.ww = __ldg(w + c);
    div_out[c] = mix_div(d, red);
    MixCell k;
    mix_cell_g(P, d, k);
    mix_cell_f(P, d, k);
    float fv[Q];
    if constexpr (!kFirst) {
        pull_regs<1>(fv, fin, g, x, y, z);
        bounce_regs(fv, g, x);
    }
    store_f_post<kFirst>(P, d, k, fv, f0[c], fout, f0, g.n, c);
    float gv[Q];
    if constexpr (!kFirst) {
        pull_regs(gv, gin, g, x, y, z);
        bounce_regs(gv, g, x);
    }
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        float in = 0.f;
        if constexpr (!kFirst) in = gv[q];
        gout[(long long)q * g.n + c] = mix_g_post<q, kFirst>(P, d, k, in);
    });
}

// Moments (CPU/Inamuro.cpp:294-346): phi = phi_G + f0 + sum_{q>=1} f_dev
// (FP64), rho(phi), u* = sum c g; red[0] += phi.
struct MixMoments {
    double fei_G, fei_L, rho_G, rho_L, fei_avg, dfei, half_drho;
};

__device__ __forceinline__ void mixc_moments(const Geom& g, const MixMoments& M, const float* __restrict__ f,
                                             const double* __restrict__ f0,
                                             const float* __restrict__ gp, float* __restrict__ phi,
                                             float* __restrict__ rho, float* __restrict__ u,
                                             float* __restrict__ v, float* __restrict__ w, int x, int y, int z,
                                             double (&red)[1])
{
    const long long c = cell_of(g, x, y, z);
    float fv[Q];
    pull_regs<1>(fv, f, g, x, y, z);
    bounce_regs(fv, g, x);
    const double fei = M.fei_G + phi_dev(f0[c], fv);
    double density;
    if (fei <= M.fei_G) density = M.rho_G;
    else if (fei >= M.fei_L) density = M.rho_L;
    else density = M.half_drho * (sin((fei - M.fei_avg) / M.dfei * CUDART_PI) + 1.0) + M.rho_G;
    float gv[Q];
    pull_regs(gv, gp, g, x, y, z);
    bounce_regs(gv, g, x);
    float uu = 0.f, vv = 0.f, ww = 0.f;
    static_for<1, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        uu = acc_signed<cx(q)>(uu, gv[q]);
        vv = acc_signed<cy(q)>(vv, gv[q]);
        ww = acc_signed<cz(q)>(ww, gv[q]);
    });
    phi[c] = (float)fei;
    rho[c] = (float)density;
    u[c] = uu;
    v[c] = vv;
    w[c] = ww;
    red[0] += fei;
}

// Source projection s = div - mean(div), omega_h = 1 / (1/rho + 1/2); red:
// sum s, non-finite flag, sum p (CPU/Inamuro.cpp:652-668).
__device__ __forceinline__ void mixc_prep(const Geom& g, double div_mean, const float* __restrict__ div,
                                          const float* __restrict__ rho, const double* __restrict__ p,
                                          float* __restrict__ s, float* __restrict__ omega, int x, int y, int z,
                                          double (&red)[3])
{
    const long long c = cell_of(g, x, y, z);
    const float sv = (float)((double)div[c] - div_mean);
    s[c] = sv;
    omega[c] = 1.f / (1.f / rho[c] + 0.5f);
    if (isfinite(sv)) red[0] += sv; else red[1] = 1.0;
    red[2] += p[c];
}

// Poisson start: h0 = E_q p (or the loaded h0) and its first collision.
__device__ __forceinline__ void mixc_init(const Geom& g, bool h_loaded, const float* __restrict__ hload,
                                          float* __restrict__ hout, const double* __restrict__ p,
                                          const float* __restrict__ omega, const float* __restrict__ s, int x,
                                          int y, int z)
{
    const long long c = cell_of(g, x, y, z);
    const double pv = p[c];
    float hv[Q];
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hv[q] = h_loaded ? hload[(long long)q * g.n + c] : (float)(pv * wE(q));
    });
    collide_h_store(hv, pv, omega[c], s[c], hout, g.n, c);
}

// Plain kinetic sweep, 32-bit offsets (15 n < 2^31): pull + slip + p = sum h
// (pairwise FP32) + collision.
__device__ __forceinline__ void mixc_sweep32(const Geom& g, const float* __restrict__ hin, float* __restrict__ hout,
                                             const float* __restrict__ omega, const float* __restrict__ s, int x,
                                             int y, int z)
{
    const int n = (int)g.n;
    const int c = (z * g.ly + y) * g.lx + x;
    float hv[Q];
    pull_regs32(hv, hin, n, g, x, y, z);
    bounce_regs(hv, g, x);
    collide_h_store32(hv, sum_q32(hv), __ldg(omega + c), __ldg(s + c), hout, n, c);
}

// Check sweep A: pull + slip + p = sum h (FP64); h_k stored uncollided, red[0] += p.
__device__ __forceinline__ void mixc_check_a(const Geom& g, const float* __restrict__ hin, float* __restrict__ hout,
                                             double* __restrict__ p_chk, int x, int y, int z, double (&red)[1])
{
    const long long c = cell_of(g, x, y, z);
    float hv[Q];
    pull_regs(hv, hin, g, x, y, z);
    bounce_regs(hv, g, x);
    const double pv = sum_q(hv);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hout[(long long)q * g.n + c] = hv[q];
    });
    p_chk[c] = pv;
    red[0] += pv;
}

// Check B: gauge (p -= shift, h -= E shift; CPU/Inamuro.cpp:699-705), the
// relative-change terms (:726-753) and, in dual mode, the R_p terms
// (GPU/InamuroCUDA.cu:2033-2055); then the collision of the next sweep.
template <bool kDual>
__device__ __forceinline__ void mixc_check_b(const Geom& g, const float* __restrict__ hin, float* __restrict__ hout,
                                             float* __restrict__ hc, const double* __restrict__ p_chk,
                                             double* __restrict__ p_prev, double* __restrict__ p,
                                             const float* __restrict__ omega, const float* __restrict__ s,
                                             double shift, double tgt, int x, int y, int z, double (&red)[5])
{
    const long long c = cell_of(g, x, y, z);
    float hv[Q];
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hv[q] = (float)((double)__ldg(hin + (long long)q * g.n + c) - wE(q) * shift);
    });
    const double pv = p_chk[c] - shift;
    if constexpr (kDual) {
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            hc[(long long)q * g.n + c] = hv[q];
        });
        const double hsum = sum_q(hv);
        red[2] += fabs(pv - hsum);
        red[3] += fabs(pv - tgt);
        red[4] += fabs(hsum - tgt);
    }
    red[0] += fabs(pv - p_prev[c]);
    red[1] += fabs(pv);
    p_prev[c] = pv;
    p[c] = pv;
    collide_h_store(hv, pv, __ldg(omega + c), __ldg(s + c), hout, g.n, c);
}

// Velocity correction u -= grad p / (2 rho), x neighbours mirrored
// (CPU/Inamuro.cpp:794-823).
__device__ __forceinline__ void mixc_correct(const Geom& g, float* __restrict__ u, float* __restrict__ v,
                                             float* __restrict__ w, const double* __restrict__ p,
                                             const float* __restrict__ rho, int x, int y, int z)
{
    const Mirror m(g, x, y, z);
    const long long c = cell_of(g, x, y, z);
    const double inv_2rho = 1.0 / (2.0 * (double)rho[c]);
    u[c] = (float)((double)u[c] - (p[cell_of(g, m.xp, y, z)] - p[cell_of(g, m.xm, y, z)]) * inv_2rho);
    v[c] = (float)((double)v[c] - (p[cell_of(g, x, m.yp, z)] - p[cell_of(g, x, m.ym, z)]) * inv_2rho);
    w[c] = (float)((double)w[c] - (p[cell_of(g, x, y, m.zp)] - p[cell_of(g, x, y, m.zm)]) * inv_2rho);
}

// Two kinetic sweeps of the z run [z0, z1) of the TX x TY column at (x0, y0)
// (temporal blocking; the single box's sweep2_kernel and the batched
// b_sweep2 run this body).  Threads: one per cell of the tile plus its
// one-cell halo, (TX+2)(TY+2) rounded up to whole warps.  Each thread owns one
// region cell for the whole march and keeps the global pulls of the NEXT
// plane in flight (registers) while the CTA works through the shared-memory
// phase of the current one; one barrier per plane.  Region cells use wrapped
// coordinates, so the periodic stream and the x slip overwrite are those of
// two single sweeps; tile cells outside the box (partial tiles) store
// nothing.  Cell arithmetic: mixc_sweep32's (collide_h, sum_q32).  The ring
// is the z-direction-grouped one of lbm_device.cuh (ring_plane, 45 population
// planes).  kRefine: the refinement form's correction sweeps instead,
// e' = K e + r with r a per-population source (src = r, 15 n floats), the
// arithmetic of refine_sweep_kernel.
__host__ __device__ constexpr int sweep2_threads(int tx, int ty) { return ((tx + 2) * (ty + 2) + 31) / 32 * 32; }
__host__ __device__ constexpr int sweep2_smem(int tx, int ty)
{
    return ring_planes() * (tx + 2) * (ty + 2) * static_cast<int>(sizeof(float));
}

// Correction-sweep update of the refinement form: K e + r in FP32.
__device__ __forceinline__ float refine_sum(const float (&ev)[Q])
{
    float pe = 0.f;
    static_for<0, Q>([&](auto qc) { pe += ev[decltype(qc)::value]; });
    return pe;
}
template <int q>
__device__ __forceinline__ float refine_cell(float ev, float pe, float om, float r)
{
    return fmaf(-om, ev - float(wE(q)) * pe, ev) + r;
}

template <int TX, int TY, bool kRefine = false>
__device__ __forceinline__ void sweep2_run(const Geom& g, int x0, int y0, int z0, int z1,
                                           const float* __restrict__ hin, float* __restrict__ hout,
                                           const float* __restrict__ omega, const float* __restrict__ s,
                                           float* __restrict__ ring)
{
    constexpr int RX = TX + 2, RC = RX * (TY + 2);
    const int t = threadIdx.x;
    const int n = (int)g.n;
    // this thread's halo-region cell (wrapped coordinates)
    const bool owner = t < RC;
    const int xw = (x0 - 1 + t % RX + g.lx) % g.lx;
    const int yw = (y0 - 1 + t / RX + g.ly) % g.ly;

    float a[Q];
    float a_om = 0.f, a_s = 0.f;
    float ar[kRefine ? Q : 1];           // kRefine: the source r of the cell's plane
    auto prefetch = [&](int zz) {        // issue sweep k's pulls for plane zz
        if (!owner) return;
        const int zw = zz < 0 ? zz + g.lz : (zz >= g.lz ? zz - g.lz : zz);
        pull_regs32(a, hin, n, g, xw, yw, zw);
        const int c = (zw * g.ly + yw) * g.lx + xw;
        a_om = __ldg(omega + c);
        if constexpr (kRefine) {
            static_for<0, Q>([&](auto qc) { ar[decltype(qc)::value] = __ldg(s + decltype(qc)::value * n + c); });
        } else {
            a_s = __ldg(s + c);
        }
    };
    auto finish = [&](int zz) {          // complete sweep k on plane zz into the ring
        if (!owner) return;
        bounce_regs(a, g, xw);
        if constexpr (kRefine) {
            const float pe = refine_sum(a);
            static_for<0, Q>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                ring[ring_plane<q>(zz) * RC + t] = refine_cell<q>(a[q], pe, a_om, ar[q]);
            });
        } else {
            const P32 p32 = sum_q32(a);
            static_for<0, Q>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                ring[ring_plane<q>(zz) * RC + t] = collide_h<q>(a[q], p32, a_om, a_s);
            });
        }
    };

    prefetch(z0 - 1);
    finish(z0 - 1);
    prefetch(z0);
    finish(z0);
    prefetch(z0 + 1);
    const int tx = t % TX, ty = t / TX;
    const int x = x0 + tx, y = y0 + ty;
    const int rc = (ty + 1) * RX + (tx + 1);
    const bool inner = t < TX * TY && x < g.lx && y < g.ly;
    for (int z = z0; z < z1; ++z) {
        finish(z + 1);
        if (z + 1 < z1) prefetch(z + 2);
        __syncthreads();
        if (inner) {
            // sweep k+1 at (x, y, z): pull q from plane z - cz(q) of the ring
            float hv[Q];
            static_for<0, Q>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                hv[q] = ring[ring_plane<q>(z - cz(q)) * RC + rc - cy(q) * RX - cx(q)];
            });
            bounce_regs(hv, g, x);
            const int c = (z * g.ly + y) * g.lx + x;
            if constexpr (kRefine) {
                const float pe = refine_sum(hv);
                const float om = __ldg(omega + c);
                static_for<0, Q>([&](auto qc) {
                    constexpr int q = decltype(qc)::value;
                    hout[q * n + c] = refine_cell<q>(hv[q], pe, om, __ldg(s + q * n + c));
                });
            } else {
                collide_h_store32(hv, sum_q32(hv), __ldg(omega + c), __ldg(s + c), hout, n, c);
            }
        }
    }
}

MixPhys mix_phys(const Phys& P)
{
    MixPhys M;
    M.rho_G = (float)P.rho_G;
    M.mu_G = (float)P.mu_G;
    M.mu_slope = (float)P.mu_slope;
    M.inv_tauf = (float)(1.0 / P.tauf);
    M.inv_taug = (float)(1.0 / P.taug);
    M.k_f = (float)P.k_f;
    M.k_g = (float)P.k_g;
    M.T = (float)P.T;
    M.a = (float)P.a;
    M.b = (float)P.b;
    M.visc = (float)P.visc;
    M.fei_G = (float)P.fei_G;
    const double fg = P.fei_G;
    M.p0_G = (float)(fg * P.T / (1.0 - P.b * fg) - P.a * fg * fg);
    return M;
}

}  // namespace
}  // namespace lbm
