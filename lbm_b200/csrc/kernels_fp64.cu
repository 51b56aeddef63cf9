// kernels_fp64.cu -- plain FP64 kernels of the Inamuro D3Q15 step (the
// drop-in precision).
//
// Compiled with -fmad=false: every expression keeps the reference's operand
// order and rounding (no FMA contraction), so per-cell arithmetic is that of
// the reference CPU build; only sin() (CUDA vs libm) and the order of global
// sums differ.
//
// Storage between kernels is the POST-COLLISION population (stream-collide
// form): each kernel pulls x - c_q from the previous kernel's output, applies
// the x slip overwrite in registers, uses the populations and writes its own
// collision result at the cell itself.  Pull reads and aligned writes are
// both coalesced along x; no population is read twice in one kernel.
//
// Kernel <-> reference map
//   collide        gradientKernel x5 + laplacianKernel x4 + collisionKernel +
//                  streamKernel x2 + slipBounceBackKernel x2 of the NEXT pull
//                  (GPU/InamuroCUDA.cu:203-451, 462-493, 1399-1425);
//                  CPU/Inamuro.cpp:134-250
//   moments        macroKernel (.cu:136-192); CPU/Inamuro.cpp:294-346
//   prep           sourceStatsBlockKernel + projectSourceMeanKernel +
//                  pressureSumBlockKernel (.cu:627-714); CPU/Inamuro.cpp:652-668
//   poisson_init   updateHHKernel + first collisionPressureKernel (.cu:503-537,
//                  1377-1396); CPU/Inamuro.cpp:755-778, 825-840
//   sweep          streamKernel + slipBounceBackKernel + computePressureKernel
//                  of sweep k and collisionPressureKernel of sweep k+1
//   sweep_check_a  sweep k's stream + bounce + getp at a check, plus sum(p)
//   sweep_check_b  applyPressureGaugeKernel + pressureErrorBlockKernel + the
//                  R_p terms of fixedPointResidualBlockKernel + collision of
//                  sweep k+1 (.cu:716-730, 1062-1171, 1977-2159)
//   sweep_check_c  the shadow map F = BS[C(h,p)] compared with h (R_h terms)
//                  fused with sweep k+1's stream/bounce/sum and k+2's collision
//   correct        correctVelocityKernel (.cu:1330-1371); CPU/Inamuro.cpp:794-823
#include <cuda_runtime.h>

#include <cstdlib>
#include <math_constants.h>

#include "collide_zm.cuh"
#include "exact_div.cuh"
#include "finalize.cuh"
#include "lbm_solver.cuh"

namespace lbm {
namespace {

// Tile of a check kernel: planes [blockIdx.z * zrun, +zrun) of one 2-D tile,
// so the CTA's block reduction and its loads of the device-side scalars are
// amortised over zrun planes.
__device__ __forceinline__ bool tile_zrun(const Geom& g, int zrun, int& x, int& y, int& z0, int& z1)
{
    x = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    z0 = blockIdx.z * zrun;
    z1 = min(z0 + zrun, g.lz);
    return x < g.lx && y < g.ly;
}

__device__ __forceinline__ bool tile_coords(const Geom& g, int& x, int& y, int& z)
{
    x = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    z = blockIdx.z;
    return x < g.lx && y < g.ly;
}

template <class T>
__device__ __forceinline__ void pull_regs(T (&v)[Q], const T* __restrict__ src, const Geom& g,
                                          int x, int y, int z)
{
    const Wrap w(g, x, y, z);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        v[q] = __ldg(src + (long long)q * g.n + pull_src<q>(g, w, x, y, z));
    });
}

// firstord + (optionally) secondord of one field at one cell:
// CPU/Inamuro.hpp:213-314.  Accumulation order k = 1..14 as in the reference.
template <bool kLap>
__device__ __forceinline__ void stencil(const double* __restrict__ f, const Geom& g, const Mirror& m,
                                        int x, int y, int z, long long c,
                                        double& gx, double& gy, double& gz, double& lap)
{
    double ax = 0.0, ay = 0.0, az = 0.0, al = 0.0;
    static_for<1, Q>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const double val = __ldg(f + stencil_nb<k>(g, m, x, y, z));
        ax = acc_signed<cx(k)>(ax, val);
        ay = acc_signed<cy(k)>(ay, val);
        az = acc_signed<cz(k)>(az, val);
        if constexpr (kLap) al = al + val;
    });
    gx = ax / 10.0;
    gy = ay / 10.0;
    gz = az / 10.0;
    if constexpr (kLap) lap = (al - 14.0 * __ldg(f + c)) / 5.0;
}

// Per-cell constants of the FP64 collision (CPU/Inamuro.cpp:134-250, the
// reference's operand order throughout).
struct Fp64Cell {
    double mu, sum_fei, sum_rho, usq, chem;
};

__device__ __forceinline__ void fp64_cell(const Phys& P, const CellDeriv<double>& d, Fp64Cell& k)
{
    k.mu = (d.lrho - P.rho_G) * P.mu_slope + P.mu_G;
    k.sum_fei = d.f_x * d.f_x + d.f_y * d.f_y + d.f_z * d.f_z;
    k.sum_rho = d.r_x * d.r_x + d.r_y * d.r_y + d.r_z * d.r_z;
    k.usq = d.uu * d.uu + d.vv * d.vv + d.ww * d.ww;
    const double p0 = d.fei * P.T / (1.0 - P.b * d.fei) - P.a * d.fei * d.fei;
    k.chem = p0 - P.k_f * d.fei * d.f_lap - P.k_f * k.sum_fei / 6.0;
}

// BGK relaxation x - (x - x_eq)/tau; kPow2: tau is a power of two, so the
// division is the exact multiplication by 1/tau.  The choice is a kernel-wide
// branch around the whole loop, so no division is evaluated when it is not used.
template <bool kPow2>
__device__ __forceinline__ double bgk(double x, double xeq, double tau, double inv_tau)
{
    const double d = x - xeq;
    return x - (kPow2 ? d * inv_tau : d / tau);
}

// Post-collision f_q; fin: the pulled, bounced f_q.
template <int q, bool kFirst, bool kPow2>
__device__ __forceinline__ double fp64_f_post(const Phys& P, const CellDeriv<double>& d, const Fp64Cell& k,
                                              double fin)
{
    constexpr double E = wE(q), F = wF(q);
    const double un = dotq<q>(d.uu, d.vv, d.ww);
    const double fe = dotq<q>(d.f_x, d.f_y, d.f_z);
    double Gfei = 4.5 * (fe * fe);
    if constexpr (csq(q) == 1) Gfei = Gfei - 1.5 * k.sum_fei;
    if constexpr (csq(q) == 3) Gfei = Gfei - 1.5 * k.sum_fei * 3.0;
    double fequ;
    if constexpr (q == 0) {
        fequ = d.fei + F * k.chem;
    } else {
        fequ = F * k.chem + 3.0 * E * d.fei * un + E * P.k_f * Gfei;
    }
    if constexpr (kFirst) return fequ;
    else return bgk<kPow2>(fin, fequ, P.tauf, P.inv_tauf);
}

// Post-collision g_q with the viscous term.
template <int q, bool kFirst, bool kPow2>
__device__ __forceinline__ double fp64_g_post(const Phys& P, const CellDeriv<double>& d, const Fp64Cell& k,
                                              double gin)
{
    constexpr double E = wE(q), F = wF(q);
    const double un = dotq<q>(d.uu, d.vv, d.ww);
    double gequ;
    if constexpr (q == 0) {
        // un = 0, grad terms vanish: E*(1 - 1.5 usq) - (2/3 F k_g / rho) sum_rho
        const double velPart = 1.0 - 1.5 * k.usq;
        gequ = E * velPart - 2.0 / 3.0 * F * P.k_g / d.lrho * k.sum_rho;
    } else {
        // c_a c_b (d_b u_a) summed in the reference's 9-term order
        const double S = cc_contract<q>(d);
        const double velPart = 1.0 + 3.0 * un - 1.5 * k.usq + 4.5 * un * un + P.visc * S;
        const double re = dotq<q>(d.r_x, d.r_y, d.r_z);
        double Grho = 4.5 * (re * re);
        if constexpr (csq(q) == 1) Grho = Grho - 1.5 * k.sum_rho;
        if constexpr (csq(q) == 3) Grho = Grho - 1.5 * k.sum_rho * 3.0;
        gequ = E * velPart + E * P.k_g / d.lrho * Grho - 2.0 / 3.0 * F * P.k_g / d.lrho * k.sum_rho;
    }
    if constexpr (kFirst) return gequ;
    double out = bgk<kPow2>(gin, gequ, P.taug, P.inv_taug);
    if constexpr (q != 0) {
        const double lapdot = dotq<q>(d.u_lap, d.v_lap, d.w_lap);
        out = out + 3.0 * E / d.lrho * k.mu * lapdot;
    }
    return out;
}

// div = u_x + v_y + w_z into the source partial sums (sum, sum |.|, non-finite flag).
__device__ __forceinline__ void fp64_div(const CellDeriv<double>& d, double (&red)[3])
{
    const double div = d.u_x + d.v_y + d.w_z;
    if (isfinite(div)) {
        red[0] += div;
        red[1] += fabs(div);
    } else {
        red[2] = 1.0;
    }
}

// Collision of f and g at cell c from their pulled, bounced populations
// (unused when kFirst); I: the index type of c and of the q-major stride n.
template <bool kFirst, bool kPowF, bool kPowG, class I>
__device__ __forceinline__ void fp64_collide_store(const Phys& P, const CellDeriv<double>& d, const Fp64Cell& k,
                                                   const double (&fv)[Q], const double (&gv)[Q],
                                                   double* __restrict__ fout, double* __restrict__ gout,
                                                   I n, I c)
{
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        double in = 0.0;
        if constexpr (!kFirst) in = fv[q];
        fout[I(q) * n + c] = fp64_f_post<q, kFirst, kPowF>(P, d, k, in);
    });
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        double in = 0.0;
        if constexpr (!kFirst) in = gv[q];
        gout[I(q) * n + c] = fp64_g_post<q, kFirst, kPowG>(P, d, k, in);
    });
}

template <bool kFirst, class I>
__device__ __forceinline__ void fp64_collide_dispatch(const Phys& P, const CellDeriv<double>& d,
                                                      const Fp64Cell& k, const double (&fv)[Q],
                                                      const double (&gv)[Q], double* __restrict__ fout,
                                                      double* __restrict__ gout, I n, I c)
{
    if (P.tauf_pow2 && P.taug_pow2)
        fp64_collide_store<kFirst, true, true>(P, d, k, fv, gv, fout, gout, n, c);
    else if (P.tauf_pow2)
        fp64_collide_store<kFirst, true, false>(P, d, k, fv, gv, fout, gout, n, c);
    else if (P.taug_pow2)
        fp64_collide_store<kFirst, false, true>(P, d, k, fv, gv, fout, gout, n, c);
    else
        fp64_collide_store<kFirst, false, false>(P, d, k, fv, gv, fout, gout, n, c);
}

// Fused collide (+ the pull of the previous collision's output), one CTA per
// 2-D tile of one plane, stencil neighbours gathered from global memory.
template <bool kFirst>
__global__ void __launch_bounds__(256)
collide_kernel(Geom g, Phys P, const double* __restrict__ fin, double* __restrict__ fout,
               const double* __restrict__ gin, double* __restrict__ gout,
               const double* __restrict__ phi, const double* __restrict__ rho,
               const double* __restrict__ u, const double* __restrict__ v,
               const double* __restrict__ w, double* __restrict__ dux,
               double* __restrict__ dvy, double* __restrict__ dwz, double* __restrict__ part,
               long long nblocks)
{
    int x, y, z;
    const bool active = tile_coords(g, x, y, z);
    double red[3] = {0.0, 0.0, 0.0};
    if (active) {
        const long long c = cell_of(g, x, y, z);
        const Mirror m(g, x, y, z);
        CellDeriv<double> d;
        double unused;
        stencil<true>(u, g, m, x, y, z, c, d.u_x, d.u_y, d.u_z, d.u_lap);
        stencil<true>(v, g, m, x, y, z, c, d.v_x, d.v_y, d.v_z, d.v_lap);
        stencil<true>(w, g, m, x, y, z, c, d.w_x, d.w_y, d.w_z, d.w_lap);
        stencil<false>(rho, g, m, x, y, z, c, d.r_x, d.r_y, d.r_z, unused);
        stencil<true>(phi, g, m, x, y, z, c, d.f_x, d.f_y, d.f_z, d.f_lap);
        (void)unused;
        dux[c] = d.u_x;
        dvy[c] = d.v_y;
        dwz[c] = d.w_z;
        fp64_div(d, red);
        d.lrho = __ldg(rho + c);
        d.fei = __ldg(phi + c);
        d.uu = __ldg(u + c);
        d.vv = __ldg(v + c);
        d.ww = __ldg(w + c);
        Fp64Cell k;
        fp64_cell(P, d, k);
        double fv[Q], gv[Q];
        if constexpr (!kFirst) {
            pull_regs(fv, fin, g, x, y, z);
            bounce_regs(fv, g, x);
            pull_regs(gv, gin, g, x, y, z);
            bounce_regs(gv, g, x);
        }
        fp64_collide_dispatch<kFirst>(P, d, k, fv, gv, fout, gout, g.n, c);
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

// z-marching collide (collide_zm.cuh): one CTA per 32 x 8 column and run of
// zlen planes, the macro fields staged through the shared-memory ring, the
// populations pulled into registers with 32-bit offsets.  Same per-cell
// arithmetic as collide_kernel (bitwise); the source partial sums are
// accumulated per thread over its planes.
template <bool kFirst, int kMinBlocks>
__global__ void __launch_bounds__(ZM_THREADS, kMinBlocks)
collide_zm_kernel(Geom g, Phys P, int zlen, const double* __restrict__ fin, double* __restrict__ fout,
                  const double* __restrict__ gin, double* __restrict__ gout,
                  const double* __restrict__ phi, const double* __restrict__ rho,
                  const double* __restrict__ u, const double* __restrict__ v,
                  const double* __restrict__ w, double* __restrict__ dux,
                  double* __restrict__ dvy, double* __restrict__ dwz, double* __restrict__ part,
                  long long nblocks)
{
    extern __shared__ __align__(16) unsigned char zm_raw[];
    const int tid = threadIdx.x;
    const int tx = tid % ZM_TX, ty = tid / ZM_TX;
    const int x0 = blockIdx.x * ZM_TX, y0 = blockIdx.y * ZM_TY;
    const int x = x0 + tx, y = y0 + ty;
    const int z0 = blockIdx.z * zlen;
    const int z1 = min(z0 + zlen, g.lz);
    const int n = static_cast<int>(g.n);
    const int t = (ty + 1) * ZM_HX + tx + 1;
    const MacroRing<double> ring(reinterpret_cast<double*>(zm_raw), g, x0, y0, phi, rho, u, v, w, tid);
    ring.issue(z0 - 1);
    ring.issue(z0);
    ring.issue(z0 + 1);
    double red[3] = {0.0, 0.0, 0.0};
    for (int z = z0; z < z1; ++z) {
        // Both population sets are requested before the plane barrier, so
        // their latency overlaps the wait and the stencil arithmetic.
        double fv[Q], gv[Q];
        if constexpr (!kFirst) {
            pull_regs32(fv, fin, n, g, x, y, z);
            pull_regs32(gv, gin, n, g, x, y, z);
        }
        cp_async_wait_all();
        __syncthreads();
        if (z + 2 <= z1) ring.issue(z + 2);
        const unsigned c = static_cast<unsigned>((z * g.ly + y) * g.lx + x);
        CellDeriv<double> d;
        zm_derivs_g(ring, z, t, d);
        zm_derivs_f(ring, z, t, d);
        dux[c] = d.u_x;
        dvy[c] = d.v_y;
        dwz[c] = d.w_z;
        fp64_div(d, red);
        Fp64Cell k;
        fp64_cell(P, d, k);
        if constexpr (!kFirst) {
            bounce_regs(fv, g, x);
            bounce_regs(gv, g, x);
        }
        fp64_collide_dispatch<kFirst>(P, d, k, fv, gv, fout, gout, static_cast<unsigned>(n), c);
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
moments_kernel(Geom g, Phys P, const double* __restrict__ f, const double* __restrict__ gp,
               double* __restrict__ phi, double* __restrict__ rho, double* __restrict__ u,
               double* __restrict__ v, double* __restrict__ w, double* __restrict__ part,
               long long nblocks)
{
    int x, y, z;
    const bool active = tile_coords(g, x, y, z);
    double red[1] = {0.0};
    if (active) {
        const long long c = cell_of(g, x, y, z);
        double fv[Q];
        pull_regs(fv, f, g, x, y, z);
        bounce_regs(fv, g, x);
        double fei = 0.0;
        static_for<0, Q>([&](auto qc) { fei = fei + fv[decltype(qc)::value]; });
        double density;
        if (fei <= P.fei_G) {
            density = P.rho_G;
        } else if (fei >= P.fei_L) {
            density = P.rho_L;
        } else {
            const double arg = (fei - P.fei_avg) / P.dfei * CUDART_PI;
            density = P.half_drho * (sin(arg) + 1.0) + P.rho_G;
        }
        double gv[Q];
        pull_regs(gv, gp, g, x, y, z);
        bounce_regs(gv, g, x);
        double uu = 0.0, vv = 0.0, ww = 0.0;
        static_for<1, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            uu = acc_signed<cx(q)>(uu, gv[q]);
            vv = acc_signed<cy(q)>(vv, gv[q]);
            ww = acc_signed<cz(q)>(ww, gv[q]);
        });
        phi[c] = fei;
        rho[c] = density;
        u[c] = uu;
        v[c] = vv;
        w[c] = ww;
        red[0] = fei;
    }
    block_sum_store<1>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
prep_kernel(Geom g, const DevState* __restrict__ ds, const double* __restrict__ dux,
            const double* __restrict__ dvy, const double* __restrict__ dwz,
            const double* __restrict__ p, double* __restrict__ s, double* __restrict__ part,
            long long nblocks)
{
    int x, y, z;
    const bool active = tile_coords(g, x, y, z);
    double red[3] = {0.0, 0.0, 0.0};
    if (active) {
        const long long c = cell_of(g, x, y, z);
        const double m = ds->div_mean;
        // u_x -= mean (CPU/Inamuro.cpp:665-668), then u_x + v_y + w_z.
        const double sv = (dux[c] - m) + dvy[c] + dwz[c];
        s[c] = sv;
        if (isfinite(sv)) red[0] = sv; else red[1] = 1.0;
        red[2] = p[c];
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
poisson_init_kernel(Geom g, int h_loaded, const double* __restrict__ hload,
                    double* __restrict__ hout, const double* __restrict__ p,
                    const double* __restrict__ rho, const double* __restrict__ s, int source_aware,
                    double sa_scale)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    const double pv = p[c];
    const double tauh = 1.0 / rho[c] + 0.5;
    const double inv_tauh = 1.0 / tauh;
    const double sv = s[c];
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr double E = wE(q);
        // h = p * E_q after update_hh (CPU/Inamuro.cpp:835), or the loaded h;
        // source-aware: E_q p - scale tau_h (E_q / 3) s (GPU/InamuroCUDA.cu:903-929).
        const double h0 = source_aware ? E * pv - sa_scale * tauh * ((E / 3.0) * sv)
                                       : (h_loaded ? hload[(long long)q * g.n + c] : pv * E);
        const double hequ = E * pv;
        hout[(long long)q * g.n + c] = h0 - div_rn(h0 - hequ, tauh, inv_tauh) - (E / 3.0) * sv;
    });
}

// I: index type (long long in general, int where 15 n < 2^31).
template <class I>
__device__ __forceinline__ void collide_h_store(const double (&hv)[Q], double pv, double tauh,
                                                double sv, double* __restrict__ hout, I n, I c)
{
    const double inv_tauh = 1.0 / tauh;   // the 15 quotients by tau_h come from it (exact_div.cuh)
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr double E = wE(q);
        const double hequ = E * pv;
        hout[(I)q * n + c] = hv[q] - div_rn(hv[q] - hequ, tauh, inv_tauh) - (E / 3.0) * sv;
    });
}


__device__ __forceinline__ double sum_q(const double (&hv)[Q])
{
    double acc = 0.0;
    static_for<0, Q>([&](auto qc) { acc = acc + hv[decltype(qc)::value]; });
    return acc;
}

// kOff32: 32-bit offsets (the launcher picks it when 15 n < 2^31).
template <bool kOff32>
__global__ void __launch_bounds__(256)
sweep_kernel(Geom g, const double* __restrict__ hin, double* __restrict__ hout,
             const double* __restrict__ rho, const double* __restrict__ s)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    double hv[Q];
    if constexpr (kOff32) {
        const int n = (int)g.n;
        const int c = (z * g.ly + y) * g.lx + x;
        pull_regs32(hv, hin, n, g, x, y, z);
        bounce_regs(hv, g, x);
        const double pv = sum_q(hv);
        const double tauh = 1.0 / __ldg(rho + c) + 0.5;
        collide_h_store(hv, pv, tauh, __ldg(s + c), hout, n, c);
    } else {
        const long long c = cell_of(g, x, y, z);
        pull_regs(hv, hin, g, x, y, z);
        bounce_regs(hv, g, x);
        const double pv = sum_q(hv);
        const double tauh = 1.0 / __ldg(rho + c) + 0.5;
        collide_h_store(hv, pv, tauh, __ldg(s + c), hout, g.n, c);
    }
}

// Two sweeps in one pass (temporal blocking; same scheme as the mixed box).
// A CTA owns a TX x TY xy tile and a run of `zlen` planes; marching in z it
// computes sweep k on the tile plus a one-cell halo (wrapped coordinates,
// pulled from global memory) into the z-grouped plane ring of lbm_device.cuh
// (45 population planes), then sweep k+1 on the tile from that ring.  Every
// cell's arithmetic is collide_h_store's expression, so (without FMA
// contraction in this file) the result is bitwise that of two sweep_kernel
// launches.  Each thread owns one halo-region cell for the whole march and
// keeps the next plane's global pulls in flight while the CTA works through
// the shared-memory phase; one barrier per plane.  lx % TX == 0,
// ly % TY == 0 and 15 n < 2^31 are required (checked by the launcher).
constexpr int F2_TX = 16, F2_TY = 8;
constexpr int F2_RX = F2_TX + 2, F2_RY = F2_TY + 2, F2_RC = F2_RX * F2_RY;
constexpr int F2_THREADS = (F2_RC + 31) / 32 * 32;   // 192: one thread per region cell
constexpr int F2_SMEM = ring_planes() * F2_RC * (int)sizeof(double);   // 64,800 B
constexpr int F2_CTAS = 2;

__global__ void __launch_bounds__(F2_THREADS, F2_CTAS)
sweep2_kernel(Geom g, int zlen, const double* __restrict__ hin, double* __restrict__ hout,
              const double* __restrict__ rho, const double* __restrict__ s)
{
    extern __shared__ double ring2[];   // [ring_planes()][F2_RC]
    const int t = threadIdx.x;
    const int n = (int)g.n;
    const int x0 = blockIdx.x * F2_TX, y0 = blockIdx.y * F2_TY;
    const int z0 = blockIdx.z * zlen;
    const int z1 = min(z0 + zlen, g.lz);
    const bool owner = t < F2_RC;
    const int xw = (x0 - 1 + t % F2_RX + g.lx) % g.lx;
    const int yw = (y0 - 1 + t / F2_RX + g.ly) % g.ly;

    double a[Q];
    double a_rho = 1.0, a_s = 0.0;
    auto prefetch = [&](int zz) {
        if (!owner) return;
        const int zw = zz < 0 ? zz + g.lz : (zz >= g.lz ? zz - g.lz : zz);
        pull_regs32(a, hin, n, g, xw, yw, zw);
        const int c = (zw * g.ly + yw) * g.lx + xw;
        a_rho = __ldg(rho + c);
        a_s = __ldg(s + c);
    };
    auto finish = [&](int zz) {
        if (!owner) return;
        bounce_regs(a, g, xw);
        const double pv = sum_q(a);
        const double tauh = 1.0 / a_rho + 0.5;
        // collide_h_store's expression, each population into its ring plane
        const double inv_tauh = 1.0 / tauh;
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr double E = wE(q);
            const double hequ = E * pv;
            ring2[ring_plane<q>(zz) * F2_RC + t] = a[q] - div_rn(a[q] - hequ, tauh, inv_tauh) - (E / 3.0) * a_s;
        });
    };

    prefetch(z0 - 1);
    finish(z0 - 1);
    prefetch(z0);
    finish(z0);
    prefetch(z0 + 1);
    const int tx = t % F2_TX, ty = t / F2_TX;
    const int x = x0 + tx, y = y0 + ty;
    const int rc = (ty + 1) * F2_RX + (tx + 1);
    for (int z = z0; z < z1; ++z) {
        finish(z + 1);
        if (z + 1 < z1) prefetch(z + 2);
        __syncthreads();
        if (t < F2_TX * F2_TY) {
            double hv[Q];
            static_for<0, Q>([&](auto qc) {
                constexpr int q = decltype(qc)::value;
                hv[q] = ring2[ring_plane<q>(z - cz(q)) * F2_RC + rc - cy(q) * F2_RX - cx(q)];
            });
            bounce_regs(hv, g, x);
            const int c = (z * g.ly + y) * g.lx + x;
            const double pv = sum_q(hv);
            const double tauh = 1.0 / __ldg(rho + c) + 0.5;
            collide_h_store(hv, pv, tauh, __ldg(s + c), hout, n, c);
        }
    }
}

__global__ void __launch_bounds__(256)
sweep_check_a_kernel(Geom g, int zrun, const double* __restrict__ hin, double* __restrict__ hout,
                     double* __restrict__ p_chk, double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[1] = {0.0};
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        double hv[Q];
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
    block_sum_store<1>(red, part, nblocks, block_linear());
}

template <bool kDual>
__global__ void __launch_bounds__(256)
sweep_check_b_kernel(Geom g, int zrun, const double* __restrict__ hin, double* __restrict__ hout,
                     double* __restrict__ hc,
                     const double* __restrict__ p_chk, double* __restrict__ p_prev,
                     double* __restrict__ p, const double* __restrict__ rho,
                     const double* __restrict__ s, const DevState* __restrict__ ds,
                     double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double shift = ds->sigma;
    const double tgt = ds->target;
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        double hv[Q];
        // Gauge (CPU/Inamuro.cpp:699-705): p -= shift, h_q -= E_q shift.
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            hv[q] = __ldg(hin + (long long)q * g.n + c) - wE(q) * shift;
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
        // Relative change (CPU/Inamuro.cpp:726-753).
        red[0] += fabs(pv - p_prev[c]);
        red[1] += fabs(pv);
        p_prev[c] = pv;
        p[c] = pv;
        const double tauh = 1.0 / __ldg(rho + c) + 0.5;
        collide_h_store(hv, pv, tauh, __ldg(s + c), hout, g.n, c);
    }
    block_sum_store<5>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
sweep_check_c_kernel(Geom g, int zrun, const double* __restrict__ hin, double* __restrict__ hout,
                     const double* __restrict__ hc, const double* __restrict__ rho,
                     const double* __restrict__ s, const DevState* __restrict__ ds,
                     double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[3] = {0.0, 0.0, 0.0};
    const double tgt = ds->target;
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        double hv[Q];
        pull_regs(hv, hin, g, x, y, z);
        bounce_regs(hv, g, x);
        // hv is F(h, p) = BS[C(h, p)] for the gauged h of the check
        // (GPU/InamuroCUDA.cu:1997-2009); compare with that h.
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const double hval = hc[(long long)q * g.n + c];
            const double ge = wE(q) * tgt;
            red[0] += fabs(hval - hv[q]);
            red[1] += fabs(hval - ge);
            red[2] += fabs(hv[q] - ge);
        });
        const double pv = sum_q(hv);
        const double tauh = 1.0 / __ldg(rho + c) + 0.5;
        collide_h_store(hv, pv, tauh, __ldg(s + c), hout, g.n, c);
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

// ---- scalar Poisson forms -------------------------------------------------
// The reference's scalar form (scalarPressureJacobiKernel,
// GPU/InamuroCUDA.cu:864-901): one Jacobi sweep of the 14-neighbour stencil,
// p' = (sum_{q=1..14} p(x - c_q) - 5 scale rho s) / 14, x neighbours mirrored
// at the slip walls (its pressure_bounce_direction, .cu:846-862), in the
// reference's operand order.  Its fixed point solves lap p = scale rho s
// with lap = (sum_nb - 14 p) / 5.
__device__ __forceinline__ double scalar_nsum(const double* __restrict__ p, const Geom& g, const Mirror& m, int x,
                                              int y, int z)
{
    double nsum = 0.0;
    static_for<1, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        nsum = nsum + __ldg(p + cell_of(g, pick<-cx(q)>(m.xm, x, m.xp), pick<-cy(q)>(m.ym, y, m.yp),
                                        pick<-cz(q)>(m.zm, z, m.zp)));
    });
    return nsum;
}

__global__ void __launch_bounds__(256)
scalar_jacobi_kernel(Geom g, const double* __restrict__ pin, double* __restrict__ pout,
                     const double* __restrict__ rho, const double* __restrict__ s, double scale)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const Mirror m(g, x, y, z);
    const long long c = cell_of(g, x, y, z);
    const double nsum = scalar_nsum(pin, g, m, x, y, z);
    const double rhs = scale * __ldg(rho + c) * __ldg(s + c);
    pout[c] = (nsum - 5.0 * rhs) / 14.0;
}

// Red-black SOR on the same equation, in place: cells with (x + y + z) % 2 ==
// color move to p + omega (p_J - p), p_J the Jacobi value above.  The 14
// neighbours of a cell all have the other colour (axis and body-diagonal
// offsets are odd; even periodic extents keep it so across the wrap), so a
// half-sweep reads only values it does not write.  For the same reason the
// Jacobi sweep maps the checkerboard chi = (-1)^(x+y+z) to -chi: at the even
// sweep counts of its checks it never takes up the right-hand side's chi
// component, and the constant one is the gauge's.  Both are removed from the
// right-hand side here (ds->rhs_mean, ds->rhs_chk), so SOR converges to the
// Jacobi sweeps' gauged limit.
__global__ void __launch_bounds__(256)
rb_sor_kernel(Geom g, double* __restrict__ p, const double* __restrict__ rho, const double* __restrict__ s,
              double scale, double omega, int color, const DevState* __restrict__ ds)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z) || ((x + y + z) & 1) != color) return;
    const Mirror m(g, x, y, z);
    const long long c = cell_of(g, x, y, z);
    double nsum = 0.0;
    static_for<1, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        nsum = nsum + p[cell_of(g, pick<-cx(q)>(m.xm, x, m.xp), pick<-cy(q)>(m.ym, y, m.yp),
                                pick<-cz(q)>(m.zm, z, m.zp))];
    });
    const double rhs = scale * __ldg(rho + c) * __ldg(s + c) - ds->rhs_mean - (color ? -ds->rhs_chk : ds->rhs_chk);
    const double pj = (nsum - 5.0 * rhs) / 14.0;
    const double pv = p[c];
    p[c] = pv + omega * (pj - pv);
}

// ---- variable-coefficient red-black form -------------------------------
// div((1/rho) grad p) = s: the continuum limit of the kinetic scheme (its
// diffusivity c_s^2 (tau_h - 1/2) = 1/(3 rho), its source -s/3 per sweep),
// discretised on the D3Q15 neighbours (6 sum_q E_q (p(x + c_q) - p(x)) is the
// isotropic laplacian, sum_q E_q c_q c_q = I/3):
//   (A p)(x) = 6 sum_{q>=1} E_q k_q(x) (p(x + c_q) - p(x)),
//   k_q(x) = (1/rho(x) + 1/rho(x + c_q)) / 2   (arithmetic face mean),
// x neighbours mirrored at the slip walls as in the stencils.  A is symmetric
// under the weights W (1/2 on the wall planes), so the right-hand side's
// W-mean is removed (ds->rhs_mean).  Not a reference form: a scalar
// discretisation whose fixed point differs from the kinetic scheme's at the
// interface (the error is measured, not claimed).

// sum_q a_q p(x + c_q) and sum_q a_q, a_q = 6 E_q k_q.
__device__ __forceinline__ void varcoef_terms(const double* __restrict__ p, const double* __restrict__ rho,
                                              const Geom& g, const Mirror& m, int x, int y, int z, double inv_rho,
                                              double& num, double& den)
{
    num = 0.0;
    den = 0.0;
    static_for<1, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const long long nb = cell_of(g, pick<cx(q)>(m.xm, x, m.xp), pick<cy(q)>(m.ym, y, m.yp),
                                     pick<cz(q)>(m.zm, z, m.zp));
        const double a = 6.0 * wE(q) * 0.5 * (inv_rho + 1.0 / __ldg(rho + nb));
        num += a * p[nb];
        den += a;
    });
}

// One colour of a red-black SOR sweep of A p = s - mean_W(s), in place.
__global__ void __launch_bounds__(256)
rb_varcoef_kernel(Geom g, double* __restrict__ p, const double* __restrict__ rho, const double* __restrict__ s,
                  double omega, int color, const DevState* __restrict__ ds)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z) || ((x + y + z) & 1) != color) return;
    const Mirror m(g, x, y, z);
    const long long c = cell_of(g, x, y, z);
    double num, den;
    varcoef_terms(p, rho, g, m, x, y, z, 1.0 / __ldg(rho + c), num, den);
    const double rhs = __ldg(s + c) - ds->rhs_mean;
    const double pv = p[c];
    p[c] = pv + omega * ((num - rhs) / den - pv);
}

// Operator residual terms at a check (after the gauge: A ignores constants):
// sum W |A p - rhs|, sum W |rhs|, sum W |A p| -- the "h" terms of the
// fixed-point test (its "p" terms stay zero), so the check's dual exit reads
// ||A p - rhs|| / max(||rhs||, ||A p||) < tolerance.
__global__ void __launch_bounds__(256)
varcoef_residual_kernel(Geom g, int zrun, const double* __restrict__ p, const double* __restrict__ rho,
                        const double* __restrict__ s, const DevState* __restrict__ ds, double* __restrict__ part,
                        long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[3] = {0.0, 0.0, 0.0};
    const double w = (!g.periodic_x && (x == 0 || x == g.lx - 1)) ? 0.5 : 1.0;
    for (int z = z0; active && z < z1; ++z) {
        const Mirror m(g, x, y, z);
        const long long c = cell_of(g, x, y, z);
        double num, den;
        varcoef_terms(p, rho, g, m, x, y, z, 1.0 / __ldg(rho + c), num, den);
        const double ap = num - den * p[c];
        const double rhs = __ldg(s + c) - ds->rhs_mean;
        red[0] += w * fabs(ap - rhs);
        red[1] += w * fabs(rhs);
        red[2] += w * fabs(ap);
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

// Block partial sums of w f, w chi f and w, f = scale rho s: the constant and
// checkerboard components the red-black form removes, projected with the
// weights w under which the mirrored stencil is symmetric (1/2 on the two
// slip-wall planes, whose cells see their inner neighbours twice; 1 elsewhere).
// (rho == nullptr: f = s, the variable-coefficient form's right-hand side.)
__global__ void __launch_bounds__(256)
scalar_rhs_sum_kernel(Geom g, int zrun, const double* __restrict__ rho, const double* __restrict__ s,
                      double scale, double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[3] = {0.0, 0.0, 0.0};
    const double w = (!g.periodic_x && (x == 0 || x == g.lx - 1)) ? 0.5 : 1.0;
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        const double f = w * (rho ? scale * __ldg(rho + c) * __ldg(s + c) : __ldg(s + c));
        red[0] += f;
        red[1] += ((x + y + z) & 1) ? -f : f;
        red[2] += w;
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

// Block partial sums of p (the gauge mean of a check).
__global__ void __launch_bounds__(256)
p_sum_kernel(Geom g, int zrun, const double* __restrict__ p, double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[1] = {0.0};
    for (int z = z0; active && z < z1; ++z) red[0] += p[cell_of(g, x, y, z)];
    block_sum_store<1>(red, part, nblocks, block_linear());
}

// Check of the scalar forms: gauge p -= shift (CPU/Inamuro.cpp:699-705; the
// h shift is moot, h = E p after the solve), relative change against the
// previous check (:726-753), result into p.  Same partial layout as
// sweep_check_b_kernel with the dual terms zero.
__global__ void __launch_bounds__(256)
scalar_check_kernel(Geom g, int zrun, const double* __restrict__ pin, double* __restrict__ p,
                    double* __restrict__ p_prev, const DevState* __restrict__ ds, double* __restrict__ part,
                    long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double shift = ds->sigma;
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        const double pv = pin[c] - shift;
        red[0] += fabs(pv - p_prev[c]);
        red[1] += fabs(pv);
        p_prev[c] = pv;
        p[c] = pv;
    }
    block_sum_store<5>(red, part, nblocks, block_linear());
}

// ---- the reference's one-pass Poisson form -------------------------------
// State: the pre-collision h (after stream and bounce) and p = sum_q h, as the
// reference's Poisson loop keeps them (GPU/InamuroCUDA.cu:2199-2330).

// h0 of a one-pass solve: the loaded h (first step after a load) or E_q p
// (updateHHKernel, .cu:1377-1396); with source_aware, the reference's
// sourceAwareHHInitKernel (.cu:903-929): E_q p - scale tau_h (E_q / 3) s.
__global__ void __launch_bounds__(256)
onepass_init_kernel(Geom g, int h_loaded, const double* __restrict__ hload, double* __restrict__ hh,
                    const double* __restrict__ p, const double* __restrict__ rho, const double* __restrict__ s,
                    int source_aware, double sa_scale)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    const double pv = p[c];
    const double tauh = 1.0 / rho[c] + 0.5;
    const double sv = s[c];
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr double E = wE(q);
        double h;
        if (source_aware) h = E * pv - sa_scale * tauh * ((E / 3.0) * sv);
        else h = h_loaded ? hload[(long long)q * g.n + c] : pv * E;
        hh[(long long)q * g.n + c] = h;
    });
}

// One one-pass sweep (collisionStreamBoundaryPressureKernel, .cu:780-844):
// each population collides at its source cell x - c_q with that cell's p,
// rho and s (relax scales the relaxation term), streams, the x walls
// overwrite the incoming ones, then h = h_old + omega (h - h_old) against the
// cell's own previous h, and p = sum_q h.
__global__ void __launch_bounds__(256)
onepass_sweep_kernel(Geom g, const double* __restrict__ hin, double* __restrict__ hout,
                     const double* __restrict__ pin, double* __restrict__ pout, const double* __restrict__ rho,
                     const double* __restrict__ s, double relax, double omega)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const Wrap w(g, x, y, z);
    double h[Q];
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr double E = wE(q);
        const long long src = pull_src<q>(g, w, x, y, z);
        const double tauh = 1.0 / __ldg(rho + src) + 0.5;
        const double hequ = E * __ldg(pin + src);
        const double h_old = __ldg(hin + (long long)q * g.n + src);
        h[q] = h_old - relax * (h_old - hequ) / tauh - (E / 3.0) * __ldg(s + src);
    });
    bounce_regs(h, g, x);
    const long long c = cell_of(g, x, y, z);
    double psum = 0.0;
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const double h_old = hin[(long long)q * g.n + c];
        const double hv = h_old + omega * (h[q] - h_old);
        hout[(long long)q * g.n + c] = hv;
        psum = psum + hv;
    });
    pout[c] = psum;
}

// Anderson-m1 on the one-pass map (.cu:931-1013, 2230-2275).  Residual r =
// image - old.  First sweep of a solve: keep r and the image.  Later sweeps:
// partial sums of prev_r (r - prev_r) and (r - prev_r)^2 (the host forms
// alpha), then image <- (1 - alpha) prev_image + alpha image, history <-
// this sweep's r and image, p = sum_q of the result.
__global__ void __launch_bounds__(256)
anderson_store_kernel(long long count, const double* __restrict__ hold, const double* __restrict__ himg,
                      double* __restrict__ prev_r, double* __restrict__ prev_img)
{
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < count; i += (long long)gridDim.x * 256) {
        prev_r[i] = himg[i] - hold[i];
        prev_img[i] = himg[i];
    }
}

__global__ void __launch_bounds__(256)
anderson_dot_kernel(long long count, const double* __restrict__ hold, const double* __restrict__ himg,
                    const double* __restrict__ prev_r, double* __restrict__ part)
{
    double red[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < count; i += (long long)gridDim.x * 256) {
        const double r = himg[i] - hold[i];
        const double d = r - prev_r[i];
        red[0] += prev_r[i] * d;
        red[1] += d * d;
    }
    block_sum_store<2>(red, part, gridDim.x, blockIdx.x);
}

__global__ void __launch_bounds__(256)
anderson_apply_kernel(Geom g, const double* __restrict__ hold, double* __restrict__ himg,
                      double* __restrict__ prev_r, double* __restrict__ prev_img, double* __restrict__ pimg,
                      double alpha)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    double psum = 0.0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const long long i = (long long)q * g.n + c;
        const double cur = himg[i];
        const double acc = (1.0 - alpha) * prev_img[i] + alpha * cur;
        prev_r[i] = cur - hold[i];
        prev_img[i] = cur;
        himg[i] = acc;
        psum += acc;
    }
    pimg[c] = psum;
}

// Check of the one-pass form: gauge p -= shift, h_q -= E_q shift
// (applyPressureGaugeKernel, .cu:716-730), relative change (:1015-1103), the
// results into the parity-0 buffers.  FIN_CHECK layout, dual terms zero.
__global__ void __launch_bounds__(256)
onepass_check_kernel(Geom g, int zrun, const double* __restrict__ hin, double* __restrict__ hout,
                     const double* __restrict__ pin, double* __restrict__ p, double* __restrict__ p_prev,
                     const DevState* __restrict__ ds, double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double shift = ds->sigma;
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            hout[(long long)q * g.n + c] = hin[(long long)q * g.n + c] - wE(q) * shift;
        });
        const double pv = pin[c] - shift;
        red[0] += fabs(pv - p_prev[c]);
        red[1] += fabs(pv);
        p_prev[c] = pv;
        p[c] = pv;
    }
    block_sum_store<5>(red, part, nblocks, block_linear());
}

// Two-grid correction (.cu:1198-1255, 1284-1328): per 4 x 4 x 4 block (partial
// at the far edges) the sum of the check's change p - p_prev (p gauged), one
// thread per block in a fixed order; after an unconverged check
// p += strength * block_sum / block_cells, p_prev = p, h_q += E_q times that.
constexpr int kTwoGridBlock = 4;

__global__ void __launch_bounds__(256)
twogrid_sums_kernel(Geom g, const double* __restrict__ p, const double* __restrict__ p_prev,
                    const DevState* __restrict__ ds, double* __restrict__ bsum, int bxn, int byn, int bzn)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bxn * byn * bzn) return;
    const int bx = b % bxn, by = (b / bxn) % byn, bz = b / (bxn * byn);
    const double shift = ds->sigma;
    double acc = 0.0;
    for (int z = bz * kTwoGridBlock; z < min(bz * kTwoGridBlock + kTwoGridBlock, g.lz); ++z)
        for (int y = by * kTwoGridBlock; y < min(by * kTwoGridBlock + kTwoGridBlock, g.ly); ++y)
            for (int x = bx * kTwoGridBlock; x < min(bx * kTwoGridBlock + kTwoGridBlock, g.lx); ++x) {
                const long long c = cell_of(g, x, y, z);
                acc += (p[c] - shift) - p_prev[c];
            }
    bsum[b] = acc;
}

// Skipped after a converged check or a zero change (read from the device state,
// so the correction sits in a captured segment without a host decision).
__global__ void __launch_bounds__(256)
block_abs_sum_kernel(const double* __restrict__ bsum, int nb, double* __restrict__ part)
{
    double red[1] = {0.0};
    for (int i = blockIdx.x * 256 + threadIdx.x; i < nb; i += gridDim.x * 256) red[0] += fabs(bsum[i]);
    block_sum_store<1>(red, part, gridDim.x, blockIdx.x);
}

__global__ void __launch_bounds__(256)
twogrid_correct_kernel(Geom g, double* __restrict__ hh, double* __restrict__ p, double* __restrict__ p_prev,
                       const double* __restrict__ bsum, int bxn, int byn, double strength,
                       const DevState* __restrict__ ds)
{
    int x, y, z;
    if (ds->converged || !(ds->l1_delta > 0.0) || ds->error) return;
    if (!tile_coords(g, x, y, z)) return;
    const int bx = x / kTwoGridBlock, by = y / kTwoGridBlock, bz = z / kTwoGridBlock;
    const int x0 = bx * kTwoGridBlock, y0 = by * kTwoGridBlock, z0 = bz * kTwoGridBlock;
    const int cells = max(1, (min(x0 + kTwoGridBlock, g.lx) - x0) * (min(y0 + kTwoGridBlock, g.ly) - y0) *
                                 (min(z0 + kTwoGridBlock, g.lz) - z0));
    const double corr = strength * bsum[(bz * byn + by) * bxn + bx] / static_cast<double>(cells);
    const long long c = cell_of(g, x, y, z);
    const double pc = p[c] + corr;
    p[c] = pc;
    p_prev[c] = pc;
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hh[(long long)q * g.n + c] += wE(q) * corr;
    });
}

__global__ void __launch_bounds__(256)
correct_kernel(Geom g, double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
               const double* __restrict__ p, const double* __restrict__ rho)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const Mirror m(g, x, y, z);
    const long long c = cell_of(g, x, y, z);
    const double inv_2rho = 1.0 / (2.0 * rho[c]);
    u[c] -= (p[cell_of(g, m.xp, y, z)] - p[cell_of(g, m.xm, y, z)]) * inv_2rho;
    v[c] -= (p[cell_of(g, x, m.yp, z)] - p[cell_of(g, x, m.ym, z)]) * inv_2rho;
    w[c] -= (p[cell_of(g, x, y, m.zp)] - p[cell_of(g, x, y, m.zm)]) * inv_2rho;
}

__global__ void __launch_bounds__(1024)
finalize_kernel(int kind, DevState* __restrict__ ds, const double* __restrict__ part,
                long long nblocks, const double* __restrict__ part2, long long nblocks2)
{
    finalize_body(kind, ds, part, nblocks, nblocks, part2, nblocks2, nblocks2);
}

}  // namespace

namespace fp64 {

static int g_zm_minb = 2;

int collide_zm_prepare(const Geom& g)
{
    if (!zm_fits(g)) return 0;
    constexpr int smem = zm_ring_bytes<double>();
    const void* kerns[] = {(const void*)collide_zm_kernel<true, 1>, (const void*)collide_zm_kernel<false, 1>,
                           (const void*)collide_zm_kernel<true, 2>, (const void*)collide_zm_kernel<false, 2>};
    for (const void* k : kerns)
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return 0;
    const char* env = std::getenv("LBM_COLLIDE_MINB");
    g_zm_minb = (env && std::atoi(env) == 1) ? 1 : 2;
    return 1;
}

long long collide(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P, bool first, int zlen,
                  const double* fin, double* fout, const double* gin, double* gout,
                  const double* phi, const double* rho, const double* u, const double* v,
                  const double* w, double* dux, double* dvy, double* dwz, double* part)
{
    if (zlen > 0) {
        const dim3 grid(g.lx / ZM_TX, g.ly / ZM_TY, (g.lz + zlen - 1) / zlen);
        const long long nb = static_cast<long long>(grid.x) * grid.y * grid.z;
        constexpr int smem = zm_ring_bytes<double>();
        auto kern = g_zm_minb == 1 ? (first ? collide_zm_kernel<true, 1> : collide_zm_kernel<false, 1>)
                                   : (first ? collide_zm_kernel<true, 2> : collide_zm_kernel<false, 2>);
        kern<<<grid, ZM_THREADS, smem, st>>>(g, P, zlen, fin, fout, gin, gout, phi, rho, u, v, w, dux, dvy, dwz,
                                             part, nb);
        return nb;
    }
    if (first)
        collide_kernel<true><<<L.grid, L.block, 0, st>>>(g, P, fin, fout, gin, gout, phi, rho, u, v,
                                                         w, dux, dvy, dwz, part, L.nblocks);
    else
        collide_kernel<false><<<L.grid, L.block, 0, st>>>(g, P, fin, fout, gin, gout, phi, rho, u, v,
                                                          w, dux, dvy, dwz, part, L.nblocks);
    return L.nblocks;
}

void moments(cudaStream_t st, const Launch& L, const Geom& g, const Phys& P, const double* f,
             const double* gpop, double* phi, double* rho, double* u, double* v, double* w,
             double* part_mass)
{
    moments_kernel<<<L.grid, L.block, 0, st>>>(g, P, f, gpop, phi, rho, u, v, w, part_mass,
                                               L.nblocks);
}

void prep(cudaStream_t st, const Launch& L, const Geom& g, const DevState* ds, const double* dux,
          const double* dvy, const double* dwz, const double* p, double* s, double* part)
{
    prep_kernel<<<L.grid, L.block, 0, st>>>(g, ds, dux, dvy, dwz, p, s, part, L.nblocks);
}

void poisson_init(cudaStream_t st, const Launch& L, const Geom& g, bool h_loaded,
                  const double* hload, double* hout, const double* p, const double* rho,
                  const double* s, bool source_aware, double sa_scale)
{
    poisson_init_kernel<<<L.grid, L.block, 0, st>>>(g, h_loaded ? 1 : 0, hload, hout, p, rho, s,
                                                    source_aware ? 1 : 0, sa_scale);
}

void sweep(cudaStream_t st, const Launch& L, const Geom& g, const double* hin, double* hout,
           const double* rho, const double* s)
{
    if (15 * g.n < 0x7fffffffLL)
        sweep_kernel<true><<<L.grid, L.block, 0, st>>>(g, hin, hout, rho, s);
    else
        sweep_kernel<false><<<L.grid, L.block, 0, st>>>(g, hin, hout, rho, s);
}

int sweep2_prepare(const Geom& g)
{
    if (g.lx % F2_TX != 0 || g.ly % F2_TY != 0 || g.lz < 3 || 15 * g.n >= 0x7fffffffLL) return 0;
    if (cudaFuncSetAttribute(sweep2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, F2_SMEM) != cudaSuccess)
        return 0;
    return 1;
}

void sweep2(cudaStream_t st, const Geom& g, int zlen, const double* hin, double* hout,
            const double* rho, const double* s)
{
    const dim3 grid(g.lx / F2_TX, g.ly / F2_TY, (g.lz + zlen - 1) / zlen);
    sweep2_kernel<<<grid, F2_THREADS, F2_SMEM, st>>>(g, zlen, hin, hout, rho, s);
}

void sweep_check_a(cudaStream_t st, const Launch& L, const Geom& g, const double* hin,
                   double* hout, double* p_chk, double* part)
{
    sweep_check_a_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, hin, hout, p_chk, part, L.cnblocks);
}

void sweep_check_b(cudaStream_t st, const Launch& L, const Geom& g, bool dual, const double* hin, double* hout,
                   double* hc, const double* p_chk, double* p_prev, double* p, const double* rho,
                   const double* s, const DevState* ds, double* part)
{
    if (dual)
        sweep_check_b_kernel<true><<<L.cgrid, L.block, 0, st>>>(g, L.zrun, hin, hout, hc, p_chk, p_prev, p, rho,
                                                                s, ds, part, L.cnblocks);
    else
        sweep_check_b_kernel<false><<<L.cgrid, L.block, 0, st>>>(g, L.zrun, hin, hout, hc, p_chk, p_prev, p, rho,
                                                                 s, ds, part, L.cnblocks);
}

void sweep_check_c(cudaStream_t st, const Launch& L, const Geom& g, const double* hin,
                   double* hout, const double* hc, const double* rho, const double* s,
                   const DevState* ds, double* part)
{
    sweep_check_c_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, hin, hout, hc, rho, s, ds, part,
                                                      L.cnblocks);
}

void scalar_jacobi(cudaStream_t st, const Launch& L, const Geom& g, const double* pin, double* pout,
                   const double* rho, const double* s, double scale)
{
    scalar_jacobi_kernel<<<L.grid, L.block, 0, st>>>(g, pin, pout, rho, s, scale);
}

void rb_sor(cudaStream_t st, const Launch& L, const Geom& g, double* p, const double* rho, const double* s,
            double scale, double omega, const DevState* ds)
{
    rb_sor_kernel<<<L.grid, L.block, 0, st>>>(g, p, rho, s, scale, omega, 0, ds);
    rb_sor_kernel<<<L.grid, L.block, 0, st>>>(g, p, rho, s, scale, omega, 1, ds);
}

void scalar_rhs_sum(cudaStream_t st, const Launch& L, const Geom& g, const double* rho, const double* s,
                    double scale, double* part)
{
    scalar_rhs_sum_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, rho, s, scale, part, L.cnblocks);
}

void rb_varcoef(cudaStream_t st, const Launch& L, const Geom& g, double* p, const double* rho, const double* s,
                double omega, const DevState* ds)
{
    rb_varcoef_kernel<<<L.grid, L.block, 0, st>>>(g, p, rho, s, omega, 0, ds);
    rb_varcoef_kernel<<<L.grid, L.block, 0, st>>>(g, p, rho, s, omega, 1, ds);
}

void varcoef_residual(cudaStream_t st, const Launch& L, const Geom& g, const double* p, const double* rho,
                      const double* s, const DevState* ds, double* part)
{
    varcoef_residual_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, p, rho, s, ds, part, L.cnblocks);
}

void p_sum(cudaStream_t st, const Launch& L, const Geom& g, const double* p, double* part)
{
    p_sum_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, p, part, L.cnblocks);
}

void scalar_check(cudaStream_t st, const Launch& L, const Geom& g, const double* pin, double* p, double* p_prev,
                  const DevState* ds, double* part)
{
    scalar_check_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, pin, p, p_prev, ds, part, L.cnblocks);
}

void onepass_init(cudaStream_t st, const Launch& L, const Geom& g, bool h_loaded, const double* hload, double* hh,
                  const double* p, const double* rho, const double* s, bool source_aware, double sa_scale)
{
    onepass_init_kernel<<<L.grid, L.block, 0, st>>>(g, h_loaded ? 1 : 0, hload, hh, p, rho, s, source_aware ? 1 : 0,
                                                    sa_scale);
}

void onepass_sweep(cudaStream_t st, const Launch& L, const Geom& g, const double* hin, double* hout, const double* pin,
                   double* pout, const double* rho, const double* s, double relax, double omega)
{
    onepass_sweep_kernel<<<L.grid, L.block, 0, st>>>(g, hin, hout, pin, pout, rho, s, relax, omega);
}

void anderson_store(cudaStream_t st, const Geom& g, const double* hold, const double* himg, double* prev_r,
                    double* prev_img)
{
    anderson_store_kernel<<<kAndersonBlocks, 256, 0, st>>>(15 * g.n, hold, himg, prev_r, prev_img);
}

void anderson_dot(cudaStream_t st, const Geom& g, const double* hold, const double* himg, const double* prev_r,
                  double* part)
{
    anderson_dot_kernel<<<kAndersonBlocks, 256, 0, st>>>(15 * g.n, hold, himg, prev_r, part);
}

void anderson_apply(cudaStream_t st, const Launch& L, const Geom& g, const double* hold, double* himg, double* prev_r,
                    double* prev_img, double* pimg, double alpha)
{
    anderson_apply_kernel<<<L.grid, L.block, 0, st>>>(g, hold, himg, prev_r, prev_img, pimg, alpha);
}

void onepass_check(cudaStream_t st, const Launch& L, const Geom& g, const double* hin, double* hout, const double* pin,
                   double* p, double* p_prev, const DevState* ds, double* part)
{
    onepass_check_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, hin, hout, pin, p, p_prev, ds, part, L.cnblocks);
}

int twogrid_blocks(const Geom& g, int* bxn, int* byn, int* bzn)
{
    *bxn = (g.lx + kTwoGridBlock - 1) / kTwoGridBlock;
    *byn = (g.ly + kTwoGridBlock - 1) / kTwoGridBlock;
    *bzn = (g.lz + kTwoGridBlock - 1) / kTwoGridBlock;
    return *bxn * *byn * *bzn;
}

void twogrid_sums(cudaStream_t st, const Geom& g, const double* p, const double* p_prev, const DevState* ds,
                  double* bsum)
{
    int bxn, byn, bzn;
    const int nb = twogrid_blocks(g, &bxn, &byn, &bzn);
    twogrid_sums_kernel<<<(nb + 255) / 256, 256, 0, st>>>(g, p, p_prev, ds, bsum, bxn, byn, bzn);
}

void twogrid_correct(cudaStream_t st, const Launch& L, const Geom& g, double* hh, double* p, double* p_prev,
                     const double* bsum, double strength, const DevState* ds)
{
    int bxn, byn, bzn;
    twogrid_blocks(g, &bxn, &byn, &bzn);
    twogrid_correct_kernel<<<L.grid, L.block, 0, st>>>(g, hh, p, p_prev, bsum, bxn, byn, strength, ds);
}

void block_abs_sum(cudaStream_t st, const Geom& g, const double* bsum, double* part)
{
    int bxn, byn, bzn;
    const int nb = twogrid_blocks(g, &bxn, &byn, &bzn);
    block_abs_sum_kernel<<<kAndersonBlocks, 256, 0, st>>>(bsum, nb, part);
}

void correct(cudaStream_t st, const Launch& L, const Geom& g, double* u, double* v, double* w,
             const double* p, const double* rho)
{
    correct_kernel<<<L.grid, L.block, 0, st>>>(g, u, v, w, p, rho);
}

}  // namespace fp64

void finalize(cudaStream_t st, FinKind kind, DevState* ds, const double* part, long long nblocks,
              const double* part2, long long nblocks2, const double* part3, long long nblocks3)
{
    finalize_kernel<<<1, 1024, 0, st>>>(static_cast<int>(kind), ds, part, nblocks, part2, nblocks2);
    (void)part3;
    (void)nblocks3;
}

}  // namespace lbm
