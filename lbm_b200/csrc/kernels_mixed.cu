// kernels_mixed.cu -- mixed-precision box: FP32 populations and macro fields,
// FP64 pressure accumulation, reductions and convergence test.
//
// Storage (all q-major SoA like the FP64 box):
//   f*  FP32, deviation from the gas rest-state equilibrium
//       f_rest,q = H_q phi_G + F_q p0(phi_G)      (sum_q f_rest,q = phi_G)
//   g*  FP32, deviation from its rest weight g_rest,q = E_q
//   h*  FP32 (its rest state E_q p_target is ~0: the gauge keeps mean p fixed)
//   phi, rho, u, v, w, div, s, omega_h  FP32;  p, p_prev, p_chk  FP64
// Equilibria and BGK are evaluated directly in deviation form (the rest
// values cancel exactly in f - (f - f_eq)/tau), so FP32 keeps its mantissa
// for the part that moves.  phi = phi_G + sum f_dev and p = sum h are
// accumulated in FP64; all block reductions are FP64.
//
// The kernel sequence and the Poisson segment structure (A/B/C check kernels)
// are those of kernels_fp64.cu; see there for the reference map.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdlib>

#include "collide_zm.cuh"
#include "lbm_mixed.cuh"
#include "mixed_cells.cuh"

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

// Plane-per-CTA collide for boxes the z-marching frame does not tile: stencil
// neighbours gathered from global memory, 64-bit indices.
template <bool kFirst>
__global__ void __launch_bounds__(256)
collide_kernel(Geom g, MixPhys P, const float* __restrict__ fin, float* __restrict__ fout,
               double* __restrict__ f0, const float* __restrict__ gin, float* __restrict__ gout,
               const float* __restrict__ phi, const float* __restrict__ rho,
               const float* __restrict__ u, const float* __restrict__ v,
               const float* __restrict__ w, float* __restrict__ div_out,
               double* __restrict__ part, long long nblocks)
{
    int x, y, z;
    double red[3] = {0.0, 0.0, 0.0};
    if (tile_coords(g, x, y, z)) mixc_collide<kFirst>(g, P, fin, fout, f0, gin, gout, phi, rho, u, v, w, div_out, x, y, z, red);
    block_sum_store<3>(red, part, nblocks, block_linear());
}

// z-marching collide (collide_zm.cuh): one CTA per 32 x 8 column and run of
// zlen planes, macro fields staged through the shared-memory ring, 32-bit
// population offsets.  Same per-cell arithmetic as collide_kernel; the
// source partial sums are accumulated per thread over its planes.
template <bool kFirst>
__global__ void __launch_bounds__(ZM_THREADS, 2)
collide_zm_kernel(Geom g, MixPhys P, int zlen, const float* __restrict__ fin, float* __restrict__ fout,
                  double* __restrict__ f0, const float* __restrict__ gin, float* __restrict__ gout,
                  const float* __restrict__ phi, const float* __restrict__ rho,
                  const float* __restrict__ u, const float* __restrict__ v,
                  const float* __restrict__ w, float* __restrict__ div_out,
                  double* __restrict__ part, long long nblocks)
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
    const MacroRing<float> ring(reinterpret_cast<float*>(zm_raw), g, x0, y0, phi, rho, u, v, w, tid);
    ring.issue(z0 - 1);
    ring.issue(z0);
    ring.issue(z0 + 1);
    double red[3] = {0.0, 0.0, 0.0};
    for (int z = z0; z < z1; ++z) {
        // Both population sets are requested before the plane barrier, so
        // their latency overlaps the wait and the stencil arithmetic.
        float gv[Q], fv[Q];
        const unsigned c = static_cast<unsigned>((z * g.ly + y) * g.lx + x);
        const double f0_in = f0[c];
        if constexpr (!kFirst) {
            pull_regs32(gv, gin, n, g, x, y, z);
            pull_regs32<1>(fv, fin, n, g, x, y, z);
        }
        cp_async_wait_all();
        __syncthreads();
        if (z + 2 <= z1) ring.issue(z + 2);
        CellDeriv<float> d;
        MixCell k;
        // g first: the phi stencil is only live for the f half.
        zm_derivs_g(ring, z, t, d);
        div_out[c] = mix_div(d, red);
        mix_cell_g(P, d, k);
        if constexpr (!kFirst) bounce_regs(gv, g, x);
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            float in = 0.f;
            if constexpr (!kFirst) in = gv[q];
            gout[q * static_cast<unsigned>(n) + c] = mix_g_post<q, kFirst>(P, d, k, in);
        });
        zm_derivs_f(ring, z, t, d);
        mix_cell_f(P, d, k);
        if constexpr (!kFirst) bounce_regs(fv, g, x);
        store_f_post<kFirst>(P, d, k, fv, f0_in, fout, f0, static_cast<unsigned>(n), c);
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
moments_kernel(Geom g, double fei_G, double fei_L, double rho_G, double rho_L, double fei_avg,
               double dfei, double half_drho, const float* __restrict__ f, const double* __restrict__ f0,
               const float* __restrict__ gp, float* __restrict__ phi, float* __restrict__ rho,
               float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
               double* __restrict__ part, long long nblocks)
{
    int x, y, z;
    double red[1] = {0.0};
    const MixMoments M{fei_G, fei_L, rho_G, rho_L, fei_avg, dfei, half_drho};
    if (tile_coords(g, x, y, z)) mixc_moments(g, M, f, f0, gp, phi, rho, u, v, w, x, y, z, red);
    block_sum_store<1>(red, part, nblocks, block_linear());
}

// s = div - mean(div); omega_h = 1 / (1/rho + 1/2); sum(p) for the gauge target.
__global__ void __launch_bounds__(256)
prep_kernel(Geom g, const DevState* __restrict__ ds, const float* __restrict__ div,
            const float* __restrict__ rho, const double* __restrict__ p, float* __restrict__ s,
            float* __restrict__ omega, double* __restrict__ part, long long nblocks)
{
    int x, y, z;
    double red[3] = {0.0, 0.0, 0.0};
    if (tile_coords(g, x, y, z)) mixc_prep(g, ds->div_mean, div, rho, p, s, omega, x, y, z, red);
    block_sum_store<3>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
poisson_init_kernel(Geom g, int h_loaded, const float* __restrict__ hload, float* __restrict__ hout,
                    const double* __restrict__ p, const float* __restrict__ omega,
                    const float* __restrict__ s)
{
    int x, y, z;
    if (tile_coords(g, x, y, z)) mixc_init(g, h_loaded != 0, hload, hout, p, omega, s, x, y, z);
}

// Plain sweep with 32-bit offsets (the launcher uses it when 15 n < 2^31).
__global__ void __launch_bounds__(256)
sweep_kernel(Geom g, const float* __restrict__ hin, float* __restrict__ hout,
             const float* __restrict__ omega, const float* __restrict__ s)
{
    int x, y, z;
    if (tile_coords(g, x, y, z)) mixc_sweep32(g, hin, hout, omega, s, x, y, z);
}

// The same with 64-bit offsets for boxes with 15 n >= 2^31.
__global__ void __launch_bounds__(256)
sweep_kernel64(Geom g, const float* __restrict__ hin, float* __restrict__ hout,
               const float* __restrict__ omega, const float* __restrict__ s)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    float hv[Q];
    pull_regs(hv, hin, g, x, y, z);
    bounce_regs(hv, g, x);
    const P32 ps = sum_q32(hv);
    collide_h_store(hv, (double)ps.hi + (double)ps.lo, __ldg(omega + c), __ldg(s + c), hout, g.n, c);
}

// Two sweeps in one pass (temporal blocking, sweep2_run in mixed_cells.cuh):
// one CTA per 32 x 8 tile of output cells and run of `zlen` planes; sweep k
// on the tile plus its one-cell halo goes into a shared-memory plane ring,
// sweep k+1 pulls from the ring and only the second result is written.
// Requires lx % 32 == 0, ly % 8 == 0 and 15 n < 2^31 (the launcher checks).
constexpr int S2_TX = 32, S2_TY = 8;
constexpr int S2_THREADS = sweep2_threads(S2_TX, S2_TY);   // 352: one thread per region cell
constexpr int S2_SMEM = sweep2_smem(S2_TX, S2_TY);

__global__ void __launch_bounds__(S2_THREADS, 2)
sweep2_kernel(Geom g, int zlen, const float* __restrict__ hin, float* __restrict__ hout,
              const float* __restrict__ omega, const float* __restrict__ s)
{
    extern __shared__ float ring[];
    const int z0 = blockIdx.z * zlen;
    sweep2_run<S2_TX, S2_TY>(g, blockIdx.x * S2_TX, blockIdx.y * S2_TY, z0, min(z0 + zlen, g.lz), hin, hout, omega,
                             s, ring);
}

// The refinement form's correction sweeps two per pass (sweep2_run<., ., true>).
__global__ void __maxnreg__(88)
sweep2_refine_kernel(Geom g, int zlen, const float* __restrict__ ein, float* __restrict__ eout,
                     const float* __restrict__ omega, const float* __restrict__ r)
{
    extern __shared__ float ring[];
    const int z0 = blockIdx.z * zlen;
    sweep2_run<S2_TX, S2_TY, true>(g, blockIdx.x * S2_TX, blockIdx.y * S2_TY, z0, min(z0 + zlen, g.lz), ein, eout,
                                   omega, r, ring);
}

__global__ void __launch_bounds__(256)
sweep_check_a_kernel(Geom g, int zrun, const float* __restrict__ hin, float* __restrict__ hout,
                     double* __restrict__ p_chk, double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[1] = {0.0};
    for (int z = z0; active && z < z1; ++z) mixc_check_a(g, hin, hout, p_chk, x, y, z, red);
    block_sum_store<1>(red, part, nblocks, block_linear());
}

template <bool kDual>
__global__ void __launch_bounds__(256)
sweep_check_b_kernel(Geom g, int zrun, const float* __restrict__ hin, float* __restrict__ hout,
                     float* __restrict__ hc,
                     const double* __restrict__ p_chk, double* __restrict__ p_prev,
                     double* __restrict__ p, const float* __restrict__ omega,
                     const float* __restrict__ s, const DevState* __restrict__ ds,
                     double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double shift = ds->sigma;
    const double tgt = ds->target;
    for (int z = z0; active && z < z1; ++z)
        mixc_check_b<kDual>(g, hin, hout, hc, p_chk, p_prev, p, omega, s, shift, tgt, x, y, z, red);
    block_sum_store<5>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
sweep_check_c_kernel(Geom g, int zrun, const float* __restrict__ hin, float* __restrict__ hout,
                     const float* __restrict__ hc, const float* __restrict__ omega,
                     const float* __restrict__ s, const DevState* __restrict__ ds,
                     double* __restrict__ part, long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[3] = {0.0, 0.0, 0.0};
    const double tgt = ds->target;
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        float hv[Q];
        pull_regs(hv, hin, g, x, y, z);
        bounce_regs(hv, g, x);
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const double hval = hc[(long long)q * g.n + c];
            const double ge = wE(q) * tgt;
            red[0] += fabs(hval - (double)hv[q]);
            red[1] += fabs(hval - ge);
            red[2] += fabs((double)hv[q] - ge);
        });
        collide_h_store(hv, sum_q(hv), __ldg(omega + c), __ldg(s + c), hout, g.n, c);
    }
    block_sum_store<3>(red, part, nblocks, block_linear());
}

// ---- iterative refinement of the Poisson solve (LBM_POISSON_REFINE) ------
// The FP32 sweeps alone stall at a relative change of ~1e-7: every sweep
// rounds h to FP32, and the kinetic map's slow modes (relaxation over ~1e5
// sweeps at 64^3) amplify that noise, so the FP32 iteration's limit sits
// ~1e-4 of max|p| away from the FP64 fixed point.  Refinement keeps the
// post-collision state H in FP64 and computes each segment's sweeps as a
// correction: r = K H + b - H in FP64 (b = -(E/3) s), then e_1 = r and
// e_(k+1) = K e_k + r in FP32, so that H + e_k is, in exact arithmetic, the
// state after k sweeps from H; the FP32 rounding now applies to the
// correction, which shrinks as the solve converges.  Checks A and B run in
// FP64 on H + e, as the FP64 box's do.  K uses the box's FP32 omega and s as
// data in both precisions, so the fixed point is the mixed box's own.

// FP64 Poisson start: H = collide(E p) (or of the loaded FP32 h).
__global__ void __launch_bounds__(256)
refine_init_kernel(Geom g, int h_loaded, const float* __restrict__ hload, double* __restrict__ hd,
                   const double* __restrict__ p, const float* __restrict__ omega, const float* __restrict__ s)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    const double pv = p[c];
    double hv[Q];
    double sum = 0.0;
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hv[q] = h_loaded ? (double)hload[(long long)q * g.n + c] : pv * wE(q);
        sum += hv[q];
    });
    const double om = omega[c], sv = s[c];
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hd[(long long)q * g.n + c] = hv[q] - om * (hv[q] - wE(q) * sum) - wE(q) / 3.0 * sv;
    });
}

// r = K H + b - H (FP64 arithmetic, stored in FP32).
__global__ void __launch_bounds__(256)
refine_residual_kernel(Geom g, const double* __restrict__ hd, float* __restrict__ r,
                       const float* __restrict__ omega, const float* __restrict__ s)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    const Wrap w(g, x, y, z);
    double hv[Q];
    double pv = 0.0;
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        hv[q] = __ldg(hd + (long long)q * g.n + pull_src<q>(g, w, x, y, z));
    });
    bounce_regs(hv, g, x);
    static_for<0, Q>([&](auto qc) { pv += hv[decltype(qc)::value]; });
    const double om = __ldg(omega + c), sv = __ldg(s + c);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const long long i = (long long)q * g.n + c;
        const double kh = hv[q] - om * (hv[q] - wE(q) * pv) - wE(q) / 3.0 * sv;
        r[i] = (float)(kh - __ldg(hd + i));
    });
}

// One correction sweep in FP32: e' = K e + r.
__global__ void __launch_bounds__(256)
refine_sweep_kernel(Geom g, const float* __restrict__ ein, float* __restrict__ eout, const float* __restrict__ r,
                    const float* __restrict__ omega)
{
    int x, y, z;
    if (!tile_coords(g, x, y, z)) return;
    const long long c = cell_of(g, x, y, z);
    float ev[Q];
    pull_regs(ev, ein, g, x, y, z);
    bounce_regs(ev, g, x);
    const float pe = refine_sum(ev);
    const float om = __ldg(omega + c);
    static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const long long i = (long long)q * g.n + c;
        eout[i] = refine_cell<q>(ev[q], pe, om, __ldg(r + i));
    });
}

// Check A in FP64: pull H + e, slip, p = sum (FP64); the uncollided values
// go to hpre, red[0] += p.
__global__ void __launch_bounds__(256)
refine_check_a_kernel(Geom g, int zrun, const double* __restrict__ hd, const float* __restrict__ e,
                      double* __restrict__ hpre, double* __restrict__ p_chk, double* __restrict__ part,
                      long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[1] = {0.0};
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        const Wrap w(g, x, y, z);
        double hv[Q];
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const long long src = (long long)q * g.n + pull_src<q>(g, w, x, y, z);
            hv[q] = __ldg(hd + src) + (double)__ldg(e + src);
        });
        bounce_regs(hv, g, x);
        double pv = 0.0;
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            pv += hv[q];
            hpre[(long long)q * g.n + c] = hv[q];
        });
        p_chk[c] = pv;
        red[0] += pv;
    }
    block_sum_store<1>(red, part, nblocks, block_linear());
}

// Check B in FP64: gauge (p -= shift, h -= E shift), relative-change terms,
// p and p_prev, then the collision of the next sweep, in place.
__global__ void __launch_bounds__(256)
refine_check_b_kernel(Geom g, int zrun, double* __restrict__ hd, const double* __restrict__ p_chk,
                      double* __restrict__ p_prev, double* __restrict__ p, const float* __restrict__ omega,
                      const float* __restrict__ s, const DevState* __restrict__ ds, double* __restrict__ part,
                      long long nblocks)
{
    int x, y, z0, z1;
    const bool active = tile_zrun(g, zrun, x, y, z0, z1);
    double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double shift = ds->sigma;
    for (int z = z0; active && z < z1; ++z) {
        const long long c = cell_of(g, x, y, z);
        const double pv = p_chk[c] - shift;
        red[0] += fabs(pv - p_prev[c]);
        red[1] += fabs(pv);
        p_prev[c] = pv;
        p[c] = pv;
        const double om = __ldg(omega + c), sv = __ldg(s + c);
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            const long long i = (long long)q * g.n + c;
            const double hv = hd[i] - wE(q) * shift;
            hd[i] = hv - om * (hv - wE(q) * pv) - wE(q) / 3.0 * sv;
        });
    }
    block_sum_store<5>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
refine_to_float_kernel(const double* __restrict__ src, float* __restrict__ dst, long long count)
{
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < count; i += (long long)gridDim.x * 256)
        dst[i] = (float)src[i];
}

__global__ void __launch_bounds__(256)
correct_kernel(Geom g, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
               const double* __restrict__ p, const float* __restrict__ rho)
{
    int x, y, z;
    if (tile_coords(g, x, y, z)) mixc_correct(g, u, v, w, p, rho, x, y, z);
}

__global__ void to_float_kernel(const double* __restrict__ src, float* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

// f0 = phi - phi_G: a loaded state keeps all of phi's deviation in the rest
// population until the first collision (which does not read the others).
__global__ void rest_from_phi_kernel(const double* __restrict__ phi, double* __restrict__ f0, double fei_G,
                                     long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        f0[i] = (phi ? phi[i] : 0.0) - fei_G;
}

__global__ void to_double_kernel(const float* __restrict__ src, double* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

float* field_f(MixedBuffers& mb, int which)
{
    switch (which) {
    case 0: return mb.phi;
    case 1: return mb.rho;
    case 2: return mb.u;
    case 3: return mb.v;
    case 4: return mb.w;
    }
    return nullptr;
}

}  // namespace

lbm_status mixed_alloc(MixedBuffers& mb, const Geom& g, const Launch& L)
{
    const size_t n = static_cast<size_t>(g.n);
    auto okf = [&](float** p, size_t count) { return cudaMalloc(p, count * sizeof(float)) == cudaSuccess; };
    auto okd = [&](double** p, size_t count) { return cudaMalloc(p, count * sizeof(double)) == cudaSuccess; };
    bool ok = true;
    for (int i = 0; i < 2; ++i) ok = ok && okf(&mb.f[i], 15 * n) && okf(&mb.g[i], 15 * n) && okf(&mb.h[i], 15 * n);
    ok = ok && okf(&mb.phi, n) && okf(&mb.rho, n) && okf(&mb.u, n) && okf(&mb.v, n) && okf(&mb.w, n) &&
         okf(&mb.s, n) && okf(&mb.dux, n) && okf(&mb.dvy, n);
    ok = ok && okd(&mb.p, n) && okd(&mb.p_prev, n) && okd(&mb.p_chk, n) && okd(&mb.scratch, n) && okd(&mb.f0, n);
    const size_t nb = static_cast<size_t>(L.nblocks);
    ok = ok && okd(&mb.part_src, 3 * nb) && okd(&mb.part_prep, 3 * nb) && okd(&mb.part_a, nb) &&
         okd(&mb.part_b, 5 * nb) && okd(&mb.part_c, 3 * nb) && okd(&mb.part_mass, nb);
    if (!ok) {
        mixed_free(mb);
        return LBM_ERR_OOM;
    }
    cudaMemset(mb.part_c, 0, 3 * nb * sizeof(double));
    mb.dwz = nullptr;
    // Two-sweep temporal blocking where the tile divides the box, on z runs
    // of the longest length in {32, 16, 8} whose grid still gives every SM
    // 1.5 CTAs (shorter runs recompute more halo planes; a grid of fewer CTAs
    // leaves SMs idle): measured on B200 (us per sweep, mixed), 128^3: 32.4
    // at runs of 32 (256 CTAs); 96^3: 15.7 at 8 (432) against 22.2 at 32;
    // 64^3 and 32^3: single sweeps 4.9 and 2.1 against 5.4 and 3.5 at the
    // best run length, so no two-sweep pass below 1.5 CTAs per SM at runs of
    // 8.  LBM_SWEEP2_ZLEN overrides (0 disables).
    mb.fuse_zlen = 0;
    int zlen = 0;
    if (const char* env = std::getenv("LBM_SWEEP2_ZLEN")) {
        zlen = std::atoi(env);
    } else if (g.lx % S2_TX == 0 && g.ly % S2_TY == 0) {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 148;
        const long long tiles = static_cast<long long>(g.lx / S2_TX) * (g.ly / S2_TY);
        for (int zl : {32, 16, 8}) {
            if (2 * tiles * ((g.lz + zl - 1) / zl) >= 3LL * sms) {
                zlen = zl;
                break;
            }
        }
    }
    if (zlen > 0 && g.lx % S2_TX == 0 && g.ly % S2_TY == 0 && g.lz >= 3 && 15 * g.n < 0x7fffffffLL &&
        cudaFuncSetAttribute(sweep2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, S2_SMEM) == cudaSuccess &&
        cudaFuncSetAttribute(sweep2_refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, S2_SMEM) ==
            cudaSuccess)
        mb.fuse_zlen = zlen;
    // z-marching collide where its tile divides the box.
    const char* cenv = std::getenv("LBM_COLLIDE_ZLEN");
    const int czlen = cenv ? std::atoi(cenv) : 16;
    mb.collide_zlen = (czlen > 0 && zm_fits(g)) ? czlen : 0;
    mb.allocated = true;
    return LBM_OK;
}

lbm_status mixed_alloc_dual(MixedBuffers& mb, const Geom& g)
{
    if (mb.hc) return LBM_OK;
    if (cudaMalloc(&mb.hc, 15 * static_cast<size_t>(g.n) * sizeof(float)) != cudaSuccess) return LBM_ERR_OOM;
    return LBM_OK;
}

void mixed_free(MixedBuffers& mb)
{
    float** fl[] = {&mb.f[0], &mb.f[1], &mb.g[0], &mb.g[1], &mb.h[0], &mb.h[1], &mb.hc, &mb.phi, &mb.rho,
                    &mb.u, &mb.v, &mb.w, &mb.s, &mb.dux, &mb.dvy, &mb.dwz};
    for (float** p : fl) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    double** db[] = {&mb.p, &mb.p_prev, &mb.p_chk, &mb.scratch, &mb.f0, &mb.part_src, &mb.part_prep, &mb.part_a,
                     &mb.part_b, &mb.part_c, &mb.part_mass, &mb.hd[0], &mb.hd[1]};
    for (double** p : db) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (mb.rr) cudaFree(mb.rr);
    mb.rr = nullptr;
    mb.allocated = false;
}

lbm_status mixed_load(cudaStream_t st, MixedBuffers& mb, const Geom& g, const Phys& P,
                      const double* const src[6], cudaMemcpyKind kind)
{
    const size_t n = static_cast<size_t>(g.n);
    const int blocks = 1184;
    for (int i = 0; i < 5; ++i) {
        float* dst = field_f(mb, i);
        if (src[i]) {
            if (cudaMemcpyAsync(mb.scratch, src[i], n * sizeof(double), kind, st) != cudaSuccess) return LBM_ERR_CUDA;
            to_float_kernel<<<blocks, 256, 0, st>>>(mb.scratch, dst, g.n);
        } else if (cudaMemsetAsync(dst, 0, n * sizeof(float), st) != cudaSuccess) {
            return LBM_ERR_CUDA;
        }
        if (i == 0) rest_from_phi_kernel<<<blocks, 256, 0, st>>>(src[0] ? mb.scratch : nullptr, mb.f0, P.fei_G, g.n);
    }
    if (src[5]) {
        if (cudaMemcpyAsync(mb.p, src[5], n * sizeof(double), kind, st) != cudaSuccess) return LBM_ERR_CUDA;
    } else if (cudaMemsetAsync(mb.p, 0, n * sizeof(double), st) != cudaSuccess) {
        return LBM_ERR_CUDA;
    }
    if (cudaMemsetAsync(mb.p_prev, 0, n * sizeof(double), st) != cudaSuccess) return LBM_ERR_CUDA;
    if (cudaMemsetAsync(mb.h[1], 0, 15 * n * sizeof(float), st) != cudaSuccess) return LBM_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

lbm_status mixed_download(cudaStream_t st, MixedBuffers& mb, const Geom& g, int which, double* host)
{
    const size_t n = static_cast<size_t>(g.n);
    if (which == 5) {
        return cudaMemcpyAsync(host, mb.p, n * sizeof(double), cudaMemcpyDeviceToHost, st) == cudaSuccess
                   ? LBM_OK : LBM_ERR_CUDA;
    }
    float* src = field_f(mb, which);
    if (!src) return LBM_ERR_BAD_ARG;
    to_double_kernel<<<1184, 256, 0, st>>>(src, mb.scratch, g.n);
    if (cudaMemcpyAsync(host, mb.scratch, n * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return LBM_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

lbm_status mixed_prologue(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g,
                          const Phys& P, bool first, int fcur, bool h_loaded, DevState* ds,
                          cudaEvent_t* ev)
{
    const MixPhys M = mix_phys(P);
    const int fin = fcur, fout = 1 - fcur;
    float* div = mb.dux;      // div = u_x + v_y + w_z
    float* omega = mb.dvy;    // 1 / tau_h
    long long src_blocks = L.nblocks;
    if (mb.collide_zlen > 0) {
        const dim3 grid(g.lx / ZM_TX, g.ly / ZM_TY, (g.lz + mb.collide_zlen - 1) / mb.collide_zlen);
        src_blocks = static_cast<long long>(grid.x) * grid.y * grid.z;
        constexpr int smem = zm_ring_bytes<float>();
        auto kern = first ? collide_zm_kernel<true> : collide_zm_kernel<false>;
        kern<<<grid, ZM_THREADS, smem, st>>>(g, M, mb.collide_zlen, mb.f[fin], mb.f[fout], mb.f0, mb.g[fin],
                                             mb.g[fout],
                                             mb.phi, mb.rho, mb.u, mb.v, mb.w, div, mb.part_src, src_blocks);
    } else if (first) {
        collide_kernel<true><<<L.grid, L.block, 0, st>>>(g, M, mb.f[fin], mb.f[fout], mb.f0, mb.g[fin], mb.g[fout],
                                                         mb.phi, mb.rho, mb.u, mb.v, mb.w, div,
                                                         mb.part_src, L.nblocks);
    } else {
        collide_kernel<false><<<L.grid, L.block, 0, st>>>(g, M, mb.f[fin], mb.f[fout], mb.f0, mb.g[fin], mb.g[fout],
                                                          mb.phi, mb.rho, mb.u, mb.v, mb.w, div,
                                                          mb.part_src, L.nblocks);
    }
    if (ev) cudaEventRecord(ev[1], st);
    moments_kernel<<<L.grid, L.block, 0, st>>>(g, P.fei_G, P.fei_L, P.rho_G, P.rho_L, P.fei_avg, P.dfei,
                                               P.half_drho, mb.f[fout], mb.f0, mb.g[fout], mb.phi, mb.rho, mb.u,
                                               mb.v, mb.w, mb.part_mass, L.nblocks);
    if (ev) cudaEventRecord(ev[2], st);
    finalize(st, FIN_SOURCE, ds, mb.part_src, src_blocks, nullptr, 0, nullptr, 0);
    finalize(st, FIN_MASS, ds, mb.part_mass, L.nblocks, nullptr, 0, nullptr, 0);
    prep_kernel<<<L.grid, L.block, 0, st>>>(g, ds, div, mb.rho, mb.p, mb.s, omega, mb.part_prep, L.nblocks);
    finalize(st, FIN_PREP, ds, mb.part_prep, L.nblocks, nullptr, 0, nullptr, 0);
    poisson_init_kernel<<<L.grid, L.block, 0, st>>>(g, h_loaded ? 1 : 0, mb.h[1], mb.h[0], mb.p, omega, mb.s);
    return cudaGetLastError() == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

int mixed_segment(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g, int start_parity,
                  int n_normal, bool dual, DevState* ds)
{
    const float* omega = mb.dvy;
    int cur = start_parity;
    if (mb.fuse_zlen > 0) {
        const dim3 grid(g.lx / S2_TX, g.ly / S2_TY, (g.lz + mb.fuse_zlen - 1) / mb.fuse_zlen);
        for (int i = 0; i + 1 < n_normal; i += 2) {
            sweep2_kernel<<<grid, S2_THREADS, S2_SMEM, st>>>(g, mb.fuse_zlen, mb.h[cur], mb.h[1 - cur],
                                                                     omega, mb.s);
            cur = 1 - cur;
        }
        n_normal &= 1;
    }
    const bool off32 = 15 * g.n < 0x7fffffffLL;
    for (int i = 0; i < n_normal; ++i) {
        if (off32)
            sweep_kernel<<<L.grid, L.block, 0, st>>>(g, mb.h[cur], mb.h[1 - cur], omega, mb.s);
        else
            sweep_kernel64<<<L.grid, L.block, 0, st>>>(g, mb.h[cur], mb.h[1 - cur], omega, mb.s);
        cur = 1 - cur;
    }
    sweep_check_a_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, mb.h[cur], mb.h[1 - cur], mb.p_chk, mb.part_a,
                                                      L.cnblocks);
    cur = 1 - cur;
    finalize(st, FIN_SIGMA, ds, mb.part_a, L.cnblocks, nullptr, 0, nullptr, 0);
    if (dual)
        sweep_check_b_kernel<true><<<L.cgrid, L.block, 0, st>>>(g, L.zrun, mb.h[cur], mb.h[1 - cur], mb.hc,
                                                                mb.p_chk, mb.p_prev, mb.p, omega, mb.s, ds,
                                                                mb.part_b, L.cnblocks);
    else
        sweep_check_b_kernel<false><<<L.cgrid, L.block, 0, st>>>(g, L.zrun, mb.h[cur], mb.h[1 - cur], mb.hc,
                                                                 mb.p_chk, mb.p_prev, mb.p, omega, mb.s, ds,
                                                                 mb.part_b, L.cnblocks);
    cur = 1 - cur;
    if (dual) {
        sweep_check_c_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, mb.h[cur], mb.h[1 - cur], mb.hc, omega, mb.s,
                                                          ds, mb.part_c, L.cnblocks);
        cur = 1 - cur;
    }
    finalize(st, FIN_CHECK, ds, mb.part_b, L.cnblocks, mb.part_c, L.cnblocks, nullptr, 0);
    return cur;
}

void mixed_correct(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g)
{
    correct_kernel<<<L.grid, L.block, 0, st>>>(g, mb.u, mb.v, mb.w, mb.p, mb.rho);
}

lbm_status mixed_alloc_refine(MixedBuffers& mb, const Geom& g)
{
    if (mb.rr) return LBM_OK;
    const size_t n15 = 15 * static_cast<size_t>(g.n);
    double* hd[2] = {nullptr, nullptr};
    float* rr = nullptr;
    if (cudaMalloc(&hd[0], n15 * sizeof(double)) != cudaSuccess || cudaMalloc(&hd[1], n15 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&rr, n15 * sizeof(float)) != cudaSuccess) {
        if (hd[0]) cudaFree(hd[0]);
        if (hd[1]) cudaFree(hd[1]);
        if (rr) cudaFree(rr);
        cudaGetLastError();
        return LBM_ERR_OOM;
    }
    mb.hd[0] = hd[0];
    mb.hd[1] = hd[1];
    mb.rr = rr;
    return LBM_OK;
}

void mixed_refine_init(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g, bool h_loaded)
{
    refine_init_kernel<<<L.grid, L.block, 0, st>>>(g, h_loaded ? 1 : 0, mb.h[1], mb.hd[0], mb.p, mb.dvy, mb.s);
}

int mixed_refine_segment(cudaStream_t st, MixedBuffers& mb, const Launch& L, const Geom& g, int start_parity,
                         int n_normal, DevState* ds)
{
    const float* omega = mb.dvy;
    double* H = mb.hd[start_parity];
    double* Hn = mb.hd[1 - start_parity];
    // sweep 1 as the residual: e_1 = r = K H + b - H
    refine_residual_kernel<<<L.grid, L.block, 0, st>>>(g, H, mb.rr, omega, mb.s);
    // sweeps 2 .. n_normal as FP32 corrections e_(k+1) = K e_k + r, two per
    // pass where the box runs two-sweep passes
    const float* e = mb.rr;
    int cur = 0;
    int i = 1;
    if (mb.fuse_zlen > 0) {
        const dim3 grid(g.lx / S2_TX, g.ly / S2_TY, (g.lz + mb.fuse_zlen - 1) / mb.fuse_zlen);
        for (; i + 1 < n_normal; i += 2) {
            sweep2_refine_kernel<<<grid, S2_THREADS, S2_SMEM, st>>>(g, mb.fuse_zlen, e, mb.h[cur], omega, mb.rr);
            e = mb.h[cur];
            cur = 1 - cur;
        }
    }
    for (; i < n_normal; ++i) {
        refine_sweep_kernel<<<L.grid, L.block, 0, st>>>(g, e, mb.h[cur], mb.rr, omega);
        e = mb.h[cur];
        cur = 1 - cur;
    }
    // the check sweep in FP64 on H + e
    refine_check_a_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, H, e, Hn, mb.p_chk, mb.part_a, L.cnblocks);
    finalize(st, FIN_SIGMA, ds, mb.part_a, L.cnblocks, nullptr, 0, nullptr, 0);
    refine_check_b_kernel<<<L.cgrid, L.block, 0, st>>>(g, L.zrun, Hn, mb.p_chk, mb.p_prev, mb.p, omega, mb.s, ds,
                                                       mb.part_b, L.cnblocks);
    finalize(st, FIN_CHECK, ds, mb.part_b, L.cnblocks, nullptr, 0, nullptr, 0);
    return 1 - start_parity;
}

void mixed_refine_finish(cudaStream_t st, MixedBuffers& mb, const Geom& g, int parity)
{
    refine_to_float_kernel<<<1184, 256, 0, st>>>(mb.hd[parity], mb.h[parity], 15 * g.n);
}

// Layout of a saved state: f (15 n floats), g (15 n floats), phi, rho, u,
// v, w (5 n floats), f0 (n doubles), p (n doubles); 8-byte aligned pieces.
size_t mixed_state_bytes(const Geom& g)
{
    const size_t n = static_cast<size_t>(g.n);
    return (35 * n * sizeof(float) + 7) / 8 * 8 + 2 * n * sizeof(double);
}

namespace {
struct StatePieces {
    float* pop[2];
    float* macro[5];
    double* f0;
    double* p;
};
StatePieces state_pieces(void* base, const Geom& g)
{
    const size_t n = static_cast<size_t>(g.n);
    float* f = static_cast<float*>(base);
    StatePieces s;
    s.pop[0] = f;
    s.pop[1] = f + 15 * n;
    for (int i = 0; i < 5; ++i) s.macro[i] = f + 30 * n + i * n;
    char* d = static_cast<char*>(base) + (35 * n * sizeof(float) + 7) / 8 * 8;
    s.f0 = reinterpret_cast<double*>(d);
    s.p = s.f0 + n;
    return s;
}
}  // namespace

lbm_status mixed_save_state(cudaStream_t st, const MixedBuffers& mb, const Geom& g, int fcur, void* dst)
{
    const size_t n = static_cast<size_t>(g.n);
    const StatePieces s = state_pieces(dst, g);
    const float* src[5] = {mb.phi, mb.rho, mb.u, mb.v, mb.w};
    bool ok = cudaMemcpyAsync(s.pop[0], mb.f[fcur], 15 * n * sizeof(float), cudaMemcpyDeviceToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(s.pop[1], mb.g[fcur], 15 * n * sizeof(float), cudaMemcpyDeviceToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(s.f0, mb.f0, n * sizeof(double), cudaMemcpyDeviceToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(s.p, mb.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    for (int i = 0; i < 5 && ok; ++i)
        ok = cudaMemcpyAsync(s.macro[i], src[i], n * sizeof(float), cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    return ok ? LBM_OK : LBM_ERR_CUDA;
}

lbm_status mixed_restore_state(cudaStream_t st, MixedBuffers& mb, const Geom& g, int fcur, const void* src)
{
    const size_t n = static_cast<size_t>(g.n);
    const StatePieces s = state_pieces(const_cast<void*>(src), g);
    float* dst[5] = {mb.phi, mb.rho, mb.u, mb.v, mb.w};
    bool ok = cudaMemcpyAsync(mb.f[fcur], s.pop[0], 15 * n * sizeof(float), cudaMemcpyDeviceToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(mb.g[fcur], s.pop[1], 15 * n * sizeof(float), cudaMemcpyDeviceToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(mb.f0, s.f0, n * sizeof(double), cudaMemcpyDeviceToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(mb.p, s.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    for (int i = 0; i < 5 && ok; ++i)
        ok = cudaMemcpyAsync(dst[i], s.macro[i], n * sizeof(float), cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    return ok ? LBM_OK : LBM_ERR_CUDA;
}

lbm_status mixed_export(cudaStream_t st, const MixedBuffers& mb, const Geom& g, int hbuf, double* macro6,
                        double* h15)
{
    const size_t n = static_cast<size_t>(g.n);
    const float* src[5] = {mb.phi, mb.rho, mb.u, mb.v, mb.w};
    for (int i = 0; i < 5; ++i) to_double_kernel<<<1184, 256, 0, st>>>(src[i], macro6 + i * n, g.n);
    if (cudaMemcpyAsync(macro6 + 5 * n, mb.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return LBM_ERR_CUDA;
    if (h15) to_double_kernel<<<1184, 256, 0, st>>>(mb.h[hbuf], h15, 15 * g.n);
    return cudaGetLastError() == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

const void* mixed_field_ptr(const MixedBuffers& mb, int which)
{
    switch (which) {
    case 0: return mb.phi;
    case 1: return mb.rho;
    case 2: return mb.u;
    case 3: return mb.v;
    case 4: return mb.w;
    case 5: return mb.p;
    }
    return nullptr;
}

}  // namespace lbm
