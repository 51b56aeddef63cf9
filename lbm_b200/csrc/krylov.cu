// krylov.cu -- the kinetic Poisson fixed point solved by BiCGSTAB
// (LBM_POISSON_KRYLOV), FP64.
//
// The production solve iterates h <- K h + b to its fixed point (Richardson):
// K = collide o (pull + x-wall overwrite) without the source,
// collide: hv -> hv - (hv - E_q sum(hv)) / tau_h, tau_h = 1/rho + 1/2, and
// b_q = -(E_q / 3) s (CPU/Inamuro.cpp:755-793).  This form solves the same
// linear system (I - K) h = b by BiCGSTAB (van der Vorst 1992) on the
// post-collision populations, so it converges to the same fixed point; p is
// then the sum of the pulled populations, gauged to the step's target mean.
// (I - K) is singular (constant p).  With x periodic the system is
// consistent (the projected source has zero sum); with the slip walls it is
// not, and the solve runs on the bordered system of the sweeps' gauged fixed
// point (bicgstab below).  One iteration is two applications of K
// (each one pass over the populations, like a sweep) and the vector updates;
// the five inner products per iteration are fixed-order block partial sums
// added on the host.  The exit: ||b - (I - K) h||_2 < tolerance ||b||_2.
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/lbm_b200.h"
#include "lbm_solver.cuh"

namespace lbm {
namespace {

constexpr int kDotBlocks = kKrylovBlocks;

__device__ __forceinline__ bool kcell(const Geom& g, int& x, int& y, int& z)
{
    x = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    z = blockIdx.z;
    return x < g.lx && y < g.ly;
}

// out = in - K src (kinds 0, 2), or out = b - (in - K src) (kind 1, a true
// residual), with b = bvec when given, else b_q = -(E/3) s; src = in for the
// plain operator I - K, src = K^(m-1) in for the polynomial form I - K^m.
// Kind 3: out = K src alone.  Partial sums: kind 0 dot(w, out) and
// dot(out, out); kind 1 dot(out, out); kind 2 dot(w, out) and dot(out, out).
// kAdj: the adjoint solve's operator B = M^T o (the transposed pull tpull:
// the slip overwrite's transpose, then the pull from x + c_q) instead of K
// (M^T m = (1 - 1/tau) m + (sum_k E_k m_k) / tau per cell), and b_q = s (the
// adjoint of p, the same for every q).  Its system is consistent on both x
// boundaries: E^T B = E^T and s has zero sum.
// Bordered form (slip walls, forward): in_delta E_q is added to in - K src
// (the drift column), and sum_p asks for the partial sums of
// sum_x (p(x) - p_ref), p = the sum of the pulled, bounced src, as one more
// column (kinds 0-2: column 2; kind 3: column 0 of `part`).
template <int kKind, bool kAdj>
__global__ void __launch_bounds__(256)
apply_kernel(Geom g, const double* __restrict__ in, const double* __restrict__ src, double* __restrict__ out,
             const double* __restrict__ rho, const double* __restrict__ s, const double* __restrict__ bvec,
             const double* __restrict__ w, double* __restrict__ part, long long nblocks, double in_delta,
             int sum_p, double p_ref)
{
    int x, y, z;
    const bool active = kcell(g, x, y, z);
    double red[3] = {0.0, 0.0, 0.0};
    if (active) {
        const long long n = g.n;
        const long long c = cell_of(g, x, y, z);
        const Wrap wr(g, x, y, z);
        double hv[Q];
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (kAdj)
                hv[q] = tpull<q>(src, n, g, wr, x, y, z);
            else
                hv[q] = __ldg(src + (long long)q * n + pull_src<q>(g, wr, x, y, z));
        });
        if constexpr (!kAdj) bounce_regs(hv, g, x);
        double p = 0.0;
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            p += kAdj ? wE(q) * hv[q] : hv[q];
        });
        red[2] = p - p_ref;
        const double inv_tau = 1.0 / (1.0 / __ldg(rho + c) + 0.5);
        const double sv = (kKind == 1 && !bvec) ? __ldg(s + c) : 0.0;
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            constexpr double E = wE(q);
            const long long i = (long long)q * n + c;
            const double kh = kAdj ? hv[q] - (hv[q] - p) * inv_tau : hv[q] - (hv[q] - E * p) * inv_tau;
            if constexpr (kKind == 3) {
                out[i] = kh;
                return;
            }
            double v = __ldg(in + i) - kh;
            if (in_delta != 0.0) v += in_delta * E;
            if constexpr (kKind == 1) v = (bvec ? __ldg(bvec + i) : (kAdj ? sv : -(E / 3.0) * sv)) - v;
            out[i] = v;
            if constexpr (kKind == 0 || kKind == 2) {
                red[0] += __ldg(w + i) * v;
                red[1] += v * v;
            }
            if constexpr (kKind == 1) red[0] += v * v;
        });
    }
    if constexpr (kKind == 3) {
        if (sum_p) {
            double r1[1] = {red[2]};
            block_sum_store<1>(r1, part, nblocks, block_linear());
        }
    } else if (sum_p) {
        block_sum_store<3>(red, part, nblocks, block_linear());
    } else {
        double r2[2] = {red[0], red[1]};
        block_sum_store<2>(r2, part, nblocks, block_linear());
    }
}

// Grid-stride vector updates over the 15 n populations.
// op 0: p = r + beta (p - omega v)
// op 1: s = r - alpha v
// op 2: x += alpha p + omega s; r = s - omega t; partials of r.r and r0.r
// op 3: copy (r0 = r, p = r)
// op 4: y0 += x0 (the polynomial right-hand side's sum)
template <int kOp>
__global__ void __launch_bounds__(256)
vec_kernel(long long count, double a0, double a1, double* __restrict__ y0, double* __restrict__ y1,
           const double* __restrict__ x0, const double* __restrict__ x1, const double* __restrict__ x2,
           const double* __restrict__ x3, double* __restrict__ part)
{
    double red[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < count; i += (long long)gridDim.x * 256) {
        if constexpr (kOp == 0) {
            y0[i] = x0[i] + a0 * (y0[i] - a1 * x1[i]);
        } else if constexpr (kOp == 1) {
            y0[i] = x0[i] - a0 * x1[i];
        } else if constexpr (kOp == 2) {
            // y0 = x (solution), y1 = r; x0 = p, x1 = s, x2 = t, x3 = r0
            y0[i] = y0[i] + a0 * x0[i] + a1 * x1[i];
            const double r = x1[i] - a1 * x2[i];
            y1[i] = r;
            red[0] += r * r;
            red[1] += x3[i] * r;
        } else if constexpr (kOp == 3) {
            y0[i] = x0[i];
            y1[i] = x0[i];
        } else {
            y0[i] += x0[i];
        }
    }
    if constexpr (kOp == 2) block_sum_store<2>(red, part, gridDim.x, blockIdx.x);
}

// p = sum of the pulled, bounced populations of the solution (the p a sweep
// would compute), and its block partial sums for the gauge mean.
__global__ void __launch_bounds__(256)
pressure_kernel(Geom g, const double* __restrict__ h, double* __restrict__ p, double* __restrict__ part,
                long long nblocks)
{
    int x, y, z;
    const bool active = kcell(g, x, y, z);
    double red[1] = {0.0};
    if (active) {
        const Wrap wr(g, x, y, z);
        double hv[Q];
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            hv[q] = __ldg(h + (long long)q * g.n + pull_src<q>(g, wr, x, y, z));
        });
        bounce_regs(hv, g, x);
        double pv = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) pv += hv[q];
        p[cell_of(g, x, y, z)] = pv;
        red[0] = pv;
    }
    block_sum_store<1>(red, part, nblocks, block_linear());
}

__global__ void __launch_bounds__(256)
shift_kernel(long long n, double* __restrict__ p, double* __restrict__ p_prev, double shift)
{
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
        const double v = p[i] - shift;
        p[i] = v;
        p_prev[i] = v;
    }
}

}  // namespace

namespace krylov {
namespace {

// BiCGSTAB iterations on (I - A_op) h = b from the initial guess in h; the
// operator and source as apply_kernel<., kAdj>.  degree m > 1: the same
// solution from the polynomially preconditioned system
// (I - A_op^m) h = (I + A_op + ... + A_op^(m-1)) b (Neumann series of
// (I - A_op)^-1 truncated after m terms as left preconditioner), which takes
// fewer iterations -- so fewer of the memory-bound vector updates and host
// round trips -- for m applications of A_op per operator.  *budget: stopped
// at the cap.
//
// Slip walls (forward): the walls' overwrite makes (I - K) h = b
// inconsistent (its left null vector is not uniform), and the sweeps' fixed
// point is that of the bordered system
//   (I - K^m) h + delta E = b_m,   sum_x p(h) = N target
// (p(h) the sum of the pulled, bounced h; delta the drift the gauge removes,
// m times the per-sweep drift for degree m; the same h for every m).  The
// method runs on the bordered vectors (h, delta): the device holds the h
// parts, the host the delta parts, each updated with the same coefficients,
// and every inner product adds the product of the delta parts.  With the row
// scaled by N the drift column E and the row have comparable norms.
template <bool kAdj>
lbm_status bicgstab(cudaStream_t st, const Launch& L, const Geom& g, const KrylovBuffers& kb, double* h,
                    const double* rho, const double* s, double target, double tol, uint64_t max_matvecs,
                    int degree, KrylovResult* res, bool* budget_out)
{
    const long long cnt = 15 * g.n;
    const int m = degree > 1 ? degree : 1;
    const bool border = !kAdj && !g.periodic_x;
    double* psum_part = kb.part + 2 * L.nblocks;   // column 2 of the apply kernels' partial sums
    // out = in - A^m in (+ in_d E) (kinds 0, 2) or b_m - (in - A^m in + in_d E)
    // (kind 1), with the kind's partial sums; A^(m-1) in goes through
    // kb.w1 / kb.w2.  p_ref: subtracted from p in the row's partial sums.
    auto apply = [&](auto kindc, const double* in, double* out, const double* w, double in_d, double p_ref) {
        constexpr int kKind = decltype(kindc)::value;
        const double* src = in;
        for (int j = 1; j < m; ++j) {
            double* dst = (j & 1) ? kb.w1 : kb.w2;
            apply_kernel<3, kAdj><<<L.grid, L.block, 0, st>>>(g, nullptr, src, dst, rho, nullptr, nullptr, nullptr,
                                                               psum_part, L.nblocks, 0.0, border && j == 1, p_ref);
            src = dst;
        }
        apply_kernel<kKind, kAdj><<<L.grid, L.block, 0, st>>>(g, in, src, out, rho, s, m > 1 ? kb.bm : nullptr, w,
                                                              kb.part, L.nblocks, border ? in_d : 0.0,
                                                              border && m == 1, p_ref);
    };
    using K0 = std::integral_constant<int, 0>;
    using K1 = std::integral_constant<int, 1>;
    using K2 = std::integral_constant<int, 2>;
    auto host_sum = [&](long long blocks, int cols, double* out) -> bool {
        if (cudaMemcpyAsync(kb.host, kb.part, static_cast<size_t>(cols) * blocks * sizeof(double),
                            cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return false;
        if (cudaStreamSynchronize(st) != cudaSuccess) return false;
        for (int c = 0; c < cols; ++c) {
            double acc = 0.0;
            for (long long b = 0; b < blocks; ++b) acc += kb.host[c * blocks + b];
            out[c] = acc;
        }
        return true;
    };
    const int ac = border ? 3 : 2;    // columns of an apply's partial sums (kinds 0, 2)
    const int rc = border ? 3 : 1;    // (kind 1)
    double d2[3];
    *res = KrylovResult{};
    if (cudaMemsetAsync(kb.v, 0, static_cast<size_t>(cnt) * sizeof(double), st) != cudaSuccess) return LBM_ERR_CUDA;
    if (m > 1) {
        // b_m = b + A b + ... + A^(m-1) b (b: the kind-1 residual of x = 0)
        apply_kernel<1, kAdj><<<L.grid, L.block, 0, st>>>(g, kb.v, kb.v, kb.bm, rho, s, nullptr, nullptr, kb.part,
                                                          L.nblocks, 0.0, 0, 0.0);
        vec_kernel<3><<<kDotBlocks, 256, 0, st>>>(cnt, 0.0, 0.0, kb.w1, kb.w2, kb.bm, nullptr, nullptr, nullptr,
                                                   nullptr);
        const double* cur = kb.w1;
        for (int j = 1; j < m; ++j) {
            double* dst = (j & 1) ? kb.w2 : kb.w1;
            apply_kernel<3, kAdj><<<L.grid, L.block, 0, st>>>(g, nullptr, cur, dst, rho, nullptr, nullptr, nullptr,
                                                               nullptr, 0, 0.0, 0, 0.0);
            vec_kernel<4><<<kDotBlocks, 256, 0, st>>>(cnt, 0.0, 0.0, kb.bm, nullptr, dst, nullptr, nullptr, nullptr,
                                                       nullptr);
            cur = dst;
        }
        res->matvecs += static_cast<uint64_t>(m - 1);
    }
    // ||b_m||: the residual of x = 0 (v is zero, and stays the v_0 = 0 of the
    // method); the h part only (the row's right-hand side N target is an
    // offset of p, not a size of the problem)
    apply(K1{}, kb.v, kb.t, nullptr, 0.0, 0.0);
    if (!host_sum(L.nblocks, 1, d2)) return LBM_ERR_CUDA;
    // a NaN/Inf source or right-hand side: NaN norms would skip the loop below
    if (!isfinite(d2[0])) return LBM_ERR_NONFINITE;
    // relative to ||b||; a zero source (absolute criterion) still drives the
    // iterate to the null-space representative nearest the start
    const double bnorm = d2[0] > 0.0 ? sqrt(d2[0]) : 1.0;
    // delta parts of the bordered vectors (zero without the walls)
    double xd = 0.0, rd = 0.0, r0d = 0.0, pd = 0.0, vd = 0.0, sd = 0.0, td = 0.0;
    // r = b - A x: the row's residual is sum_x (target - p(h))
    auto residual = [&]() -> bool {
        apply(K1{}, h, kb.r, nullptr, xd, target);
        if (!host_sum(L.nblocks, rc, d2)) return false;
        rd = border ? -d2[2] : 0.0;
        d2[0] += rd * rd;
        return true;
    };
    if (!residual()) return LBM_ERR_CUDA;
    double rr = d2[0];
    if (!isfinite(rr)) return LBM_ERR_NONFINITE;   // a NaN/Inf start iterate
    vec_kernel<3><<<kDotBlocks, 256, 0, st>>>(cnt, 0.0, 0.0, kb.r0, kb.p, kb.r, nullptr, nullptr, nullptr, nullptr);
    r0d = pd = rd;
    res->matvecs += static_cast<uint64_t>(m);
    double rho_old = 1.0, alpha = 1.0, omega = 1.0, rho_new = rr, r0r0 = rr;
    bool first = true, budget = false;
    int since = 0;
    // Restarts whose true residual is not below the best true residual of
    // the earlier starts: a tolerance below
    // the attainable rounding floor would otherwise restart forever when no
    // matvec budget is set.  After kStalledRestarts of them the solve stops
    // with LBM_ERR_POISSON_BUDGET (the iterate is the last one).
    constexpr int kStalledRestarts = 20;
    double best = rr;
    int stalled = 0;
    // Restart from the true residual of the current iterate: r = b - A h,
    // r0 = p = r.
    auto restart = [&]() -> lbm_status {
        if (!residual()) return LBM_ERR_CUDA;
        res->matvecs += static_cast<uint64_t>(m);
        rr = d2[0];
        if (!isfinite(rr)) return LBM_ERR_NONFINITE;
        vec_kernel<3><<<kDotBlocks, 256, 0, st>>>(cnt, 0.0, 0.0, kb.r0, kb.p, kb.r, nullptr, nullptr, nullptr,
                                                   nullptr);
        r0d = pd = rd;
        rho_new = r0r0 = rr;
        rho_old = alpha = omega = 1.0;
        first = true;
        since = 0;
        ++res->restarts;
        res->rel_residual = sqrt(rr) / bnorm;
        if (rr < best) {
            best = rr;
            stalled = 0;
        } else if (++stalled >= kStalledRestarts) {
            budget = true;
        }
        return LBM_OK;
    };
    res->rel_residual = sqrt(rr) / bnorm;
    while (res->rel_residual >= tol) {
        if (max_matvecs && res->matvecs + 3 * static_cast<uint64_t>(m) > max_matvecs) {
            budget = true;
            break;
        }
        // a collapsed recurrence (rho or omega zero: breakdown or stagnation)
        // or 200 iterations since the last start
        if (!first && (rho_old == 0.0 || omega == 0.0 || since >= 200)) {
            const lbm_status rs = restart();
            if (rs != LBM_OK) return rs;
            if (budget) break;
            continue;
        }
        if (!first) {
            const double beta = (rho_new / rho_old) * (alpha / omega);
            vec_kernel<0><<<kDotBlocks, 256, 0, st>>>(cnt, beta, omega, kb.p, nullptr, kb.r, kb.v, nullptr, nullptr,
                                                       nullptr);
            pd = rd + beta * (pd - omega * vd);
        }
        const bool fresh = first;
        first = false;
        apply(K0{}, kb.p, kb.v, kb.r0, pd, 0.0);
        if (!host_sum(L.nblocks, ac, d2)) return LBM_ERR_CUDA;
        if (border) {
            vd = d2[2];
            d2[0] += r0d * vd;
            d2[1] += vd * vd;
        }
        res->matvecs += static_cast<uint64_t>(m);
        if (!isfinite(d2[0]) || !isfinite(d2[1])) return LBM_ERR_NONFINITE;
        // near-breakdown: r0 . v ~ 0 against |r0| |v| (as at the rounding floor)
        if (fabs(d2[0]) <= 1e-12 * sqrt(r0r0 * d2[1])) {
            if (fresh) return LBM_ERR_NONFINITE;   // even a fresh start breaks down
            const lbm_status rs = restart();
            if (rs != LBM_OK) return rs;
            if (budget) break;
            continue;
        }
        alpha = rho_new / d2[0];
        vec_kernel<1><<<kDotBlocks, 256, 0, st>>>(cnt, alpha, 0.0, kb.s, nullptr, kb.r, kb.v, nullptr, nullptr, nullptr);
        sd = rd - alpha * vd;
        apply(K2{}, kb.s, kb.t, kb.s, sd, 0.0);
        if (!host_sum(L.nblocks, ac, d2)) return LBM_ERR_CUDA;
        if (border) {
            td = d2[2];
            d2[0] += sd * td;
            d2[1] += td * td;
        }
        omega = d2[1] > 0.0 ? d2[0] / d2[1] : 0.0;
        vec_kernel<2><<<kDotBlocks, 256, 0, st>>>(cnt, alpha, omega, h, kb.r, kb.p, kb.s, kb.t, kb.r0, kb.part);
        if (!host_sum(kDotBlocks, 2, d2)) return LBM_ERR_CUDA;
        xd += alpha * pd + omega * sd;
        rd = sd - omega * td;
        rr = d2[0] + rd * rd;
        rho_old = rho_new;
        rho_new = d2[1] + r0d * rd;
        res->matvecs += static_cast<uint64_t>(m);
        ++res->iterations;
        ++since;
        if (!isfinite(rr)) return LBM_ERR_NONFINITE;
        res->rel_residual = sqrt(rr) / bnorm;
    }
    *budget_out = budget;
    return LBM_OK;
}

}  // namespace

lbm_status solve(cudaStream_t st, const Launch& L, const Geom& g, const KrylovBuffers& kb, double* h, const double* rho,
                 const double* s, double* p, double* p_prev, double target, double tol, uint64_t max_matvecs,
                 int degree, KrylovResult* res)
{
    bool budget = false;
    const lbm_status it = bicgstab<false>(st, L, g, kb, h, rho, s, target, tol, max_matvecs, degree, res, &budget);
    if (it != LBM_OK) return it;
    // p of the solution, gauged to the target mean (p_prev follows, as after a check)
    pressure_kernel<<<L.grid, L.block, 0, st>>>(g, h, p, kb.part, L.nblocks);
    if (cudaMemcpyAsync(kb.host, kb.part, L.nblocks * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return LBM_ERR_CUDA;
    double sum = 0.0;
    for (long long b = 0; b < L.nblocks; ++b) sum += kb.host[b];
    const double shift = sum / static_cast<double>(g.n) - target;
    if (!isfinite(shift)) return LBM_ERR_NONFINITE;
    shift_kernel<<<kDotBlocks, 256, 0, st>>>(g.n, p, p_prev, shift);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) return LBM_ERR_CUDA;
    res->gauge_shift = shift;
    return budget ? LBM_ERR_POISSON_BUDGET : LBM_OK;
}

lbm_status solve_adjoint(cudaStream_t st, const Launch& L, const Geom& g, const KrylovBuffers& kb, double* y,
                         const double* rho, const double* lp, double tol, uint64_t max_matvecs, KrylovResult* res)
{
    bool budget = false;
    const lbm_status it = bicgstab<true>(st, L, g, kb, y, rho, lp, 0.0, tol, max_matvecs, 1, res, &budget);
    if (it != LBM_OK) return it;
    return budget ? LBM_ERR_POISSON_BUDGET : LBM_OK;
}

}  // namespace krylov
}  // namespace lbm
