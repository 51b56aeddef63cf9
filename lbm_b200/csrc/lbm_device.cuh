// lbm_device.cuh -- compile-time D3Q15 tables and device helpers shared by the
// sm_100a kernels.
//
// The velocity set, weights and slip pairs are those of the reference
// (CPU/common.hpp:3-45, CPU/Inamuro.cpp:592-593).  They are compile-time
// functions so that every per-direction loop is unrolled with the direction as
// a constant: zero components vanish and +-1 components become adds/subtracts
// at compile time, with no constant-memory traffic.
#pragma once

#include <cstdint>
#include <type_traits>
#include <utility>

namespace lbm {

constexpr int Q = 15;

__host__ __device__ constexpr int cx(int q)
{
    return (q == 1 || q == 7 || q == 9 || q == 10 || q == 12) ? 1
         : (q == 4 || q == 8 || q == 11 || q == 13 || q == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int q)
{
    return (q == 2 || q == 7 || q == 8 || q == 10 || q == 13) ? 1
         : (q == 5 || q == 9 || q == 11 || q == 12 || q == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int q)
{
    return (q == 3 || q == 7 || q == 8 || q == 9 || q == 14) ? 1
         : (q == 6 || q == 10 || q == 11 || q == 12 || q == 13) ? -1 : 0;
}
// Weights E_i (2/9, 1/9, 1/72), H_i and F_i (-7/3, 1/3, 1/24).
__host__ __device__ constexpr double wE(int q)
{
    return q == 0 ? 2.0 / 9.0 : (q <= 6 ? 1.0 / 9.0 : 1.0 / 72.0);
}
__host__ __device__ constexpr double wF(int q)
{
    return q == 0 ? -7.0 / 3.0 : (q <= 6 ? 1.0 / 3.0 : 1.0 / 24.0);
}
__host__ __device__ constexpr int csq(int q) { return cx(q) * cx(q) + cy(q) * cy(q) + cz(q) * cz(q); }

// x slip wall (CPU/Inamuro.cpp:589-623): at x = 0 the incoming directions
// (1,7,9,10,12) take the value of their mirror (4,8,14,13,11); at x = lx-1 the
// reverse.  Returns the source direction of q at the left / right wall.
__host__ __device__ constexpr int bounce_left(int q)
{
    return q == 1 ? 4 : q == 7 ? 8 : q == 9 ? 14 : q == 10 ? 13 : q == 12 ? 11 : q;
}
__host__ __device__ constexpr int bounce_right(int q)
{
    return q == 4 ? 1 : q == 8 ? 7 : q == 14 ? 9 : q == 13 ? 10 : q == 11 ? 12 : q;
}

template <int... Is, class F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, F&& f)
{
    (f(std::integral_constant<int, Is>{}), ...);
}
// Calls f(integral_constant<int, B>) ... f(integral_constant<int, E-1>).
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F&& f)
{
    static_for_impl(std::make_integer_sequence<int, E - B>{}, [&](auto i) {
        f(std::integral_constant<int, decltype(i)::value + B>{});
    });
}

// Adds c*v to acc for a compile-time c in {-1, 0, +1}, keeping the reference's
// left-to-right accumulation (acc + v*(+-1) is acc +- v exactly in IEEE; the
// c = 0 term only adds a signed zero and is dropped).
template <int C, class T>
__device__ __forceinline__ T acc_signed(T acc, T v)
{
    if constexpr (C == 1) return acc + v;
    else if constexpr (C == -1) return acc - v;
    else return acc;
}

// (c_x a + c_y b) + c_z c with zero terms dropped: the reference's
// `uc[i]*a + vc[i]*b + wc[i]*c` for a compile-time direction.
template <int A, int B, int Cc, class T>
__device__ __forceinline__ T dot3c(T a, T b, T c)
{
    // The first non-zero term starts the sum (0 + t == t), the rest follow in order.
    if constexpr (A != 0) {
        const T s = (A == 1) ? a : -a;
        return acc_signed<Cc>(acc_signed<B>(s, b), c);
    } else if constexpr (B != 0) {
        const T s = (B == 1) ? b : -b;
        return acc_signed<Cc>(s, c);
    } else if constexpr (Cc != 0) {
        return (Cc == 1) ? c : -c;
    } else {
        return T(0);
    }
}
template <int q, class T>
__device__ __forceinline__ T dotq(T a, T b, T c)
{
    return dot3c<cx(q), cy(q), cz(q)>(a, b, c);
}

// Box geometry.  Cells are x fastest: cell = (z*ly + y)*lx + x.
struct Geom {
    int lx, ly, lz;
    int periodic_x;     // 0: slip walls at x = 0 and lx-1 (reference)
    long long n;        // lx*ly*lz
};

// Periodic neighbours for streaming (all three axes wrap; the walls are an
// overwrite afterwards, as in the reference).
struct Wrap {
    int xm, xp, ym, yp, zm, zp;
    __device__ __forceinline__ Wrap(const Geom& g, int x, int y, int z)
    {
        xm = (x == 0) ? g.lx - 1 : x - 1;
        xp = (x == g.lx - 1) ? 0 : x + 1;
        ym = (y == 0) ? g.ly - 1 : y - 1;
        yp = (y == g.ly - 1) ? 0 : y + 1;
        zm = (z == 0) ? g.lz - 1 : z - 1;
        zp = (z == g.lz - 1) ? 0 : z + 1;
    }
};

// Neighbours for the finite-difference stencils: x mirrored at the walls
// (x+1 -> lx-2 at x = lx-1, x-1 -> 1 at x = 0), y and z periodic
// (CPU/Inamuro.hpp:230-248).
struct Mirror {
    int xm, xp, ym, yp, zm, zp;
    __device__ __forceinline__ Mirror(const Geom& g, int x, int y, int z)
    {
        if (g.periodic_x) {
            xm = (x == 0) ? g.lx - 1 : x - 1;
            xp = (x == g.lx - 1) ? 0 : x + 1;
        } else {
            xm = (x == 0) ? 1 : x - 1;
            xp = (x == g.lx - 1) ? g.lx - 2 : x + 1;
        }
        ym = (y == 0) ? g.ly - 1 : y - 1;
        yp = (y == g.ly - 1) ? 0 : y + 1;
        zm = (z == 0) ? g.lz - 1 : z - 1;
        zp = (z == g.lz - 1) ? 0 : z + 1;
    }
};

template <int D>
__device__ __forceinline__ int pick(int m, int c, int p)
{
    if constexpr (D < 0) return m;
    else if constexpr (D > 0) return p;
    else return c;
}

__device__ __forceinline__ long long cell_of(const Geom& g, int x, int y, int z)
{
    return ((long long)z * g.ly + y) * g.lx + x;
}

// Source cell of direction q for a pull stream into (x, y, z): x - c_q.
template <int q>
__device__ __forceinline__ long long pull_src(const Geom& g, const Wrap& w, int x, int y, int z)
{
    return cell_of(g, pick<-cx(q)>(w.xm, x, w.xp), pick<-cy(q)>(w.ym, y, w.yp),
                   pick<-cz(q)>(w.zm, z, w.zp));
}

template <int D, class T>
__device__ __forceinline__ T pick_t(T m, T c, T p)
{
    if constexpr (D < 0) return m;
    else if constexpr (D > 0) return p;
    else return c;
}

// Pull stream of populations Q0..14 into (x, y, z) with 32-bit offsets: the
// caller guarantees 15 * n < 2^31 (the 64-bit form is pull_src + cell_of).
// Q0 = 1 leaves out the rest population (it does not move).
template <int Q0 = 0, class T>
__device__ __forceinline__ void pull_regs32(T (&v)[Q], const T* __restrict__ src, int n,
                                            const Geom& g, int x, int y, int z)
{
    const Wrap w(g, x, y, z);
    static_for<Q0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const int idx = (pick<-cz(q)>(w.zm, z, w.zp) * g.ly + pick<-cy(q)>(w.ym, y, w.yp)) * g.lx +
                        pick<-cx(q)>(w.xm, x, w.xp);
        v[q] = __ldg(src + static_cast<unsigned>(q * n + idx));
    });
}

// ---- plane ring of the two-sweep passes --------------------------------
// A two-sweep pass marches a tile in z: at iteration z it writes sweep k's
// populations of plane z+1 into a shared-memory ring (before the iteration's
// barrier) and, after the barrier, pulls sweep k+1's populations of plane z
// from it -- population q from plane z - cz(q).  So plane P's population q is
// read at iteration P-1 (cz = -1), P (cz = 0) or P+1 (cz = +1), and a slot may
// be rewritten only after every thread has passed the barrier that follows
// its last read: the three groups of five populations (by cz) need 2, 3 and 4
// plane slots, 45 population planes in all (4 x 15 without the grouping).
__host__ __device__ constexpr int ring_group_slots(int g) { return g + 2; }   // g = cz + 1
__host__ __device__ constexpr int ring_group_base(int g) { return g == 0 ? 0 : (g == 1 ? 10 : 25); }
__host__ __device__ constexpr int ring_planes() { return 45; }   // population planes
// Rank of q among the populations with the same cz.
__host__ __device__ constexpr int ring_rank(int q)
{
    int r = 0;
    for (int k = 0; k < q; ++k) r += (cz(k) == cz(q)) ? 1 : 0;
    return r;
}
// Population plane of (q, plane zz) in the ring.
template <int q>
__device__ __forceinline__ int ring_plane(int zz)
{
    constexpr int gq = cz(q) + 1;
    constexpr int S = ring_group_slots(gq);
    const int slot = ((zz % S) + S) % S;
    return ring_group_base(gq) + slot * 5 + ring_rank(q);
}

// x slip overwrite of pulled populations (CPU/Inamuro.cpp:589-623).
template <class T>
__device__ __forceinline__ void bounce_regs(T (&v)[Q], const Geom& g, int x)
{
    if (g.periodic_x) return;
    if (x == 0) {
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (bounce_left(q) != q) v[q] = v[bounce_left(q)];
        });
    }
    if (x == g.lx - 1) {
        static_for<0, Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            if constexpr (bounce_right(q) != q) v[q] = v[bounce_right(q)];
        });
    }
}

// Transpose of the overwrite for population q at cell x: the adjoint of the
// pulled (not yet overwritten) q, given a(q') = the adjoint of overwritten
// population q' at the same cell.  A population the overwrite discards (the
// incoming ones: c_x = +1 at x = 0, c_x = -1 at x = lx-1) gets 0; the one it
// copies from gains the adjoint of its copy.
template <int q, class A>
__device__ __forceinline__ auto slip_T(const Geom& g, int x, A&& a) -> decltype(a(std::integral_constant<int, q>{}))
{
    using T = decltype(a(std::integral_constant<int, q>{}));
    T v = a(std::integral_constant<int, q>{});
    if (g.periodic_x) return v;
    if constexpr (cx(q) == 1) {
        if (x == 0) return T(0);
        if (x == g.lx - 1) v += a(std::integral_constant<int, bounce_left(q)>{});
    } else if constexpr (cx(q) == -1) {
        if (x == g.lx - 1) return T(0);
        if (x == 0) v += a(std::integral_constant<int, bounce_right(q)>{});
    }
    return v;
}

// Transposed pull: the value the transpose of "pull from x - c_q, then the
// slip overwrite" (the sweeps' stream) sends to population q of cell
// (x, y, z), i.e. slip_T at the neighbour x + c_q of y's populations there.
// I: the offset type (32-bit when 15 n < 2^31).
template <int q, class I, class T>
__device__ __forceinline__ T tpull(const T* __restrict__ y, I n, const Geom& g, const Wrap& w, int x, int yy, int z)
{
    const int xs = pick<cx(q)>(w.xm, x, w.xp);
    const I src = (static_cast<I>(pick<cz(q)>(w.zm, z, w.zp)) * static_cast<I>(g.ly) +
                   static_cast<I>(pick<cy(q)>(w.ym, yy, w.yp))) * static_cast<I>(g.lx) + static_cast<I>(xs);
    return slip_T<q>(g, xs, [&](auto qq) { return __ldg(y + static_cast<I>(decltype(qq)::value) * n + src); });
}

// Stencil neighbour x + c_k.
template <int k>
__device__ __forceinline__ long long stencil_nb(const Geom& g, const Mirror& m, int x, int y, int z)
{
    return cell_of(g, pick<cx(k)>(m.xm, x, m.xp), pick<cy(k)>(m.ym, y, m.yp),
                   pick<cz(k)>(m.zm, z, m.zp));
}

// ---- deterministic block reductions -------------------------------------
// Fixed lane/warp assignment and a fixed tree: the result depends only on the
// launch shape, never on scheduling.
constexpr int kMaxTerms = 6;

template <int T>
__device__ __forceinline__ void block_sum_store(double (&v)[T], double* __restrict__ partials,
                                                long long nblocks, long long blk)
{
    __shared__ double red[32][kMaxTerms];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        double s = v[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp][t] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < T; ++t) {
            double s = lane < nwarps ? red[lane][t] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) partials[(long long)t * nblocks + blk] = s;
        }
    }
}

__device__ __forceinline__ long long block_linear()
{
    return blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
}

}  // namespace lbm
