// collide_zm.cuh -- the z-marching frame of the collide kernels.
//
// One CTA owns a 32 x 8 column of cells and marches it through a run of z
// planes.  The five macro fields (phi, rho, u, v, w) that the finite-difference
// stencils read are staged plane by plane in a four-slot shared-memory ring
// (34 x 10 cells per plane: the tile and its one-cell halo, x mirrored at the
// slip walls, y and z periodic), filled by cp.async so the copy of plane z+2
// is in flight while plane z is computed, with one barrier per plane.  Every
// stencil neighbour is then a shared-memory read at a constant offset instead
// of a gather from L1/L2; only the 30 population pulls of a cell (into
// registers) and its stores go to global memory.
//
// Ring protocol (plane z of the run, slots indexed by plane & 3):
//   wait for this thread's copies of plane z+1, barrier
//   issue the copies of plane z+2 into slot (z+2) & 3 (= (z-2) & 3, last read
//   while computing plane z-1, which every thread finished before the barrier)
//   compute plane z from slots (z-1) & 3, z & 3, (z+1) & 3.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "lbm_device.cuh"

namespace lbm {

constexpr int ZM_TX = 32, ZM_TY = 8;
constexpr int ZM_THREADS = ZM_TX * ZM_TY;
constexpr int ZM_HX = ZM_TX + 2, ZM_HY = ZM_TY + 2;
constexpr int ZM_PLANE = ZM_HX * ZM_HY;          // 340 halo-region cells
constexpr int ZM_FIELDS = 5;                      // phi, rho, u, v, w
constexpr int ZM_SLOTS = 4;

// Shared memory of the macro ring.
template <class T>
__host__ __device__ constexpr int zm_ring_bytes()
{
    return ZM_SLOTS * ZM_FIELDS * ZM_PLANE * static_cast<int>(sizeof(T));
}

// A box runs through the z-marching collide when the tile divides it and all
// population indices fit 32-bit offsets.
inline bool zm_fits(const Geom& g)
{
    return g.lx % ZM_TX == 0 && g.ly % ZM_TY == 0 && 15LL * g.n < 0x7fffffffLL;
}

__device__ __forceinline__ void cp_async_elem(float* dst, const float* src)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(double* dst, const double* src)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Per-thread part of the ring: the halo-region cells this thread copies
// (region cells tid and tid + 256; the second exists for tid < 84) and their
// in-plane source offsets, fixed for the whole march.
template <class T>
struct MacroRing {
    T* smem;                 // [slot][field][ZM_HY][ZM_HX]
    const T* field[ZM_FIELDS];
    int plane_cells;         // lx * ly
    int lz;
    int r0, r1;              // region cells copied by this thread (r1 < 0: none)
    int o0, o1;              // their in-plane source offsets

    // ctid: this thread's index among the 256 copying threads.
    __device__ __forceinline__ MacroRing(T* s, const Geom& g, int x0, int y0, const T* phi,
                                         const T* rho, const T* u, const T* v, const T* w, int ctid)
        : smem(s), plane_cells(g.lx * g.ly), lz(g.lz)
    {
        field[0] = phi;
        field[1] = rho;
        field[2] = u;
        field[3] = v;
        field[4] = w;
        const int tid = ctid;
        r0 = tid;
        r1 = tid + ZM_THREADS < ZM_PLANE ? tid + ZM_THREADS : -1;
        o0 = offset_of(g, x0, y0, r0);
        o1 = r1 >= 0 ? offset_of(g, x0, y0, r1) : 0;
    }

    // In-plane offset of halo-region cell r: x mirrored at the slip walls
    // (x = -1 -> 1, x = lx -> lx-2; CPU/Inamuro.hpp:230-248) or wrapped when
    // x is periodic, y wrapped.
    static __device__ __forceinline__ int offset_of(const Geom& g, int x0, int y0, int r)
    {
        int x = x0 - 1 + r % ZM_HX;
        int y = y0 - 1 + r / ZM_HX;
        if (g.periodic_x) {
            x = x < 0 ? g.lx - 1 : (x >= g.lx ? 0 : x);
        } else {
            x = x < 0 ? 1 : (x >= g.lx ? g.lx - 2 : x);
        }
        y = y < 0 ? g.ly - 1 : (y >= g.ly ? 0 : y);
        return y * g.lx + x;
    }

    __device__ __forceinline__ T* slot(int plane) const
    {
        return smem + (plane & (ZM_SLOTS - 1)) * (ZM_FIELDS * ZM_PLANE);
    }

    // Issues the copies of plane zp (any integer; wrapped into [0, lz)).
    __device__ __forceinline__ void issue(int zp) const
    {
        int zw = zp % lz;
        if (zw < 0) zw += lz;
        const int base = zw * plane_cells;
        T* s = slot(zp);
#pragma unroll
        for (int f = 0; f < ZM_FIELDS; ++f) {
            cp_async_elem(s + f * ZM_PLANE + r0, field[f] + (base + o0));
            if (r1 >= 0) cp_async_elem(s + f * ZM_PLANE + r1, field[f] + (base + o1));
        }
        cp_async_commit();
    }
};

// firstord + (optionally) secondord of one staged field at the thread's cell,
// neighbours k = 1..14 accumulated in the reference's order
// (CPU/Inamuro.hpp:213-314): grad = sum_k c_k v_k / 10, lap = (sum_k v_k - 14 v) / 5.
// sm, sc, sp: the field's slot for planes z-1, z, z+1; t: the cell's index in a
// plane of the slot.
template <bool kLap, class T>
__device__ __forceinline__ void zm_stencil(const T* sm, const T* sc, const T* sp, int t, T& gx, T& gy,
                                           T& gz, T& lap)
{
    T ax = T(0), ay = T(0), az = T(0), al = T(0);
    static_for<1, Q>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        const T* pl = cz(k) < 0 ? sm : (cz(k) > 0 ? sp : sc);
        const T val = pl[t + cy(k) * ZM_HX + cx(k)];
        ax = acc_signed<cx(k)>(ax, val);
        ay = acc_signed<cy(k)>(ay, val);
        az = acc_signed<cz(k)>(az, val);
        if constexpr (kLap) al = al + val;
    });
    if constexpr (sizeof(T) == 8) {
        gx = ax / T(10);
        gy = ay / T(10);
        gz = az / T(10);
        if constexpr (kLap) lap = (al - T(14) * sc[t]) / T(5);
    } else {
        gx = ax * T(0.1);
        gy = ay * T(0.1);
        gz = az * T(0.1);
        if constexpr (kLap) lap = (al - T(14) * sc[t]) * T(0.2);
    }
}

// The 19 stencil values of a cell and its own macro values.
template <class T>
struct CellDeriv {
    T u_x, u_y, u_z, v_x, v_y, v_z, w_x, w_y, w_z;
    T r_x, r_y, r_z, f_x, f_y, f_z;
    T u_lap, v_lap, w_lap, f_lap;
    T lrho, fei, uu, vv, ww;
};

// c_a c_b (d_b u_a) of direction q: the reference's 9 terms in its order
// (u_x, u_y, u_z, v_x, ..., w_z), zero-coefficient terms dropped at compile
// time and +-1 coefficients applied as add/subtract, the first non-zero term
// starting the sum.
template <int q, class T>
__device__ __forceinline__ T cc_contract(const CellDeriv<T>& d)
{
    constexpr int X = cx(q), Y = cy(q), Z = cz(q);
    T S = T(0);
    bool started = false;
    auto addt = [&](int coef, T val) {
        if (coef == 0) return;
        if (!started) {
            S = coef > 0 ? val : -val;
            started = true;
        } else {
            S = coef > 0 ? S + val : S - val;
        }
    };
    addt(X * X, d.u_x); addt(X * Y, d.u_y); addt(X * Z, d.u_z);
    addt(Y * X, d.v_x); addt(Y * Y, d.v_y); addt(Y * Z, d.v_z);
    addt(Z * X, d.w_x); addt(Z * Y, d.w_y); addt(Z * Z, d.w_z);
    return S;
}

// Stencils of u, v, w and rho (what the g collision needs) and the cell's own
// rho, u, v, w from the ring (field order phi, rho, u, v, w).
template <class T>
__device__ __forceinline__ void zm_derivs_g(const MacroRing<T>& ring, int z, int t, CellDeriv<T>& d)
{
    const T* a = ring.slot(z - 1);
    const T* b = ring.slot(z);
    const T* c = ring.slot(z + 1);
    T unused;
    zm_stencil<true>(a + 2 * ZM_PLANE, b + 2 * ZM_PLANE, c + 2 * ZM_PLANE, t, d.u_x, d.u_y, d.u_z, d.u_lap);
    zm_stencil<true>(a + 3 * ZM_PLANE, b + 3 * ZM_PLANE, c + 3 * ZM_PLANE, t, d.v_x, d.v_y, d.v_z, d.v_lap);
    zm_stencil<true>(a + 4 * ZM_PLANE, b + 4 * ZM_PLANE, c + 4 * ZM_PLANE, t, d.w_x, d.w_y, d.w_z, d.w_lap);
    zm_stencil<false>(a + 1 * ZM_PLANE, b + 1 * ZM_PLANE, c + 1 * ZM_PLANE, t, d.r_x, d.r_y, d.r_z, unused);
    (void)unused;
    d.lrho = b[1 * ZM_PLANE + t];
    d.uu = b[2 * ZM_PLANE + t];
    d.vv = b[3 * ZM_PLANE + t];
    d.ww = b[4 * ZM_PLANE + t];
}

// Stencil of phi (what the f collision needs) and the cell's own phi.
template <class T>
__device__ __forceinline__ void zm_derivs_f(const MacroRing<T>& ring, int z, int t, CellDeriv<T>& d)
{
    zm_stencil<true>(ring.slot(z - 1), ring.slot(z), ring.slot(z + 1), t, d.f_x, d.f_y, d.f_z, d.f_lap);
    d.fei = ring.slot(z)[t];
}

// The cell's own u, v, w from the ring.
template <class T>
__device__ __forceinline__ void zm_velocity(const MacroRing<T>& ring, int z, int t, CellDeriv<T>& d)
{
    const T* b = ring.slot(z);
    d.uu = b[2 * ZM_PLANE + t];
    d.vv = b[3 * ZM_PLANE + t];
    d.ww = b[4 * ZM_PLANE + t];
}

}  // namespace lbm
