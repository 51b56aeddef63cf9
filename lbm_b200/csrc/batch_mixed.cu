// batch_mixed.cu -- batched mixed-precision boxes (include/lbm_b200.h,
// lbm_batch_*): many independent droplet boxes of different sizes and physics
// on one GPU.
//
// Layout: every instance's populations, macro fields and pressures sit in
// pooled buffers at its own offsets (q-major SoA inside each instance, as in
// a single box).  A work list of (instance, xy tile, z run) items covers all
// instances; every phase of a step is ONE launch of a persistent grid
// (ctas_per_sm x SMs CTAs striding over the items), whatever the number of
// instances.  The per-cell arithmetic is the single mixed box's
// (mixed_cells.cuh), so an instance of a batch steps as the same box alone.
//
// Poisson loop: each instance carries its own device state (DevState: source
// mean, gauge, relative change, ...) and control word (BCtl: active flag,
// parity of its current h buffer, sweep cap).  A segment (check_interval
// sweeps, check kernels A and B, the per-instance finalisations) is one
// captured CUDA graph for the whole batch; items of instances that have left
// the loop are skipped, and each instance's h parity advances only while it is
// active.  The segments repeat on the device (a conditional WHILE graph node
// and b_loop_decide) until no instance is active, at most 64 per launch; the
// host reads the control words once per launch and relaunches while any
// instance is still active.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "finalize.cuh"
#include "mixed_cells.cuh"
#include "phys_host.hpp"

namespace lbm {
namespace {

struct BInst {
    Geom g;
    MixPhys M;
    MixMoments mom;
    long long pop;      // element offset of the instance in the pooled population buffers
    long long fld;      // element offset in the pooled macro-field buffers
    int item0, nitems;  // its work items (contiguous)
};

struct BItem {
    int inst;
    int x0, y0, z0, z1;
};

struct BCtl {
    int active;                 // 1 while the instance is in its Poisson loop
    int parity;                 // h buffer holding its current post-collision state
    unsigned long long cap;     // sweep cap (0: none) or the replayed count
    int replay;                 // 1: stop exactly at cap
    int fail_on_limit;          // 1: a cap without convergence is LBM_ERR_POISSON_BUDGET
};

struct BPool {
    float *f[2], *g[2], *h[2];
    double* f0;         // rest populations in FP64 (pooled like the macro fields)
    float *phi, *rho, *u, *v, *w, *div, *s, *omega;
    double *p, *p_prev, *p_chk;
};

// This thread's cell of item w (tile_x x tile_y tile of 256 threads).
__device__ __forceinline__ void item_cell(const BItem& w, int tile_x, int& x, int& y)
{
    x = w.x0 + static_cast<int>(threadIdx.x) % tile_x;
    y = w.y0 + static_cast<int>(threadIdx.x) / tile_x;
}

// Block partial sums of item it (column t at part[t * n_items + it]); the
// trailing barrier lets the CTA reuse the reduction scratch for its next item.
template <int T>
__device__ __forceinline__ void item_sum(double (&red)[T], double* part, int n_items, int it)
{
    block_sum_store<T>(red, part, n_items, it);
    __syncthreads();
}

template <bool kFirst>
__global__ void __launch_bounds__(256)
b_collide(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x,
          const float* __restrict__ fin, float* __restrict__ fout, const float* __restrict__ gin,
          float* __restrict__ gout, BPool B, double* __restrict__ part)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BInst I = inst[w.inst];
        int x, y;
        item_cell(w, tile_x, x, y);
        double red[3] = {0.0, 0.0, 0.0};
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z)
                mixc_collide<kFirst>(I.g, I.M, fin + I.pop, fout + I.pop, B.f0 + I.fld, gin + I.pop, gout + I.pop,
                                     B.phi + I.fld,
                                     B.rho + I.fld, B.u + I.fld, B.v + I.fld, B.w + I.fld, B.div + I.fld, x, y, z,
                                     red);
        item_sum<3>(red, part, n_items, it);
    }
}

__global__ void __launch_bounds__(256)
b_moments(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x,
          const float* __restrict__ f, const float* __restrict__ gp, BPool B, double* __restrict__ part)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BInst I = inst[w.inst];
        int x, y;
        item_cell(w, tile_x, x, y);
        double red[1] = {0.0};
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z)
                mixc_moments(I.g, I.mom, f + I.pop, B.f0 + I.fld, gp + I.pop, B.phi + I.fld, B.rho + I.fld, B.u + I.fld,
                             B.v + I.fld, B.w + I.fld, x, y, z, red);
        item_sum<1>(red, part, n_items, it);
    }
}

__global__ void __launch_bounds__(256)
b_prep(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x,
       const DevState* __restrict__ ds, BPool B, double* __restrict__ part)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BInst I = inst[w.inst];
        const double mean = ds[w.inst].div_mean;
        int x, y;
        item_cell(w, tile_x, x, y);
        double red[3] = {0.0, 0.0, 0.0};
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z)
                mixc_prep(I.g, mean, B.div + I.fld, B.rho + I.fld, B.p + I.fld, B.s + I.fld, B.omega + I.fld, x, y,
                          z, red);
        item_sum<3>(red, part, n_items, it);
    }
}

// h0 and its first collision, into h[0] (each solve starts at parity 0):
// h0 = E_q p (update_hh, CPU/Inamuro.cpp:825-840), or on the first step after
// a load the loaded h, zero (the reference's arrays after initializeArrays),
// staged in h[1].
__global__ void __launch_bounds__(256)
b_init(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x, int h_loaded,
       BPool B)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BInst I = inst[w.inst];
        int x, y;
        item_cell(w, tile_x, x, y);
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z)
                mixc_init(I.g, h_loaded != 0, B.h[1] + I.pop, B.h[0] + I.pop, B.p + I.fld, B.omega + I.fld,
                          B.s + I.fld, x, y, z);
    }
}

// Plain sweep j of the segment for every active instance: state in
// h[(parity + j) & 1].
__global__ void __launch_bounds__(256)
b_sweep(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x,
        const BCtl* __restrict__ ctl, int j, BPool B)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BCtl cw = ctl[w.inst];
        if (!cw.active) continue;
        const BInst I = inst[w.inst];
        const bool odd = ((cw.parity + j) & 1) != 0;
        const float* hin = (odd ? B.h[1] : B.h[0]) + I.pop;
        float* hout = (odd ? B.h[0] : B.h[1]) + I.pop;
        int x, y;
        item_cell(w, tile_x, x, y);
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z)
                mixc_sweep32(I.g, hin, hout, B.omega + I.fld, B.s + I.fld, x, y, z);
    }
}

// Two plain sweeps (flip index j: state in h[(parity + j) & 1], result in the
// other buffer) for every active instance, 16 x 8 tiles with temporal
// blocking (sweep2_run).
constexpr int B2_TX = 16, B2_TY = 8;
constexpr int B2_THREADS = sweep2_threads(B2_TX, B2_TY);   // 192
constexpr int B2_SMEM = sweep2_smem(B2_TX, B2_TY);         // 32,400 B
constexpr int B2_CTAS_PER_SM = 4;

__global__ void __launch_bounds__(B2_THREADS, B2_CTAS_PER_SM)
b_sweep2(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst,
         const BCtl* __restrict__ ctl, int j, BPool B)
{
    extern __shared__ float ring[];
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BCtl cw = ctl[w.inst];
        if (!cw.active) continue;
        const BInst I = inst[w.inst];
        const bool odd = ((cw.parity + j) & 1) != 0;
        const float* hin = (odd ? B.h[1] : B.h[0]) + I.pop;
        float* hout = (odd ? B.h[0] : B.h[1]) + I.pop;
        sweep2_run<B2_TX, B2_TY>(I.g, w.x0, w.y0, w.z0, w.z1, hin, hout, B.omega + I.fld, B.s + I.fld, ring);
        __syncthreads();   // the ring is reused by the CTA's next item
    }
}

__global__ void __launch_bounds__(256)
b_check_a(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x,
          const BCtl* __restrict__ ctl, int j, BPool B, double* __restrict__ part)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BCtl cw = ctl[w.inst];
        if (!cw.active) continue;
        const BInst I = inst[w.inst];
        const bool odd = ((cw.parity + j) & 1) != 0;
        const float* hin = (odd ? B.h[1] : B.h[0]) + I.pop;
        float* hout = (odd ? B.h[0] : B.h[1]) + I.pop;
        int x, y;
        item_cell(w, tile_x, x, y);
        double red[1] = {0.0};
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z) mixc_check_a(I.g, hin, hout, B.p_chk + I.fld, x, y, z, red);
        item_sum<1>(red, part, n_items, it);
    }
}

__global__ void __launch_bounds__(256)
b_check_b(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x,
          const BCtl* __restrict__ ctl, const DevState* __restrict__ ds, int j, BPool B, double* __restrict__ part)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BCtl cw = ctl[w.inst];
        if (!cw.active) continue;
        const BInst I = inst[w.inst];
        const double shift = ds[w.inst].sigma;
        const double tgt = ds[w.inst].target;
        const bool odd = ((cw.parity + j) & 1) != 0;
        const float* hin = (odd ? B.h[1] : B.h[0]) + I.pop;
        float* hout = (odd ? B.h[0] : B.h[1]) + I.pop;
        int x, y;
        item_cell(w, tile_x, x, y);
        double red[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z)
                mixc_check_b<false>(I.g, hin, hout, nullptr, B.p_chk + I.fld, B.p_prev + I.fld, B.p + I.fld,
                                    B.omega + I.fld, B.s + I.fld, shift, tgt, x, y, z, red);
        item_sum<5>(red, part, n_items, it);
    }
}

__global__ void __launch_bounds__(256)
b_correct(const BItem* __restrict__ items, int n_items, const BInst* __restrict__ inst, int tile_x, BPool B)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BItem w = items[it];
        const BInst I = inst[w.inst];
        int x, y;
        item_cell(w, tile_x, x, y);
        if (x < I.g.lx && y < I.g.ly)
            for (int z = w.z0; z < w.z1; ++z)
                mixc_correct(I.g, B.u + I.fld, B.v + I.fld, B.w + I.fld, B.p + I.fld, B.rho + I.fld, x, y, z);
    }
}

// One finalisation of kind `kind` per instance (one CTA each).  FIN_SIGMA and
// FIN_CHECK skip instances outside their Poisson loop (their items wrote no
// partials).  FIN_PREP opens the loop (active, parity 0); FIN_CHECK advances
// the parity by the segment's n_flips buffer swaps and closes the loop on
// convergence, on the replayed count or at the cap.
__global__ void __launch_bounds__(256)
b_finalize(int kind, DevState* __restrict__ ds, BCtl* __restrict__ ctl, const BInst* __restrict__ inst,
           const double* __restrict__ part, long long stride, int n_flips)
{
    const int i = blockIdx.x;
    if ((kind == FIN_SIGMA || kind == FIN_CHECK) && !ctl[i].active) return;
    const BInst I = inst[i];
    finalize_body(kind, ds + i, part + I.item0, stride, I.nitems, nullptr, 0, 0);
    if (threadIdx.x != 0) return;
    if (kind == FIN_PREP) {
        ctl[i].active = 1;
        ctl[i].parity = 0;
    } else if (kind == FIN_CHECK) {
        BCtl& c = ctl[i];
        DevState& d = ds[i];
        c.parity = (c.parity + n_flips) & 1;
        bool done;
        if (c.replay) {
            done = d.iterations >= c.cap;
        } else {
            done = d.converged != 0;
            if (!done && c.cap && d.iterations >= c.cap) {
                done = true;
                if (c.fail_on_limit && d.error == 0) d.error = LBM_ERR_POISSON_BUDGET;
            }
        }
        if (d.error) done = true;
        c.active = done ? 0 : 1;
    }
}

__global__ void b_to_float(const double* __restrict__ src, float* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

__global__ void b_to_double(const float* __restrict__ src, double* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

__global__ void b_fill(float* __restrict__ dst, long long n, float v)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = v;
}

// f0 = phi - phi_G from the loaded phi (or the uniform fill when none is given).
__global__ void b_rest_from_phi(const double* __restrict__ phi, double fill, double* __restrict__ f0, double fei_G,
                                long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        f0[i] = (phi ? phi[i] : fill) - fei_G;
}

thread_local std::string g_batch_create_error;

const char* site_message(int site)
{
    switch (site) {
    case SITE_SOURCE: return "Poisson source contains NaN/Inf";
    case SITE_PROJECTED: return "projected Poisson source contains NaN/Inf";
    case SITE_GAUGE_TARGET: return "pressure mean is NaN/Inf";
    case SITE_GAUGE_SHIFT: return "pressure gauge shift is NaN/Inf";
    case SITE_RESIDUAL: return "Poisson pressure/residual contains NaN/Inf";
    default: return "non-finite value";
    }
}

constexpr int kLoopKey = 1 << 20;           // graph-map key offset of the device-side loop
constexpr unsigned kBatchLoopSegments = 64;   // segments per launch of the device-side loop

// After a segment: continue while any instance is still in its Poisson loop,
// for at most kBatchLoopSegments segments per launch.
__global__ void __launch_bounds__(256)
b_loop_decide(const BCtl* __restrict__ ctl, int n, unsigned* __restrict__ segs, cudaGraphConditionalHandle w)
{
    int any = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) any |= ctl[i].active;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        const unsigned s = ++*segs;
        cudaGraphSetConditional(w, (any && s < kBatchLoopSegments) ? 1u : 0u);
    }
}

}  // namespace
}  // namespace lbm

using namespace lbm;

struct lbm_batch {
    int device = 0;
    int n = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::vector<lbm_params> prm;
    std::vector<BInst> inst_h;
    long long total_cells = 0;
    long long max_cells = 0;
    long long pop_elems = 0;         // elements of one pooled population buffer
    long long item_capacity = 0;     // partial-sum slots allocated (largest work list of any tuning)
    int n_items = 0;
    int n_items2 = 0;                // two-sweep work list (16 x 8 tiles, sweep2_zrun)
    BInst* inst_d = nullptr;
    BItem* items_d = nullptr;
    BItem* items2_d = nullptr;
    DevState* ds = nullptr;
    DevState* ds_host = nullptr;     // pinned, n entries
    BCtl* ctl = nullptr;
    BCtl* ctl_host = nullptr;        // pinned, n entries
    BPool pool{};
    double *part_src = nullptr, *part_mass = nullptr, *part_prep = nullptr, *part_a = nullptr, *part_b = nullptr;
    double* scratch = nullptr;       // FP64 staging of one instance's field
    lbm_poisson_cfg pcfg{100, 1.0e-3, 0, 0, 0};
    lbm_batch_tuning tune{32, 8, 4, 4, 0, 0, 0.0};
    int fcur = 0;
    bool first_step = true;
    std::map<int, cudaGraphExec_t> graphs;    // key: plain sweeps per segment (+ kLoopKey: the loop)
    unsigned* loop_segs = nullptr;            // device-side loop: segments run by a launch, pinned copy
    unsigned* loop_segs_host = nullptr;
    bool loop_ok = true;                      // false once the loop graph failed to build
    cudaEvent_t ev[6]{};
    lbm_timing acc{};
    std::string err;
};

namespace {

lbm_status bfail(lbm_batch* b, lbm_status s, const std::string& msg)
{
    if (b) b->err = msg;
    return s;
}

#define BCUDA(b, call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,   \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

bool valid_tuning(const lbm_batch_tuning& t)
{
    const bool tile = (t.tile_x == 32 && t.tile_y == 8) || (t.tile_x == 16 && t.tile_y == 16) ||
                      (t.tile_x == 8 && t.tile_y == 32);
    return tile && t.zrun >= 1 && t.zrun <= 64 && t.ctas_per_sm >= 1 && t.ctas_per_sm <= 16 &&
           t.sweep2_zrun >= 0 && t.sweep2_zrun <= 64;
}

long long count_items(const std::vector<lbm_params>& prm, int tx, int ty, int zrun)
{
    long long c = 0;
    for (const auto& p : prm)
        c += static_cast<long long>((p.lx + tx - 1) / tx) * ((p.ly + ty - 1) / ty) * ((p.lz + zrun - 1) / zrun);
    return c;
}

// Rebuilds the work list for the batch's tuning (instance-major items).
lbm_status build_items(lbm_batch* b)
{
    const lbm_batch_tuning& t = b->tune;
    std::vector<BItem> items;
    for (int i = 0; i < b->n; ++i) {
        BInst& I = b->inst_h[i];
        I.item0 = static_cast<int>(items.size());
        for (int z0 = 0; z0 < I.g.lz; z0 += t.zrun)
            for (int y0 = 0; y0 < I.g.ly; y0 += t.tile_y)
                for (int x0 = 0; x0 < I.g.lx; x0 += t.tile_x)
                    items.push_back(BItem{i, x0, y0, z0, std::min(z0 + t.zrun, I.g.lz)});
        I.nitems = static_cast<int>(items.size()) - I.item0;
    }
    if (static_cast<long long>(items.size()) > b->item_capacity)
        return bfail(b, LBM_ERR_BAD_ARG, "work list larger than the partial-sum buffers");
    b->n_items = static_cast<int>(items.size());
    if (b->items_d) cudaFree(b->items_d);
    b->items_d = nullptr;
    BCUDA(b, cudaMalloc(&b->items_d, items.size() * sizeof(BItem)));
    BCUDA(b, cudaMemcpy(b->items_d, items.data(), items.size() * sizeof(BItem), cudaMemcpyHostToDevice));
    // the two-sweep list: 16 x 8 tiles, z runs of sweep2_zrun (no partial sums)
    std::vector<BItem> items2;
    if (t.sweep2_zrun > 0)
        for (int i = 0; i < b->n; ++i) {
            const BInst& I = b->inst_h[i];
            for (int z0 = 0; z0 < I.g.lz; z0 += t.sweep2_zrun)
                for (int y0 = 0; y0 < I.g.ly; y0 += B2_TY)
                    for (int x0 = 0; x0 < I.g.lx; x0 += B2_TX)
                        items2.push_back(BItem{i, x0, y0, z0, std::min(z0 + t.sweep2_zrun, I.g.lz)});
        }
    b->n_items2 = static_cast<int>(items2.size());
    if (b->items2_d) cudaFree(b->items2_d);
    b->items2_d = nullptr;
    if (!items2.empty()) {
        BCUDA(b, cudaMalloc(&b->items2_d, items2.size() * sizeof(BItem)));
        BCUDA(b, cudaMemcpy(b->items2_d, items2.data(), items2.size() * sizeof(BItem), cudaMemcpyHostToDevice));
    }
    BCUDA(b, cudaMemcpy(b->inst_d, b->inst_h.data(), b->n * sizeof(BInst), cudaMemcpyHostToDevice));
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    return LBM_OK;
}

int grid_of(const lbm_batch* b)
{
    return std::max(1, std::min(b->n_items, b->tune.ctas_per_sm * b->sm_count));
}

void free_batch(lbm_batch* b)
{
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    float** fl[] = {&b->pool.f[0], &b->pool.f[1], &b->pool.g[0], &b->pool.g[1], &b->pool.h[0], &b->pool.h[1],
                    &b->pool.phi, &b->pool.rho, &b->pool.u, &b->pool.v, &b->pool.w, &b->pool.div, &b->pool.s,
                    &b->pool.omega};
    for (float** p : fl) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    double** db[] = {&b->pool.p, &b->pool.p_prev, &b->pool.p_chk, &b->pool.f0, &b->part_src, &b->part_mass, &b->part_prep,
                     &b->part_a, &b->part_b, &b->scratch};
    for (double** p : db) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (b->inst_d) cudaFree(b->inst_d);
    if (b->items_d) cudaFree(b->items_d);
    if (b->items2_d) cudaFree(b->items2_d);
    b->items2_d = nullptr;
    if (b->ds) cudaFree(b->ds);
    if (b->ctl) cudaFree(b->ctl);
    if (b->ds_host) cudaFreeHost(b->ds_host);
    if (b->ctl_host) cudaFreeHost(b->ctl_host);
    if (b->loop_segs) cudaFree(b->loop_segs);
    if (b->loop_segs_host) cudaFreeHost(b->loop_segs_host);
    b->loop_segs = nullptr;
    b->loop_segs_host = nullptr;
    b->inst_d = nullptr;
    b->items_d = nullptr;
    b->ds = nullptr;
    b->ctl = nullptr;
    b->ds_host = nullptr;
    b->ctl_host = nullptr;
    for (auto& e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    b->stream = nullptr;
}

lbm_status load_instance(lbm_batch* b, int i, const double* const src[6])
{
    cudaStream_t st = b->stream;
    const BInst& I = b->inst_h[i];
    const long long n = I.g.n;
    const lbm_params& p = b->prm[i];
    float* dst[5] = {b->pool.phi + I.fld, b->pool.rho + I.fld, b->pool.u + I.fld, b->pool.v + I.fld,
                     b->pool.w + I.fld};
    const float bg[5] = {(float)p.fei_min, (float)p.rho_G, 0.f, 0.f, 0.f};
    for (int f = 0; f < 5; ++f) {
        if (src[f]) {
            BCUDA(b, cudaMemcpyAsync(b->scratch, src[f], n * sizeof(double), cudaMemcpyHostToDevice, st));
            b_to_float<<<592, 256, 0, st>>>(b->scratch, dst[f], n);
        } else {
            b_fill<<<592, 256, 0, st>>>(dst[f], n, bg[f]);
        }
        // the rest population holds phi - phi_G until the first collision
        if (f == 0) b_rest_from_phi<<<592, 256, 0, st>>>(src[0] ? b->scratch : nullptr, p.fei_min,
                                                         b->pool.f0 + I.fld, I.mom.fei_G, n);
    }
    if (src[5])
        BCUDA(b, cudaMemcpyAsync(b->pool.p + I.fld, src[5], n * sizeof(double), cudaMemcpyHostToDevice, st));
    else
        BCUDA(b, cudaMemsetAsync(b->pool.p + I.fld, 0, n * sizeof(double), st));
    BCUDA(b, cudaMemsetAsync(b->pool.p_prev + I.fld, 0, n * sizeof(double), st));
    BCUDA(b, cudaGetLastError());
    BCUDA(b, cudaStreamSynchronize(st));
    return LBM_OK;
}

// One segment's kernels on st (a capturing stream): n_normal plain sweeps,
// check A, FIN_SIGMA, check B, FIN_CHECK.
void enqueue_segment(lbm_batch* b, int n_normal, cudaStream_t st)
{
    const int grid = grid_of(b);
    const int tx = b->tune.tile_x;
    // j counts buffer swaps: a two-sweep launch swaps once, a single sweep once
    int j = 0;
    int singles = n_normal;
    if (b->n_items2 > 0) {
        const int grid2 = std::max(1, std::min(b->n_items2, B2_CTAS_PER_SM * b->sm_count));
        for (int k = 0; k + 1 < n_normal; k += 2)
            b_sweep2<<<grid2, B2_THREADS, B2_SMEM, st>>>(b->items2_d, b->n_items2, b->inst_d, b->ctl, j++, b->pool);
        singles = n_normal & 1;
    }
    for (int k = 0; k < singles; ++k)
        b_sweep<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->ctl, j++, b->pool);
    b_check_a<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->ctl, j++, b->pool, b->part_a);
    b_finalize<<<b->n, 256, 0, st>>>(FIN_SIGMA, b->ds, b->ctl, b->inst_d, b->part_a, b->n_items, 0);
    b_check_b<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->ctl, b->ds, j++, b->pool, b->part_b);
    b_finalize<<<b->n, 256, 0, st>>>(FIN_CHECK, b->ds, b->ctl, b->inst_d, b->part_b, b->n_items, j);
}

// One segment graph: the segment's kernels and the copy of the control words
// to the host.
lbm_status get_segment(lbm_batch* b, int n_normal, cudaGraphExec_t* out)
{
    auto it = b->graphs.find(n_normal);
    if (it != b->graphs.end()) {
        *out = it->second;
        return LBM_OK;
    }
    cudaStream_t st = b->stream;
    BCUDA(b, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    enqueue_segment(b, n_normal, st);
    cudaMemcpyAsync(b->ctl_host, b->ctl, b->n * sizeof(BCtl), cudaMemcpyDeviceToHost, st);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) return bfail(b, LBM_ERR_CUDA, std::string("segment capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return bfail(b, LBM_ERR_CUDA, std::string("segment instantiate: ") + cudaGetErrorString(ie));
    b->graphs[n_normal] = ex;
    *out = ex;
    return LBM_OK;
}

void fill_batch_stats(const DevState& d, lbm_step_stats* s)
{
    std::memset(s, 0, sizeof(*s));
    const double nan = std::nan("");
    s->iterations = d.iterations;
    s->relative_error = d.rel;
    s->pressure_l1_delta = d.l1_delta;
    s->pressure_l1_norm = d.l1_norm;
    s->fixed_point_h_l1 = nan;
    s->fixed_point_h_scale = nan;
    s->fixed_point_h_relative = nan;
    s->fixed_point_p_l1 = nan;
    s->fixed_point_p_scale = nan;
    s->fixed_point_p_relative = nan;
    s->fixed_point_relative = nan;
    s->source_mean = -d.div_mean / 3.0;
    s->source_abs_mean = d.div_abs_sum / (3.0 * d.n_cells);
    s->projected_source_mean = -d.proj_sum / (3.0 * d.n_cells);
    s->pressure_gauge_target = d.target;
    s->pressure_gauge_max_shift = d.max_shift;
    s->mass = d.mass;
    s->pressure_converged = d.pressure_converged;
    s->converged = d.converged;
}

// One step of every instance.  replay: per-instance sweep counts, or null.
// The device-side loop of segments: a graph whose conditional WHILE node runs
// the segment's kernels and b_loop_decide until no instance is active (or
// kBatchLoopSegments ran), then copies the control words and the segment
// count to the host.  False (and nothing reported) when it cannot be built:
// the host then launches one segment graph at a time.
bool get_loop(lbm_batch* b, int n_normal, cudaGraphExec_t* out)
{
    auto it = b->graphs.find(kLoopKey + n_normal);
    if (it != b->graphs.end()) {
        *out = it->second;
        return true;
    }
    if (!b->loop_segs) {
        if (cudaMalloc(&b->loop_segs, sizeof(unsigned)) != cudaSuccess) {
            b->loop_segs = nullptr;
            return false;
        }
        if (cudaMallocHost(&b->loop_segs_host, sizeof(unsigned)) != cudaSuccess) {
            cudaFree(b->loop_segs);
            b->loop_segs = nullptr;
            b->loop_segs_host = nullptr;
            return false;
        }
    }
    cudaStream_t st = b->stream;
    cudaGraph_t top = nullptr;
    if (cudaGraphCreate(&top, 0) != cudaSuccess) return false;
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaSuccess;
    cudaGraphConditionalHandle hw = 0;
    cudaGraphNode_t wnode = nullptr, c1 = nullptr, c2 = nullptr;
    cudaGraphNodeParams wp{};
    e = cudaGraphConditionalHandleCreate(&hw, top, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        wp.type = cudaGraphNodeTypeConditional;
        wp.conditional.handle = hw;
        wp.conditional.type = cudaGraphCondTypeWhile;
        wp.conditional.size = 1;
        e = cudaGraphAddNode(&wnode, top, nullptr, 0, &wp);
    }
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(st, wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                            cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_segment(b, n_normal, st);
        b_loop_decide<<<1, 256, 0, st>>>(b->ctl, b->n, b->loop_segs, hw);
        cudaGraph_t captured = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(st, &captured);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = ec;
    }
    if (e == cudaSuccess)
        e = cudaGraphAddMemcpyNode1D(&c1, top, &wnode, 1, b->ctl_host, b->ctl, b->n * sizeof(BCtl),
                                     cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaGraphAddMemcpyNode1D(&c2, top, &c1, 1, b->loop_segs_host, b->loop_segs, sizeof(unsigned),
                                     cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, top, 0);
    cudaGraphDestroy(top);
    if (e != cudaSuccess) {
        cudaStreamCaptureStatus cs;
        if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        return false;
    }
    b->graphs[kLoopKey + n_normal] = ex;
    *out = ex;
    return true;
}

lbm_status batch_step_once(lbm_batch* b, const uint64_t* replay, lbm_step_stats* stats)
{
    cudaStream_t st = b->stream;
    const int ci = b->pcfg.check_interval;
    const int grid = grid_of(b);
    const int tx = b->tune.tile_x;
    for (int i = 0; i < b->n; ++i) {
        DevState& d = b->ds_host[i];
        std::memset(&d, 0, sizeof(DevState));
        d.check_interval = ci;
        d.tolerance = b->pcfg.tolerance;
        d.dual = 0;
        d.n_cells = static_cast<double>(b->inst_h[i].g.n);
        BCtl& c = b->ctl_host[i];
        c.active = 0;
        c.parity = 0;
        c.replay = replay ? 1 : 0;
        c.cap = replay ? replay[i] : b->pcfg.max_sweeps;
        c.fail_on_limit = b->pcfg.fail_on_limit;
    }
    BCUDA(b, cudaMemcpyAsync(b->ds, b->ds_host, b->n * sizeof(DevState), cudaMemcpyHostToDevice, st));
    BCUDA(b, cudaMemcpyAsync(b->ctl, b->ctl_host, b->n * sizeof(BCtl), cudaMemcpyHostToDevice, st));
    BCUDA(b, cudaEventRecord(b->ev[0], st));
    const int fin = b->fcur, fout = 1 - b->fcur;
    const bool first = b->first_step;
    if (first)
        b_collide<true><<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->pool.f[fin], b->pool.f[fout],
                                              b->pool.g[fin], b->pool.g[fout], b->pool, b->part_src);
    else
        b_collide<false><<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->pool.f[fin], b->pool.f[fout],
                                               b->pool.g[fin], b->pool.g[fout], b->pool, b->part_src);
    BCUDA(b, cudaEventRecord(b->ev[1], st));
    b_moments<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->pool.f[fout], b->pool.g[fout], b->pool,
                                    b->part_mass);
    BCUDA(b, cudaEventRecord(b->ev[2], st));
    b_finalize<<<b->n, 256, 0, st>>>(FIN_SOURCE, b->ds, b->ctl, b->inst_d, b->part_src, b->n_items, 0);
    b_finalize<<<b->n, 256, 0, st>>>(FIN_MASS, b->ds, b->ctl, b->inst_d, b->part_mass, b->n_items, 0);
    b_prep<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->ds, b->pool, b->part_prep);
    b_finalize<<<b->n, 256, 0, st>>>(FIN_PREP, b->ds, b->ctl, b->inst_d, b->part_prep, b->n_items, 0);
    if (first) BCUDA(b, cudaMemsetAsync(b->pool.h[1], 0, b->pop_elems * sizeof(float), st));
    b_init<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, first ? 1 : 0, b->pool);
    BCUDA(b, cudaGetLastError());
    BCUDA(b, cudaEventRecord(b->ev[3], st));
    b->fcur = fout;
    b->first_step = false;

    cudaGraphExec_t seg = nullptr;
    const lbm_status gs = get_segment(b, ci - 1, &seg);
    if (gs != LBM_OK) return gs;
    uint64_t segments = 0, decides = 0;
    const char* lenv = std::getenv("LBM_POISSON_LOOP");
    cudaGraphExec_t loop = nullptr;
    const bool use_loop = b->loop_ok && !(lenv && lenv[0] == '0') && (b->loop_ok = get_loop(b, ci - 1, &loop));
    for (;;) {
        if (use_loop) {
            *b->loop_segs_host = 0;
            BCUDA(b, cudaMemcpyAsync(b->loop_segs, b->loop_segs_host, sizeof(unsigned), cudaMemcpyHostToDevice, st));
            BCUDA(b, cudaGraphLaunch(loop, st));
            BCUDA(b, cudaStreamSynchronize(st));
            const unsigned ran = *b->loop_segs_host;
            if (ran < 1) return bfail(b, LBM_ERR_CUDA, "device Poisson loop ran no segment");
            segments += ran;
            decides += ran;
        } else {
            BCUDA(b, cudaGraphLaunch(seg, st));
            BCUDA(b, cudaStreamSynchronize(st));
            ++segments;
        }
        bool any = false;
        for (int i = 0; i < b->n; ++i) any = any || b->ctl_host[i].active;
        if (!any) break;
        if (segments > (1ull << 40)) return bfail(b, LBM_ERR_OVERFLOW, "Poisson segment counter overflow");
    }
    BCUDA(b, cudaEventRecord(b->ev[4], st));
    b_correct<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, tx, b->pool);
    BCUDA(b, cudaGetLastError());
    BCUDA(b, cudaEventRecord(b->ev[5], st));
    BCUDA(b, cudaMemcpyAsync(b->ds_host, b->ds, b->n * sizeof(DevState), cudaMemcpyDeviceToHost, st));
    BCUDA(b, cudaStreamSynchronize(st));
    float t[5];
    for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&t[i], b->ev[i], b->ev[i + 1]);
    b->acc.collide_ms += t[0];
    b->acc.moments_ms += t[1];
    b->acc.prep_ms += t[2];
    b->acc.poisson_ms += t[3];
    b->acc.correct_ms += t[4];
    b->acc.steps += 1;
    // per segment: ci - 1 plain sweeps (in pairs when two-sweep passes are on)
    // + check A + check B (together one sweep) + two finalisations; per step:
    // 7 prologue launches and the correction
    b->acc.sweep_kernels += segments * static_cast<uint64_t>(ci + 1);
    const uint64_t plain = b->n_items2 > 0 ? static_cast<uint64_t>((ci - 1) / 2 + (ci - 1) % 2) : ci - 1;
    b->acc.kernel_launches += 8 + segments * (plain + 4) + decides;
    if (b->n_items2 > 0) b->acc.fused_sweeps += segments * static_cast<uint64_t>((ci - 1) / 2 * 2);
    lbm_status status = LBM_OK;
    for (int i = 0; i < b->n; ++i) {
        const DevState& d = b->ds_host[i];
        b->acc.sweeps += d.iterations;
        if (stats) fill_batch_stats(d, stats + i);
        if (d.error && status == LBM_OK) {
            status = static_cast<lbm_status>(d.error);
            b->err = "instance " + std::to_string(i) + ": " +
                     (d.error == LBM_ERR_POISSON_BUDGET ? std::string("Poisson sweep limit reached without convergence")
                                                        : std::string(site_message(d.error_site)));
        }
    }
    return status;
}

}  // namespace

extern "C" {

lbm_status lbm_batch_create(const lbm_params* params, int n_instances, int device, lbm_batch** out)
{
    if (!params || !out || n_instances < 1) return LBM_ERR_BAD_ARG;
    *out = nullptr;
    for (int i = 0; i < n_instances; ++i) {
        const lbm_params& p = params[i];
        if (p.lx < 2 || p.ly < 1 || p.lz < 1 || !(p.rho_L != p.rho_G) || !(p.tauf > 0.0) || !(p.taug > 0.0)) {
            g_batch_create_error = "instance " + std::to_string(i) + ": invalid box or physics";
            return LBM_ERR_BAD_ARG;
        }
        if (15LL * p.lx * p.ly * p.lz >= 0x7fffffffLL) {
            g_batch_create_error = "instance " + std::to_string(i) + ": box too large for a batch";
            return LBM_ERR_BAD_ARG;
        }
    }
    int ndev = 0;
    const cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev <= 0 || device < 0 || device >= ndev) {
        cudaGetLastError();
        g_batch_create_error = std::string("no usable CUDA device: ") + cudaGetErrorString(ce);
        return LBM_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        g_batch_create_error = "device is not sm_100";
        return LBM_ERR_NO_DEVICE;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        g_batch_create_error = "cudaSetDevice failed";
        return LBM_ERR_NO_DEVICE;
    }
    lbm_batch* b = new lbm_batch();
    b->device = device;
    b->n = n_instances;
    b->sm_count = prop.multiProcessorCount;
    b->prm.assign(params, params + n_instances);
    b->inst_h.resize(n_instances);
    long long pop = 0, fld = 0;
    for (int i = 0; i < n_instances; ++i) {
        const lbm_params& p = params[i];
        BInst& I = b->inst_h[i];
        std::memset(&I, 0, sizeof(I));
        I.g.lx = p.lx;
        I.g.ly = p.ly;
        I.g.lz = p.lz;
        I.g.periodic_x = p.periodic_x ? 1 : 0;
        I.g.n = static_cast<long long>(p.lx) * p.ly * p.lz;
        const Phys P = make_phys(p);
        I.M = mix_phys(P);
        I.mom = MixMoments{P.fei_G, P.fei_L, P.rho_G, P.rho_L, P.fei_avg, P.dfei, P.half_drho};
        // Offsets rounded to 64 elements keep every instance's arrays aligned.
        I.pop = pop;
        I.fld = fld;
        pop += (15 * I.g.n + 63) / 64 * 64;
        fld += (I.g.n + 63) / 64 * 64;
        b->max_cells = std::max(b->max_cells, I.g.n);
        b->total_cells += I.g.n;
    }
    b->pop_elems = pop;
    auto bail = [&](lbm_status s) {
        g_batch_create_error = b->err;
        free_batch(b);
        delete b;
        return s;
    };
    const int tiles[3][2] = {{32, 8}, {16, 16}, {8, 32}};
    for (auto& t : tiles) b->item_capacity = std::max(b->item_capacity, count_items(b->prm, t[0], t[1], 1));
    auto okf = [&](float** p, long long count) { return cudaMalloc(p, count * sizeof(float)) == cudaSuccess; };
    auto okd = [&](double** p, long long count) { return cudaMalloc(p, count * sizeof(double)) == cudaSuccess; };
    bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess;
    for (int k = 0; k < 2 && ok; ++k)
        ok = okf(&b->pool.f[k], pop) && okf(&b->pool.g[k], pop) && okf(&b->pool.h[k], pop);
    ok = ok && okf(&b->pool.phi, fld) && okf(&b->pool.rho, fld) && okf(&b->pool.u, fld) && okf(&b->pool.v, fld) &&
         okf(&b->pool.w, fld) && okf(&b->pool.div, fld) && okf(&b->pool.s, fld) && okf(&b->pool.omega, fld);
    ok = ok && okd(&b->pool.p, fld) && okd(&b->pool.p_prev, fld) && okd(&b->pool.p_chk, fld) && okd(&b->pool.f0, fld) &&
         okd(&b->scratch, b->max_cells);
    const long long cap = b->item_capacity;
    ok = ok && okd(&b->part_src, 3 * cap) && okd(&b->part_mass, cap) && okd(&b->part_prep, 3 * cap) &&
         okd(&b->part_a, cap) && okd(&b->part_b, 5 * cap);
    ok = ok && cudaMalloc(&b->inst_d, n_instances * sizeof(BInst)) == cudaSuccess &&
         cudaMalloc(&b->ds, n_instances * sizeof(DevState)) == cudaSuccess &&
         cudaMalloc(&b->ctl, n_instances * sizeof(BCtl)) == cudaSuccess &&
         cudaMallocHost(&b->ds_host, n_instances * sizeof(DevState)) == cudaSuccess &&
         cudaMallocHost(&b->ctl_host, n_instances * sizeof(BCtl)) == cudaSuccess;
    for (auto& e : b->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        b->err = "device allocation failed";
        return bail(LBM_ERR_OOM);
    }
    cudaMemset(b->pool.s, 0, fld * sizeof(float));
    cudaMemset(b->pool.omega, 0, fld * sizeof(float));
    if (const char* e = std::getenv("LBM_BATCH_TUNING")) {
        lbm_batch_tuning t{};
        const int got = std::sscanf(e, "%d,%d,%d,%d,%d", &t.tile_x, &t.tile_y, &t.zrun, &t.ctas_per_sm,
                                    &t.sweep2_zrun);
        if (got >= 4 && valid_tuning(t)) b->tune = t;
    }
    lbm_status s = build_items(b);
    if (s != LBM_OK) return bail(s);
    const double* none[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int i = 0; i < n_instances && s == LBM_OK; ++i) s = load_instance(b, i, none);
    if (s != LBM_OK) return bail(s);
    *out = b;
    return LBM_OK;
}

void lbm_batch_destroy(lbm_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_batch(b);
    delete b;
}

int lbm_batch_size(const lbm_batch* b) { return b ? b->n : 0; }

// A load restarts every instance of the batch from its current macro fields
// (equilibrium populations, h0 = 0), as constructing the reference's class
// from a CPU object does.
lbm_status lbm_batch_load_fields(lbm_batch* b, int inst, const double* phi, const double* rho, const double* u,
                                 const double* v, const double* w, const double* p)
{
    if (!b || inst < 0 || inst >= b->n) return LBM_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    const double* src[6] = {phi, rho, u, v, w, p};
    const lbm_status s = load_instance(b, inst, src);
    if (s == LBM_OK) b->first_step = true;
    return s;
}

lbm_status lbm_batch_set_poisson(lbm_batch* b, const lbm_poisson_cfg* cfg)
{
    if (!b || !cfg) return LBM_ERR_BAD_ARG;
    if (cfg->check_interval < 2 || !(cfg->tolerance > 0.0) || cfg->dual_residual != 0)
        return bfail(b, LBM_ERR_BAD_ARG, "batched boxes: check_interval >= 2, tolerance > 0, no dual residual");
    if (cfg->max_sweeps % static_cast<uint64_t>(cfg->check_interval) != 0)
        return bfail(b, LBM_ERR_BAD_ARG, "max_sweeps must be a multiple of check_interval");
    b->pcfg = *cfg;
    return LBM_OK;
}

lbm_status lbm_batch_step(lbm_batch* b, int n_steps, lbm_step_stats* stats)
{
    if (!b || n_steps < 0) return LBM_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    for (int s = 0; s < n_steps; ++s) {
        const lbm_status st = batch_step_once(b, nullptr, stats ? stats + static_cast<size_t>(s) * b->n : nullptr);
        if (st != LBM_OK) return st;
    }
    return LBM_OK;
}

lbm_status lbm_batch_step_replay(lbm_batch* b, int n_steps, const uint64_t* sweeps, lbm_step_stats* stats)
{
    if (!b || n_steps < 0 || !sweeps) return LBM_ERR_BAD_ARG;
    const uint64_t ci = static_cast<uint64_t>(b->pcfg.check_interval);
    for (long long k = 0; k < static_cast<long long>(n_steps) * b->n; ++k)
        if (sweeps[k] == 0 || sweeps[k] % ci != 0)
            return bfail(b, LBM_ERR_BAD_ARG, "replayed sweep counts must be positive multiples of check_interval");
    cudaSetDevice(b->device);
    for (int s = 0; s < n_steps; ++s) {
        const lbm_status st = batch_step_once(b, sweeps + static_cast<size_t>(s) * b->n,
                                              stats ? stats + static_cast<size_t>(s) * b->n : nullptr);
        if (st != LBM_OK) return st;
    }
    return LBM_OK;
}

lbm_status lbm_batch_download(lbm_batch* b, int inst, lbm_field which, double* host)
{
    if (!b || !host || inst < 0 || inst >= b->n || which < LBM_FIELD_PHI || which > LBM_FIELD_P)
        return LBM_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    cudaStream_t st = b->stream;
    const BInst& I = b->inst_h[inst];
    const long long n = I.g.n;
    if (which == LBM_FIELD_P) {
        BCUDA(b, cudaMemcpyAsync(host, b->pool.p + I.fld, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    } else {
        float* src[5] = {b->pool.phi, b->pool.rho, b->pool.u, b->pool.v, b->pool.w};
        b_to_double<<<592, 256, 0, st>>>(src[which] + I.fld, b->scratch, n);
        BCUDA(b, cudaGetLastError());
        BCUDA(b, cudaMemcpyAsync(host, b->scratch, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    BCUDA(b, cudaStreamSynchronize(st));
    return LBM_OK;
}

lbm_status lbm_batch_set_tuning(lbm_batch* b, const lbm_batch_tuning* t)
{
    if (!b || !t || !valid_tuning(*t)) return LBM_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    b->tune = *t;
    return build_items(b);
}

lbm_status lbm_batch_get_tuning(const lbm_batch* b, lbm_batch_tuning* out)
{
    if (!b || !out) return LBM_ERR_BAD_ARG;
    *out = b->tune;
    return LBM_OK;
}

lbm_status lbm_batch_tune(lbm_batch* b, lbm_batch_tuning* chosen)
{
    if (!b) return LBM_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    cudaStream_t st = b->stream;
    // Every instance active at parity 0: the batched sweep then does the
    // work of a real segment.  h, s and omega are rebuilt at the next step.
    for (int i = 0; i < b->n; ++i) b->ctl_host[i] = BCtl{1, 0, 0, 0, 0};
    BCUDA(b, cudaMemcpyAsync(b->ctl, b->ctl_host, b->n * sizeof(BCtl), cudaMemcpyHostToDevice, st));
    const int tiles[3][2] = {{32, 8}, {16, 16}, {8, 32}};
    const int zruns[4] = {1, 2, 4, 8};
    const int ctas[3] = {2, 4, 8};
    lbm_batch_tuning best = b->tune;
    best.sweep_ms = 1e30;
    const int reps = 6;
    for (auto& tl : tiles)
        for (int zr : zruns)
            for (int cp : ctas) {
                const lbm_batch_tuning t{tl[0], tl[1], zr, cp, 0, 0, 0.0};
                b->tune = t;
                lbm_status s = build_items(b);
                if (s != LBM_OK) return s;
                const int grid = grid_of(b);
                for (int r = 0; r < 2; ++r)
                    b_sweep<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, t.tile_x, b->ctl, r, b->pool);
                BCUDA(b, cudaEventRecord(b->ev[0], st));
                for (int r = 0; r < reps; ++r)
                    b_sweep<<<grid, 256, 0, st>>>(b->items_d, b->n_items, b->inst_d, t.tile_x, b->ctl, r, b->pool);
                BCUDA(b, cudaEventRecord(b->ev[1], st));
                BCUDA(b, cudaGetLastError());
                BCUDA(b, cudaEventSynchronize(b->ev[1]));
                float ms = 0.f;
                cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
                if (ms / reps < best.sweep_ms) {
                    best = t;
                    best.sweep_ms = ms / reps;
                }
            }
    // two sweeps per launch on z runs of 8, 16, 32 (per-sweep time = launch / 2)
    const int zr2[3] = {8, 16, 32};
    for (int zr : zr2) {
        lbm_batch_tuning t = best;
        t.sweep2_zrun = zr;
        t.sweep_ms = 0.0;
        b->tune = t;
        lbm_status s = build_items(b);
        if (s != LBM_OK) return s;
        const int grid2 = std::max(1, std::min(b->n_items2, B2_CTAS_PER_SM * b->sm_count));
        b_sweep2<<<grid2, B2_THREADS, B2_SMEM, st>>>(b->items2_d, b->n_items2, b->inst_d, b->ctl, 0, b->pool);
        BCUDA(b, cudaEventRecord(b->ev[0], st));
        for (int r = 0; r < reps / 2; ++r)
            b_sweep2<<<grid2, B2_THREADS, B2_SMEM, st>>>(b->items2_d, b->n_items2, b->inst_d, b->ctl, r, b->pool);
        BCUDA(b, cudaEventRecord(b->ev[1], st));
        BCUDA(b, cudaGetLastError());
        BCUDA(b, cudaEventSynchronize(b->ev[1]));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
        const double per_sweep = ms / (reps / 2) / 2.0;
        if (per_sweep < best.sweep_ms) {
            best = t;
            best.sweep_ms = per_sweep;
        }
    }
    b->tune = best;
    const lbm_status s = build_items(b);
    if (s != LBM_OK) return s;
    if (chosen) *chosen = best;
    return LBM_OK;
}

lbm_status lbm_batch_get_timing(const lbm_batch* b, lbm_timing* out)
{
    if (!b || !out) return LBM_ERR_BAD_ARG;
    *out = b->acc;
    return LBM_OK;
}

lbm_status lbm_batch_reset_timing(lbm_batch* b)
{
    if (!b) return LBM_ERR_BAD_ARG;
    b->acc = lbm_timing{};
    return LBM_OK;
}

const char* lbm_batch_last_error(const lbm_batch* b)
{
    if (!b) return g_batch_create_error.c_str();
    return b->err.c_str();
}

}  // extern "C"
