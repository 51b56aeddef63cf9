// lbm_capi.cu -- the C ABI (include/lbm_b200.h): device buffers, the step
// sequence and the Poisson loop control of one box.
//
// Step sequence (InamuroCUDA::performTimeStepGPU, GPU/InamuroCUDA.cu:2372-2442;
// Inamuro::performTimeStep, CPU/Inamuro.cpp:347-363):
//   collide   fused stencils + collide of f, g (pulling the previous step's
//             post-collision populations) -> f*, g*, u_x, v_y, w_z, sum(div)
//   moments   pull f*, g* + x slip -> phi, rho, u*, sum(phi)
//   prep      source projection s = (u_x - mean) + v_y + w_z, sum(p)
//   Poisson   h* = C(h0, p); then segments of check_interval sweeps, each
//             ending in the device-side convergence test, run by a CUDA
//             graph whose conditional WHILE node repeats them until a
//             one-thread decide kernel stops it (exit, replayed count, sweep
//             cap, error, or 64 segments per launch), then one device->host
//             copy of the solver state
//   correct   u -= grad p / (2 rho)
//
// All scalars that the reference brings to the host between kernels (source
// mean, gauge target, gauge shift, residual norms) are reduced and used on the
// device, and so is the decision to run the next segment; the host reads the
// state once per loop launch.  With a per-check callback (and for the one-pass
// and Krylov forms) the host launches one segment graph at a time instead.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "alloc_set.hpp"
#include "field_stats.cuh"
#include "handle_internal.hpp"
#include "lbm_solver.cuh"
#include "lbm_mixed.cuh"
#include "phys_host.hpp"

using namespace lbm;

namespace {

struct SegKey {
    int start_parity, n_normal, dual;
    int form = 0;   // lbm_poisson_form
    int accel = 0;  // 1: two-grid correction, 2: spatial diagnostics
    int loop = 0;   // 1: the device-side loop of such segments (build_loop)
    bool operator<(const SegKey& o) const
    {
        if (start_parity != o.start_parity) return start_parity < o.start_parity;
        if (n_normal != o.n_normal) return n_normal < o.n_normal;
        if (dual != o.dual) return dual < o.dual;
        if (form != o.form) return form < o.form;
        if (accel != o.accel) return accel < o.accel;
        return loop < o.loop;
    }
};

// Control block of the device-side Poisson loop.  The host writes replay,
// max_sweeps and segs = 0 before each launch; the decide kernel counts the
// segments and stops the loop.
struct LoopCtl {
    unsigned long long replay;       // 0: natural exit; else stop once this many sweeps ran
    unsigned long long max_sweeps;   // 0: no cap
    unsigned int segs;               // segments run in this launch
    unsigned int pad;
};

// Segments one launch of the loop runs at most before the host looks at the
// state again (a bounded launch; at 256^3 FP64 about 4 s of sweeps).
constexpr unsigned kLoopSegments = 64;

// After a segment's convergence test: stop on an error, at the natural exit
// (or the replayed count), at the sweep cap or at the launch's segment cap;
// mode 1 (the first of two parity-alternating segments) drives the IF node of
// the second segment and ends the WHILE loop only when it stops.
__global__ void poisson_loop_decide(const DevState* __restrict__ ds, LoopCtl* __restrict__ ctl,
                                    cudaGraphConditionalHandle w, cudaGraphConditionalHandle second, int mode)
{
    const unsigned long long it = ds->iterations;
    const unsigned segs = ++ctl->segs;
    bool stop = ds->error != 0;
    if (ctl->replay) stop = stop || it >= ctl->replay;
    else stop = stop || ds->converged != 0;
    if (ctl->max_sweeps && it >= ctl->max_sweeps) stop = true;
    if (segs >= kLoopSegments) stop = true;
    if (mode == 1) {
        cudaGraphSetConditional(second, stop ? 0u : 1u);
        if (stop) cudaGraphSetConditional(w, 0u);
    } else {
        cudaGraphSetConditional(w, stop ? 0u : 1u);
    }
}

}  // namespace

struct lbm_handle {
    lbm_params prm{};
    Geom geom{};
    Phys phys{};
    lbm_precision precision = LBM_PRECISION_FP64;
    int device = 0;
    cudaStream_t stream = nullptr;
    Launch L{};
    Fp64Buffers b{};
    MixedBuffers mb{};
    bool dual_allocated = false;
    int fcur = 0;           // f/g buffer holding the current post-collision state
    bool first_step = true;
    bool h_loaded = true;   // h0 of the next solve comes from h[1] (a load), not E p
    lbm_poisson_cfg pcfg{100, 1.0e-3, 0, 0, 0};
    DevState* ds = nullptr;
    DevState* ds_host = nullptr;    // pinned
    std::map<SegKey, std::pair<cudaGraphExec_t, int>> graphs;   // graph, end parity
    std::vector<double> ghost;      // 6 fields x 2 planes x lx*ly
    std::string err;
    bool timing = true;
    cudaEvent_t ev[6]{};
    lbm_timing acc{};
    uint64_t steps_done = 0;
    lbm_check_callback check_cb = nullptr;
    void* check_user = nullptr;
    int fuse_zlen = 0;                   // FP64: >0 runs plain sweeps two per launch
    int collide_zlen = 0;                // FP64: >0 runs the z-marching collide
    double* stats_part = nullptr;        // field-statistics partials
    lbm_field_stats* stats_dev = nullptr;   // 7 results (lbm_diagnostics)
    int h_last = 0;                      // h buffer the last Poisson solve ended in
    int pform = LBM_POISSON_KINETIC;     // lbm_poisson_form
    double scalar_scale = 2.0;           // scalar forms: source scale (reference default 2.0)
    double sor_omega = 0.0;              // red-black form: relaxation (0: from the box size)
    lbm_poisson_accel paccel{1.0, 1.0, 0, 1.0, 0, 0.5, 0, 1.0, 0, 0};   // the reference's accelerator settings
    double* and_r = nullptr;             // Anderson-m1 history: previous residual, previous image (15 n each)
    double* and_i = nullptr;
    double* and_part = nullptr;          // 2 x kAndersonBlocks dot partials, and their pinned copy
    double* and_host = nullptr;
    double* tg_sum = nullptr;            // two-grid / spatial diagnostics: 4^3 block sums of the change
    double* blk_part = nullptr;          // spatial diagnostics: partials of sum |block sum|
    KrylovBuffers kb{};                  // BiCGSTAB work vectors (LBM_POISSON_KRYLOV)
    LoopCtl* loopctl = nullptr;          // device-side Poisson loop: control block, its pinned copy
    LoopCtl* loopctl_host = nullptr;
    bool loop_ok = true;                 // false once a loop graph failed to build (host loop then)
};

namespace {

// Why the calling thread's last lbm_create failed (lbm_last_error(NULL)).
thread_local std::string g_create_error;

lbm_status fail(lbm_handle* h, lbm_status s, const std::string& msg)
{
    if (h) h->err = msg;
    return s;
}

#define LBM_CUDA(h, call)                                                                     \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail((h), e_ == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,    \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

int pick_bx(int lx)
{
    if (const char* e = std::getenv("LBM_TILE_BX")) {
        const int v = std::atoi(e);
        if (v == 16 || v == 32 || v == 64 || v == 128) return v;
    }
    if (lx % 32 == 0 || lx > 48) return 32;
    return 16;
}

void free_all(lbm_handle* h)
{
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second.first);
    h->graphs.clear();
    double** ptrs[] = {&h->b.f[0], &h->b.f[1], &h->b.g[0], &h->b.g[1], &h->b.h[0], &h->b.h[1],
                       &h->b.hc, &h->b.phi, &h->b.rho, &h->b.u, &h->b.v, &h->b.w, &h->b.p,
                       &h->b.p_prev, &h->b.p_chk, &h->b.dux, &h->b.dvy, &h->b.dwz, &h->b.s,
                       &h->b.part_src, &h->b.part_prep, &h->b.part_a, &h->b.part_b,
                       &h->b.part_c, &h->b.part_mass};
    for (double** p : ptrs) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    mixed_free(h->mb);
    double** extra[] = {&h->and_r, &h->and_i, &h->and_part, &h->tg_sum, &h->blk_part};
    for (double** p : extra) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (h->and_host) cudaFreeHost(h->and_host);
    h->and_host = nullptr;
    double** kv[] = {&h->kb.r, &h->kb.r0, &h->kb.p, &h->kb.v, &h->kb.s, &h->kb.t, &h->kb.part,
                     &h->kb.w1, &h->kb.w2, &h->kb.bm};
    for (double** p : kv) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (h->kb.host) cudaFreeHost(h->kb.host);
    h->kb.host = nullptr;
    if (h->stats_part) cudaFree(h->stats_part);
    if (h->stats_dev) cudaFree(h->stats_dev);
    h->stats_part = nullptr;
    h->stats_dev = nullptr;
    if (h->ds) cudaFree(h->ds);
    if (h->ds_host) cudaFreeHost(h->ds_host);
    if (h->loopctl) cudaFree(h->loopctl);
    if (h->loopctl_host) cudaFreeHost(h->loopctl_host);
    h->loopctl = nullptr;
    h->loopctl_host = nullptr;
    h->ds = nullptr;
    h->ds_host = nullptr;
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    h->stream = nullptr;
}

lbm_status alloc_fp64(lbm_handle* h)
{
    const size_t n = static_cast<size_t>(h->geom.n);
    const size_t pop = 15 * n * sizeof(double);
    const size_t fld = n * sizeof(double);
    for (int i = 0; i < 2; ++i) {
        LBM_CUDA(h, cudaMalloc(&h->b.f[i], pop));
        LBM_CUDA(h, cudaMalloc(&h->b.g[i], pop));
        LBM_CUDA(h, cudaMalloc(&h->b.h[i], pop));
    }
    double** flds[] = {&h->b.phi, &h->b.rho, &h->b.u, &h->b.v, &h->b.w, &h->b.p, &h->b.p_prev,
                       &h->b.p_chk, &h->b.dux, &h->b.dvy, &h->b.dwz, &h->b.s};
    for (double** p : flds) {
        LBM_CUDA(h, cudaMalloc(p, fld));
        LBM_CUDA(h, cudaMemset(*p, 0, fld));
    }
    const size_t nb = static_cast<size_t>(h->L.nblocks) * sizeof(double);
    LBM_CUDA(h, cudaMalloc(&h->b.part_src, 3 * nb));
    LBM_CUDA(h, cudaMalloc(&h->b.part_prep, 3 * nb));
    LBM_CUDA(h, cudaMalloc(&h->b.part_a, 1 * nb));
    LBM_CUDA(h, cudaMalloc(&h->b.part_b, 5 * nb));
    LBM_CUDA(h, cudaMalloc(&h->b.part_c, 3 * nb));
    LBM_CUDA(h, cudaMalloc(&h->b.part_mass, 1 * nb));
    LBM_CUDA(h, cudaMemset(h->b.part_c, 0, 3 * nb));
    return LBM_OK;
}

lbm_status ensure_dual_buffer(lbm_handle* h)
{
    if (h->dual_allocated) return LBM_OK;
    const size_t pop = 15 * static_cast<size_t>(h->geom.n) * sizeof(double);
    if (h->precision == LBM_PRECISION_FP64) {
        LBM_CUDA(h, cudaMalloc(&h->b.hc, pop));
    } else {
        const lbm_status st = mixed_alloc_dual(h->mb, h->geom);
        if (st != LBM_OK) return fail(h, st, "cannot allocate the dual-residual buffer");
    }
    h->dual_allocated = true;
    return LBM_OK;
}

void upload_state_config(lbm_handle* h)
{
    h->ds_host->check_interval = h->pcfg.check_interval;
    h->ds_host->tolerance = h->pcfg.tolerance;
    h->ds_host->dual = h->pform == LBM_POISSON_VARCOEF_RB ? 1 : h->pcfg.dual_residual;
    h->ds_host->n_cells = static_cast<double>(h->geom.lx) * h->geom.ly * h->geom.lz;
}

// Enqueues one Poisson segment's kernels on st (a capturing stream): n_normal
// plain sweeps, the check pair (A: stream/bounce/sum at the check sweep, B:
// gauge + relative change + R_p terms + collision of the next sweep), in dual
// mode the shadow sweep C (R_h terms), and the convergence test.  Returns
// the h buffer parity the segment ends on.
int enqueue_segment(lbm_handle* h, const SegKey& key, cudaStream_t st)
{
    int cur = key.start_parity;
    const Geom& g = h->geom;
    const Launch& L = h->L;
    if (key.form == LBM_POISSON_REFINE) {
        cur = mixed_refine_segment(st, h->mb, L, g, key.start_parity, key.n_normal, h->ds);
    } else if (key.form != LBM_POISSON_KINETIC) {
        // Scalar forms: n_normal sweeps, the gauge mean, the check; p ends in b.p.
        Fp64Buffers& b = h->b;
        double* P[2] = {b.p, b.p_chk};
        int pc = 0;
        for (int i = 0; i < key.n_normal; ++i) {
            if (key.form == LBM_POISSON_SCALAR_JACOBI) {
                fp64::scalar_jacobi(st, L, g, P[pc], P[1 - pc], b.rho, b.s, h->scalar_scale);
                pc = 1 - pc;
            } else if (key.form == LBM_POISSON_VARCOEF_RB) {
                fp64::rb_varcoef(st, L, g, b.p, b.rho, b.s, h->sor_omega, h->ds);
            } else {
                fp64::rb_sor(st, L, g, b.p, b.rho, b.s, h->scalar_scale, h->sor_omega, h->ds);
            }
        }
        fp64::p_sum(st, L, g, P[pc], b.part_a);
        finalize(st, FIN_SIGMA, h->ds, b.part_a, L.cnblocks, nullptr, 0, nullptr, 0);
        fp64::scalar_check(st, L, g, P[pc], b.p, b.p_prev, h->ds, b.part_b);
        // the variable-coefficient form's operator residual rides on the
        // fixed-point terms of the check (DevState.dual is 1 for it)
        if (key.form == LBM_POISSON_VARCOEF_RB) fp64::varcoef_residual(st, L, g, b.p, b.rho, b.s, h->ds, b.part_c);
        finalize(st, FIN_CHECK, h->ds, b.part_b, L.cnblocks, b.part_c, L.cnblocks, nullptr, 0);
    } else if (h->precision == LBM_PRECISION_FP64) {
        Fp64Buffers& b = h->b;
        int n_single = key.n_normal;
        if (h->fuse_zlen > 0) {
            for (int i = 0; i + 1 < key.n_normal; i += 2) {
                fp64::sweep2(st, g, h->fuse_zlen, b.h[cur], b.h[1 - cur], b.rho, b.s);
                cur = 1 - cur;
            }
            n_single = key.n_normal & 1;
        }
        for (int i = 0; i < n_single; ++i) {
            fp64::sweep(st, L, g, b.h[cur], b.h[1 - cur], b.rho, b.s);
            cur = 1 - cur;
        }
        fp64::sweep_check_a(st, L, g, b.h[cur], b.h[1 - cur], b.p_chk, b.part_a);
        cur = 1 - cur;
        finalize(st, FIN_SIGMA, h->ds, b.part_a, L.cnblocks, nullptr, 0, nullptr, 0);
        if (key.accel) fp64::twogrid_sums(st, g, b.p_chk, b.p_prev, h->ds, h->tg_sum);
        fp64::sweep_check_b(st, L, g, key.dual != 0, b.h[cur], b.h[1 - cur], b.hc, b.p_chk, b.p_prev, b.p,
                            b.rho, b.s, h->ds, b.part_b);
        cur = 1 - cur;
        if (key.dual) {
            fp64::sweep_check_c(st, L, g, b.h[cur], b.h[1 - cur], b.hc, b.rho, b.s, h->ds, b.part_c);
            cur = 1 - cur;
        }
        finalize(st, FIN_CHECK, h->ds, b.part_b, L.cnblocks, b.part_c, L.cnblocks, nullptr, 0);
        if (key.accel & 2) {
            fp64::block_abs_sum(st, g, h->tg_sum, h->blk_part);
            finalize(st, FIN_BLOCK, h->ds, h->blk_part, fp64::kAndersonBlocks, nullptr, 0, nullptr, 0);
        }
        // Two-grid correction (GPU/InamuroCUDA.cu:2149-2156): h here is the
        // next sweep's post-collision h; adding E_q c to it equals colliding the
        // corrected pre-collision h with the corrected p.
        if (key.accel & 1)
            fp64::twogrid_correct(st, L, g, b.h[cur], b.p, b.p_prev, h->tg_sum, h->paccel.two_grid_strength,
                                  h->ds);
    } else {
        cur = mixed_segment(st, h->mb, L, g, key.start_parity, key.n_normal, key.dual != 0, h->ds);
    }
    return cur;
}

// Captures one segment as a CUDA graph, ending in the state copy to the host.
lbm_status build_segment(lbm_handle* h, const SegKey& key, cudaGraphExec_t* out, int* end_parity)
{
    cudaStream_t st = h->stream;
    LBM_CUDA(h, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int cur = enqueue_segment(h, key, st);
    cudaMemcpyAsync(h->ds_host, h->ds, sizeof(DevState), cudaMemcpyDeviceToHost, st);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) return fail(h, LBM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(h, LBM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    *end_parity = cur;
    return LBM_OK;
}

// Cached segment graph for `key` and the h buffer parity it ends on.
lbm_status get_segment(lbm_handle* h, const SegKey& key, cudaGraphExec_t* out, int* end_parity)
{
    auto it = h->graphs.find(key);
    if (it != h->graphs.end()) {
        *out = it->second.first;
        *end_parity = it->second.second;
        return LBM_OK;
    }
    cudaGraphExec_t ex = nullptr;
    const lbm_status st = build_segment(h, key, &ex, end_parity);
    if (st != LBM_OK) return st;
    h->graphs[key] = {ex, *end_parity};
    *out = ex;
    return LBM_OK;
}

// Captures the device-side loop of the segments `key` describes: a WHILE
// node whose body runs one segment and poisson_loop_decide; when a segment
// ends on the other h buffer, a nested IF node runs the segment from that
// buffer and its decide, so that every body iteration returns to the start
// parity.  After the loop the state and the control block go to the host.
// Returns cudaSuccess or the first error (the caller then keeps the host
// loop); *end_parity: where one segment ends.
cudaError_t build_loop(lbm_handle* h, const SegKey& key, cudaGraphExec_t* out, int* end_parity)
{
    cudaStream_t st = h->stream;
    SegKey k1 = key;
    k1.loop = 0;
    cudaGraphExec_t seg = nullptr;
    int end1 = key.start_parity;
    if (get_segment(h, k1, &seg, &end1) != LBM_OK) return cudaErrorUnknown;
    const bool flip = end1 != key.start_parity;
    cudaGraph_t top = nullptr;
    cudaError_t e = cudaGraphCreate(&top, 0);
    if (e != cudaSuccess) return e;
    auto done = [&](cudaError_t err) {
        cudaGraphDestroy(top);
        return err;
    };
    cudaGraphConditionalHandle hw = 0, hi = 0;
    e = cudaGraphConditionalHandleCreate(&hw, top, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return done(e);
    cudaGraphNodeParams wp{};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hw;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode = nullptr;
    e = cudaGraphAddNode(&wnode, top, nullptr, 0, &wp);
    if (e != cudaSuccess) return done(e);
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    if (flip) {
        e = cudaGraphConditionalHandleCreate(&hi, body, 0, 0);
        if (e != cudaSuccess) return done(e);
    }
    // body: segment + decide
    e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return done(e);
    enqueue_segment(h, k1, st);
    poisson_loop_decide<<<1, 1, 0, st>>>(h->ds, h->loopctl, hw, hi, flip ? 1 : 0);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
    std::vector<cudaGraphNode_t> last;
    if (e == cudaSuccess && deps) last.assign(deps, deps + ndeps);
    cudaGraph_t captured = nullptr;
    cudaError_t ec = cudaStreamEndCapture(st, &captured);
    if (e == cudaSuccess) e = ec;
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return done(e);
    if (flip) {
        if (last.empty()) return done(cudaErrorInvalidValue);
        cudaGraphNodeParams ip{};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = hi;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t inode = nullptr;
        e = cudaGraphAddNode(&inode, body, last.data(), last.size(), &ip);
        if (e != cudaSuccess) return done(e);
        cudaGraph_t ibody = ip.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(st, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return done(e);
        SegKey k2 = k1;
        k2.start_parity = end1;
        const int end2 = enqueue_segment(h, k2, st);
        poisson_loop_decide<<<1, 1, 0, st>>>(h->ds, h->loopctl, hw, hi, 0);
        ec = cudaStreamEndCapture(st, &captured);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = ec;
        if (e == cudaSuccess && end2 != key.start_parity) e = cudaErrorInvalidValue;
        if (e != cudaSuccess) return done(e);
    }
    cudaGraphNode_t c1 = nullptr, c2 = nullptr;
    e = cudaGraphAddMemcpyNode1D(&c1, top, &wnode, 1, h->ds_host, h->ds, sizeof(DevState), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaGraphAddMemcpyNode1D(&c2, top, &c1, 1, h->loopctl_host, h->loopctl, sizeof(LoopCtl),
                                     cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, top, 0);
    *end_parity = end1;
    return done(e);
}

// Cached loop graph for `key` (build_loop); false when it cannot be built.
bool get_loop(lbm_handle* h, const SegKey& key, cudaGraphExec_t* out, int* end_parity)
{
    auto it = h->graphs.find(key);
    if (it != h->graphs.end()) {
        *out = it->second.first;
        *end_parity = it->second.second;
        return true;
    }
    if (!h->loopctl) {
        if (cudaMalloc(&h->loopctl, sizeof(LoopCtl)) != cudaSuccess) {
            h->loopctl = nullptr;
            return false;
        }
        if (cudaMallocHost(&h->loopctl_host, sizeof(LoopCtl)) != cudaSuccess) {
            cudaFree(h->loopctl);
            h->loopctl = nullptr;
            h->loopctl_host = nullptr;
            return false;
        }
    }
    cudaGraphExec_t ex = nullptr;
    if (build_loop(h, key, &ex, end_parity) != cudaSuccess) {
        // leave the stream usable and report nothing: the host loop takes over
        cudaStreamCaptureStatus cs;
        if (cudaStreamIsCapturing(h->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(h->stream, &g);
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        return false;
    }
    h->graphs[key] = {ex, *end_parity};
    *out = ex;
    return true;
}

const char* site_text(int site)
{
    switch (site) {
    case SITE_SOURCE: return "Poisson source contains NaN/Inf";
    case SITE_PROJECTED: return "projected Poisson source contains NaN/Inf";
    case SITE_GAUGE_TARGET: return "pressure mean is NaN/Inf";
    case SITE_GAUGE_SHIFT: return "pressure gauge shift is NaN/Inf";
    case SITE_FIXED_POINT: return "kinetic fixed-point residual contains NaN/Inf";
    case SITE_RESIDUAL: return "Poisson pressure/residual contains NaN/Inf";
    default: return "non-finite value";
    }
}

void fill_stats(const lbm_handle* h, const DevState& d, lbm_step_stats* s)
{
    std::memset(s, 0, sizeof(*s));
    s->iterations = d.iterations;
    s->relative_error = d.rel;
    s->pressure_l1_delta = d.l1_delta;
    s->pressure_l1_norm = d.l1_norm;
    const double nan = std::nan("");
    const bool fp = d.fp_evaluated != 0;
    s->fixed_point_h_l1 = fp ? d.fp_terms[0] : nan;
    s->fixed_point_h_scale = fp ? d.fp_h_scale : nan;
    s->fixed_point_h_relative = fp ? d.fp_h_rel : nan;
    s->fixed_point_p_l1 = fp ? d.fp_terms[3] : nan;
    s->fixed_point_p_scale = fp ? d.fp_p_scale : nan;
    s->fixed_point_p_relative = fp ? d.fp_p_rel : nan;
    s->fixed_point_relative = fp ? d.fp_rel : nan;
    // GPU/InamuroCUDA.cu:1892-1893, 1920
    s->source_mean = -d.div_mean / 3.0;
    s->source_abs_mean = d.div_abs_sum / (3.0 * d.n_cells);
    s->projected_source_mean = -d.proj_sum / (3.0 * d.n_cells);
    s->pressure_gauge_target = d.target;
    s->pressure_gauge_max_shift = d.max_shift;
    s->mass = d.mass;
    s->fixed_point_evaluated = d.fp_evaluated;
    s->pressure_converged = d.pressure_converged;
    s->fixed_point_converged = d.fp_converged;
    s->dual_residual_enabled = h->pcfg.dual_residual == 1;
    s->converged = d.converged;
}

// A buffer set allocated whole or not at all (alloc_set.hpp): kind 0 device
// memory, kind 1 pinned host memory.  On failure no slot changes, so the
// set's "allocated" test (its first pointer) stays false and a retry
// allocates again.
lbm_status alloc_buffers(lbm_handle* h, const AllocSlot* slots, int n, const char* what)
{
    auto alloc = [](int kind, void** p, size_t bytes) {
        return (kind == 0 ? cudaMalloc(p, bytes) : cudaMallocHost(p, bytes)) == cudaSuccess;
    };
    auto release = [](int kind, void* p) {
        if (kind == 0) cudaFree(p);
        else cudaFreeHost(p);
    };
    if (alloc_set(slots, n, alloc, release)) return LBM_OK;
    cudaGetLastError();
    return fail(h, LBM_ERR_OOM, what);
}

lbm_status ensure_accel_buffers(lbm_handle* h)
{
    const size_t pop = 15 * static_cast<size_t>(h->geom.n) * sizeof(double);
    if (h->paccel.anderson_m1 && !h->and_r) {
        const size_t part = 2 * fp64::kAndersonBlocks * sizeof(double);
        const AllocSlot set[] = {{reinterpret_cast<void**>(&h->and_r), pop, 0},
                                 {reinterpret_cast<void**>(&h->and_i), pop, 0},
                                 {reinterpret_cast<void**>(&h->and_part), part, 0},
                                 {reinterpret_cast<void**>(&h->and_host), part, 1}};
        const lbm_status s = alloc_buffers(h, set, 4, "Anderson-m1 buffers: device allocation failed");
        if (s != LBM_OK) return s;
    }
    if ((h->paccel.two_grid || h->paccel.spatial_diagnostics) && !h->tg_sum) {
        int bx, by, bz;
        const int nb = fp64::twogrid_blocks(h->geom, &bx, &by, &bz);
        LBM_CUDA(h, cudaMalloc(&h->tg_sum, static_cast<size_t>(nb) * sizeof(double)));
    }
    if (h->paccel.spatial_diagnostics && !h->blk_part)
        LBM_CUDA(h, cudaMalloc(&h->blk_part, fp64::kAndersonBlocks * sizeof(double)));
    return LBM_OK;
}

// One segment of the one-pass form (check_interval sweeps, the check, the
// two-grid correction after an unconverged check), launched directly: the
// Anderson mixing needs its coefficient on the host every sweep, as in the
// reference (GPU/InamuroCUDA.cu:2199-2275).  h and p start and end in the
// parity-0 buffers (b.h[0], b.p); *has_history: Anderson history of this solve.
lbm_status onepass_segment(lbm_handle* h, bool* has_history, uint64_t* launches)
{
    cudaStream_t st = h->stream;
    const Geom& g = h->geom;
    const Launch& L = h->L;
    Fp64Buffers& b = h->b;
    const lbm_poisson_accel& acc = h->paccel;
    double* H[2] = {b.h[0], b.h[1]};
    double* P[2] = {b.p, b.p_chk};
    int c = 0;
    for (int i = 0; i < h->pcfg.check_interval; ++i) {
        fp64::onepass_sweep(st, L, g, H[c], H[1 - c], P[c], P[1 - c], b.rho, b.s, acc.pressure_relax_scale,
                            acc.fixed_point_relax);
        ++*launches;
        if (acc.anderson_m1) {
            if (!*has_history) {
                fp64::anderson_store(st, g, H[c], H[1 - c], h->and_r, h->and_i);
                *has_history = true;
                ++*launches;
            } else {
                fp64::anderson_dot(st, g, H[c], H[1 - c], h->and_r, h->and_part);
                LBM_CUDA(h, cudaMemcpyAsync(h->and_host, h->and_part, 2 * fp64::kAndersonBlocks * sizeof(double),
                                            cudaMemcpyDeviceToHost, st));
                LBM_CUDA(h, cudaStreamSynchronize(st));
                double num = 0.0, den = 0.0;
                for (int k = 0; k < fp64::kAndersonBlocks; ++k) num += h->and_host[k];
                for (int k = 0; k < fp64::kAndersonBlocks; ++k) den += h->and_host[fp64::kAndersonBlocks + k];
                double alpha = 1.0;
                if (den > 1.0e-300) alpha = -num / den;
                if (!std::isfinite(alpha)) alpha = 1.0;
                alpha = std::max(-acc.anderson_beta_max, std::min(1.0 + acc.anderson_beta_max, alpha));
                fp64::anderson_apply(st, L, g, H[c], H[1 - c], h->and_r, h->and_i, P[1 - c], alpha);
                *launches += 2;
            }
        }
        c = 1 - c;
    }
    fp64::p_sum(st, L, g, P[c], b.part_a);
    finalize(st, FIN_SIGMA, h->ds, b.part_a, L.cnblocks, nullptr, 0, nullptr, 0);
    const bool sums = acc.two_grid || acc.spatial_diagnostics;
    if (sums) fp64::twogrid_sums(st, g, P[c], b.p_prev, h->ds, h->tg_sum);
    fp64::onepass_check(st, L, g, H[c], H[0], P[c], b.p, b.p_prev, h->ds, b.part_b);
    finalize(st, FIN_CHECK, h->ds, b.part_b, L.cnblocks, nullptr, 0, nullptr, 0);
    if (acc.spatial_diagnostics) {
        fp64::block_abs_sum(st, g, h->tg_sum, h->blk_part);
        finalize(st, FIN_BLOCK, h->ds, h->blk_part, fp64::kAndersonBlocks, nullptr, 0, nullptr, 0);
    }
    // after an unconverged check only (the kernel reads the verdict on the device)
    if (acc.two_grid) fp64::twogrid_correct(st, L, g, b.h[0], b.p, b.p_prev, h->tg_sum, acc.two_grid_strength, h->ds);
    LBM_CUDA(h, cudaMemcpyAsync(h->ds_host, h->ds, sizeof(DevState), cudaMemcpyDeviceToHost, st));
    LBM_CUDA(h, cudaStreamSynchronize(st));
    *launches += 4 + (sums ? 1 : 0) + (acc.spatial_diagnostics ? 2 : 0) + (acc.two_grid ? 1 : 0);
    return LBM_OK;
}

lbm_status step_once(lbm_handle* h, uint64_t replay, lbm_step_stats* stats)
{
    cudaStream_t st = h->stream;
    const Geom& g = h->geom;
    const Launch& L = h->L;
    const int ci = h->pcfg.check_interval;
    const int dual = h->pcfg.dual_residual != 0;   // residual kernels run in exit and shadow mode
    const int form = h->pform;
    const lbm_poisson_accel& acc = h->paccel;
    const bool onepass_only = acc.pressure_relax_scale != 1.0 || acc.fixed_point_relax != 1.0 || acc.anderson_m1;
    const bool block_sums = acc.two_grid || acc.spatial_diagnostics;
    if (dual && (form != LBM_POISSON_KINETIC || onepass_only || block_sums || acc.source_aware_init))
        return fail(h, LBM_ERR_BAD_ARG,
                    "fixed-point residual requires the kinetic (split) Poisson form with unit relaxation and "
                    "all accelerators disabled");
    if (form == LBM_POISSON_KRYLOV && replay)
        return fail(h, LBM_ERR_BAD_ARG, "the Krylov form stops on its residual: there is no sweep count to replay");
    if (onepass_only && form != LBM_POISSON_ONEPASS)
        return fail(h, LBM_ERR_BAD_ARG, "relaxation scales and Anderson-m1 need the one-pass Poisson form");
    if (block_sums && form != LBM_POISSON_ONEPASS && form != LBM_POISSON_KINETIC)
        return fail(h, LBM_ERR_BAD_ARG,
                    "two-grid correction and spatial diagnostics need the kinetic or one-pass Poisson form");
    if (form == LBM_POISSON_ONEPASS || block_sums) {
        const lbm_status s = ensure_accel_buffers(h);
        if (s != LBM_OK) return s;
    }
    if (form == LBM_POISSON_KRYLOV && !h->kb.r) {
        const size_t pop = 15 * static_cast<size_t>(g.n) * sizeof(double);
        const size_t parts = 3 * static_cast<size_t>(std::max<long long>(L.nblocks, kKrylovBlocks)) * sizeof(double);
        // kb.r doubles as the set's "allocated" flag: alloc_set stores it
        // only with all the others
        const AllocSlot set[] = {{reinterpret_cast<void**>(&h->kb.r0), pop, 0},
                                 {reinterpret_cast<void**>(&h->kb.p), pop, 0},
                                 {reinterpret_cast<void**>(&h->kb.v), pop, 0},
                                 {reinterpret_cast<void**>(&h->kb.s), pop, 0},
                                 {reinterpret_cast<void**>(&h->kb.t), pop, 0},
                                 {reinterpret_cast<void**>(&h->kb.part), parts, 0},
                                 {reinterpret_cast<void**>(&h->kb.host), parts, 1},
                                 {reinterpret_cast<void**>(&h->kb.r), pop, 0}};
        const lbm_status s = alloc_buffers(h, set, 8, "Krylov work vectors: device allocation failed");
        if (s != LBM_OK) return s;
    }
    if (form == LBM_POISSON_KRYLOV && h->paccel.krylov_degree > 1 && !h->kb.w1) {
        const size_t pop = 15 * static_cast<size_t>(g.n) * sizeof(double);
        const AllocSlot set[] = {{reinterpret_cast<void**>(&h->kb.w2), pop, 0},
                                 {reinterpret_cast<void**>(&h->kb.bm), pop, 0},
                                 {reinterpret_cast<void**>(&h->kb.w1), pop, 0}};
        const lbm_status s = alloc_buffers(h, set, 3, "Krylov polynomial buffers: device allocation failed");
        if (s != LBM_OK) return s;
    }
    if (dual) {
        const lbm_status s = ensure_dual_buffer(h);
        if (s != LBM_OK) return s;
    }
    if (form == LBM_POISSON_REFINE && !h->mb.rr) {
        const lbm_status s = mixed_alloc_refine(h->mb, g);
        if (s != LBM_OK) return fail(h, s, "refinement buffers: device allocation failed");
    }
    // Reset per-solve flags, keep config.
    DevState& dh = *h->ds_host;
    std::memset(&dh, 0, sizeof(DevState));
    upload_state_config(h);
    LBM_CUDA(h, cudaMemcpyAsync(h->ds, h->ds_host, sizeof(DevState), cudaMemcpyHostToDevice, st));
    if (h->timing) LBM_CUDA(h, cudaEventRecord(h->ev[0], st));

    int hcur = 0;
    if (h->precision == LBM_PRECISION_FP64) {
        Fp64Buffers& b = h->b;
        const int fin = h->fcur, fout = 1 - h->fcur;
        const long long src_blocks =
            fp64::collide(st, L, g, h->phys, h->first_step, h->collide_zlen, b.f[fin], b.f[fout], b.g[fin],
                          b.g[fout], b.phi, b.rho, b.u, b.v, b.w, b.dux, b.dvy, b.dwz, b.part_src);
        h->fcur = fout;
        if (h->timing) LBM_CUDA(h, cudaEventRecord(h->ev[1], st));
        fp64::moments(st, L, g, h->phys, b.f[fout], b.g[fout], b.phi, b.rho, b.u, b.v, b.w,
                      b.part_mass);
        if (h->timing) LBM_CUDA(h, cudaEventRecord(h->ev[2], st));
        finalize(st, FIN_SOURCE, h->ds, b.part_src, src_blocks, nullptr, 0, nullptr, 0);
        finalize(st, FIN_MASS, h->ds, b.part_mass, L.nblocks, nullptr, 0, nullptr, 0);
        fp64::prep(st, L, g, h->ds, b.dux, b.dvy, b.dwz, b.p, b.s, b.part_prep);
        finalize(st, FIN_PREP, h->ds, b.part_prep, L.nblocks, nullptr, 0, nullptr, 0);
        if (form == LBM_POISSON_KINETIC || form == LBM_POISSON_KRYLOV) {
            fp64::poisson_init(st, L, g, h->h_loaded, b.h[1], b.h[0], b.p, b.rho, b.s, acc.source_aware_init != 0,
                               acc.source_aware_scale);
        } else if (form == LBM_POISSON_ONEPASS) {
            fp64::onepass_init(st, L, g, h->h_loaded, b.h[1], b.h[0], b.p, b.rho, b.s, acc.source_aware_init != 0,
                               acc.source_aware_scale);
        } else if (form == LBM_POISSON_SCALAR_RB || form == LBM_POISSON_VARCOEF_RB) {
            fp64::scalar_rhs_sum(st, L, g, form == LBM_POISSON_SCALAR_RB ? b.rho : nullptr, b.s, h->scalar_scale,
                                 b.part_a);
            finalize(st, FIN_RHS, h->ds, b.part_a, L.cnblocks, nullptr, 0, nullptr, 0);
        }
    } else {
        const lbm_status s2 = mixed_prologue(st, h->mb, L, g, h->phys, h->first_step, h->fcur,
                                             h->h_loaded, h->ds, h->timing ? h->ev : nullptr);
        if (s2 != LBM_OK) return fail(h, s2, "mixed prologue launch failed");
        h->fcur = 1 - h->fcur;
        if (form == LBM_POISSON_REFINE) mixed_refine_init(st, h->mb, L, g, h->h_loaded);
    }
    LBM_CUDA(h, cudaGetLastError());
    h->first_step = false;
    h->h_loaded = false;
    if (h->timing) LBM_CUDA(h, cudaEventRecord(h->ev[3], st));

    // Poisson segments.
    uint64_t iters = 0;
    bool first_seg = true;
    uint64_t kernels = 0;
    // collide, moments, 2 finalize, prep, finalize, poisson_init (+ correct below)
    uint64_t launches = 7;
    if (form == LBM_POISSON_SCALAR_JACOBI) launches = 6;   // no h initialisation
    if (form == LBM_POISSON_SCALAR_RB || form == LBM_POISSON_VARCOEF_RB)
        launches = 8;   // no h initialisation; right-hand-side mean
    uint64_t fused_sweeps = 0;
    bool anderson_history = false;
    if (form == LBM_POISSON_KRYLOV) {
        // The step's source and gauge target are on the device (FIN_SOURCE, FIN_PREP).
        LBM_CUDA(h, cudaMemcpyAsync(h->ds_host, h->ds, sizeof(DevState), cudaMemcpyDeviceToHost, st));
        LBM_CUDA(h, cudaStreamSynchronize(st));
        if (dh.error) return fail(h, static_cast<lbm_status>(dh.error), site_text(dh.error_site));
        KrylovResult kr;
        Fp64Buffers& b = h->b;
        const lbm_status ks = krylov::solve(st, L, g, h->kb, b.h[0], b.rho, b.s, b.p, b.p_prev, dh.target,
                                            h->pcfg.tolerance, h->pcfg.max_sweeps, h->paccel.krylov_degree, &kr);
        if (ks != LBM_OK && ks != LBM_ERR_POISSON_BUDGET)
            return fail(h, ks, ks == LBM_ERR_NONFINITE ? "Krylov Poisson solve broke down or diverged"
                                                       : "Krylov Poisson solve failed");
        if (ks == LBM_ERR_POISSON_BUDGET && h->pcfg.fail_on_limit)
            return fail(h, LBM_ERR_POISSON_BUDGET, "Poisson sweep limit reached without convergence");
        iters = kr.matvecs;
        kernels = kr.matvecs;
        launches += 4 * kr.iterations + 6;
        dh.iterations = kr.matvecs;
        dh.rel = kr.rel_residual;
        dh.max_shift = std::fabs(kr.gauge_shift);
        dh.pressure_converged = ks == LBM_OK;
        dh.converged = ks == LBM_OK;
        hcur = 0;
        h->h_last = 0;
        if (h->check_cb) {
            lbm_check_record rec{};
            rec.step = h->steps_done + 1;
            rec.iteration = iters;
            rec.relative_error = kr.rel_residual;
            rec.fixed_point_h_l1 = rec.fixed_point_h_scale = rec.fixed_point_h_relative = std::nan("");
            rec.fixed_point_p_l1 = rec.fixed_point_p_scale = rec.fixed_point_p_relative = std::nan("");
            rec.fixed_point_relative = std::nan("");
            rec.block_low_frequency_fraction = std::nan("");
            rec.pressure_converged = rec.converged = dh.converged;
            h->check_cb(h->check_user, &rec);
        }
    }
    for (; form != LBM_POISSON_KRYLOV;) {
        uint64_t nseg = 1;   // segments run by this pass (the device-side loop runs several)
        bool looped = false;
        const int n_normal = form == LBM_POISSON_REFINE ? ci - 1
                             : form != LBM_POISSON_KINETIC ? ci
                                                           : (dual ? (first_seg ? ci - 1 : ci - 2) : ci - 1);
        if (form == LBM_POISSON_ONEPASS) {
            const lbm_status os = onepass_segment(h, &anderson_history, &launches);
            if (os != LBM_OK) return os;
            hcur = 0;
        } else {
            const int accel = (acc.two_grid ? 1 : 0) | (acc.spatial_diagnostics ? 2 : 0);
            SegKey key{hcur, n_normal, dual, form, accel};
            cudaGraphExec_t ex = nullptr;
            int end_parity = hcur;
            // The device-side loop (no host round trip between segments), except
            // with a per-check callback and for the dual form's shorter first
            // segment; LBM_POISSON_LOOP=0 keeps the host loop.
            const char* lenv = std::getenv("LBM_POISSON_LOOP");
            const bool try_loop = h->loop_ok && !h->check_cb && !(lenv && lenv[0] == '0') &&
                                  !(form == LBM_POISSON_KINETIC && dual && first_seg);
            SegKey lk = key;
            lk.loop = 1;
            if (try_loop && get_loop(h, lk, &ex, &end_parity)) {
                h->loopctl_host->replay = replay;
                h->loopctl_host->max_sweeps = h->pcfg.max_sweeps;
                h->loopctl_host->segs = 0;
                LBM_CUDA(h, cudaMemcpyAsync(h->loopctl, h->loopctl_host, sizeof(LoopCtl), cudaMemcpyHostToDevice, st));
                LBM_CUDA(h, cudaGraphLaunch(ex, st));
                LBM_CUDA(h, cudaStreamSynchronize(st));
                nseg = h->loopctl_host->segs;
                looped = true;
                if (nseg < 1) return fail(h, LBM_ERR_CUDA, "device Poisson loop ran no segment");
                if (end_parity != hcur && (nseg & 1)) hcur = end_parity;
            } else {
                if (try_loop) h->loop_ok = false;
                const lbm_status gs = get_segment(h, key, &ex, &end_parity);
                if (gs != LBM_OK) return gs;
                LBM_CUDA(h, cudaGraphLaunch(ex, st));
                LBM_CUDA(h, cudaStreamSynchronize(st));
                hcur = end_parity;
            }
        }
        h->h_last = hcur;
        // sweep-equivalents executed (plain, A, B, C) and actual launches
        // (two plain sweeps per launch where the mixed box fuses them)
        if (looped) launches += nseg;   // the device-side loop's decide kernels
        if (form == LBM_POISSON_ONEPASS) {
            kernels += static_cast<uint64_t>(n_normal);   // launches counted by onepass_segment
        } else if (form == LBM_POISSON_REFINE) {
            // residual + n_normal - 1 corrections (in pairs where the box runs
            // two-sweep passes), checks A and B, two finalisations
            const uint64_t nc = static_cast<uint64_t>(n_normal) - 1;
            const uint64_t pairs = h->mb.fuse_zlen > 0 ? nc / 2 : 0;
            kernels += (static_cast<uint64_t>(n_normal) + 2) * nseg;
            launches += (1 + (nc - 2 * pairs) + pairs + 4) * nseg;
            fused_sweeps += 2 * pairs * nseg;
        } else if (form != LBM_POISSON_KINETIC) {
            // scalar sweeps (red-black: two launches each), p sum, check, 2 finalize
            // (+ the operator residual of the variable-coefficient form)
            const bool rb = form == LBM_POISSON_SCALAR_RB || form == LBM_POISSON_VARCOEF_RB;
            kernels += static_cast<uint64_t>(n_normal) * nseg;
            launches += (static_cast<uint64_t>(n_normal) * (rb ? 2 : 1) + 4 +
                         (form == LBM_POISSON_VARCOEF_RB ? 1 : 0)) * nseg;
        } else {
            kernels += (static_cast<uint64_t>(n_normal) + 2 + (dual ? 1 : 0)) * nseg;
            const bool fused = h->precision == LBM_PRECISION_MIXED ? h->mb.fuse_zlen > 0 : h->fuse_zlen > 0;
            const uint64_t plain_launches = fused ? static_cast<uint64_t>(n_normal / 2 + n_normal % 2)
                                                  : static_cast<uint64_t>(n_normal);
            launches += (plain_launches + 4 + (dual ? 1 : 0)) * nseg;
            if (fused) fused_sweeps += static_cast<uint64_t>(n_normal / 2) * 2 * nseg;
        }
        first_seg = false;
        if (dh.error) {
            return fail(h, static_cast<lbm_status>(dh.error), site_text(dh.error_site));
        }
        if (iters > UINT64_MAX - static_cast<uint64_t>(ci) * nseg)
            return fail(h, LBM_ERR_OVERFLOW, "Poisson iteration counter overflow");
        iters += static_cast<uint64_t>(ci) * nseg;
        if (h->check_cb) {
            lbm_step_stats tmp;
            fill_stats(h, dh, &tmp);
            lbm_check_record rec{};
            rec.step = h->steps_done + 1;
            rec.iteration = iters;
            rec.pressure_l1_delta = tmp.pressure_l1_delta;
            rec.pressure_l1_norm = tmp.pressure_l1_norm;
            rec.relative_error = tmp.relative_error;
            rec.fixed_point_h_l1 = tmp.fixed_point_h_l1;
            rec.fixed_point_h_scale = tmp.fixed_point_h_scale;
            rec.fixed_point_h_relative = tmp.fixed_point_h_relative;
            rec.fixed_point_p_l1 = tmp.fixed_point_p_l1;
            rec.fixed_point_p_scale = tmp.fixed_point_p_scale;
            rec.fixed_point_p_relative = tmp.fixed_point_p_relative;
            rec.fixed_point_relative = tmp.fixed_point_relative;
            rec.fixed_point_evaluated = tmp.fixed_point_evaluated;
            rec.pressure_converged = tmp.pressure_converged;
            rec.fixed_point_converged = tmp.fixed_point_converged;
            rec.dual_residual_enabled = h->pcfg.dual_residual == 1;
            rec.converged = tmp.converged;
            rec.block_low_frequency_fraction = acc.spatial_diagnostics ? dh.block_frac : std::nan("");
            if (block_sums) {
                int bx, by, bz;
                rec.spatial_block_size = 4;
                rec.spatial_block_count = fp64::twogrid_blocks(g, &bx, &by, &bz);
            }
            h->check_cb(h->check_user, &rec);
        }
        if (replay) {
            if (iters >= replay) break;
        } else if (dh.converged) {
            break;
        }
        if (h->pcfg.max_sweeps && iters >= h->pcfg.max_sweeps) {
            if (h->pcfg.fail_on_limit)
                return fail(h, LBM_ERR_POISSON_BUDGET, "Poisson sweep limit reached without convergence");
            break;
        }
    }
    if (form == LBM_POISSON_REFINE) {
        mixed_refine_finish(st, h->mb, g, hcur);   // the FP32 h the rest of the box reads
        ++launches;
    }
    if (h->timing) LBM_CUDA(h, cudaEventRecord(h->ev[4], st));
    if (h->precision == LBM_PRECISION_FP64) {
        fp64::correct(st, L, g, h->b.u, h->b.v, h->b.w, h->b.p, h->b.rho);
    } else {
        mixed_correct(st, h->mb, L, g);
    }
    LBM_CUDA(h, cudaGetLastError());
    if (h->timing) LBM_CUDA(h, cudaEventRecord(h->ev[5], st));
    LBM_CUDA(h, cudaStreamSynchronize(st));
    double dev_ms = 0.0;
    if (h->timing) {
        float t[5];
        for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&t[i], h->ev[i], h->ev[i + 1]);
        h->acc.collide_ms += t[0];
        h->acc.moments_ms += t[1];
        h->acc.prep_ms += t[2];
        h->acc.poisson_ms += t[3];
        h->acc.correct_ms += t[4];
        dev_ms = double(t[0]) + t[1] + t[2] + t[3] + t[4];
    }
    h->acc.steps += 1;
    h->acc.sweeps += iters;
    h->acc.sweep_kernels += kernels;
    h->acc.kernel_launches += launches + 1;
    h->acc.fused_sweeps += fused_sweeps;
    h->steps_done += 1;
    if (stats) {
        fill_stats(h, dh, stats);
        stats->iterations = iters;
        stats->device_ms = dev_ms;
    }
    return LBM_OK;
}

lbm_status check_handle(const lbm_handle* h)
{
    return h ? LBM_OK : LBM_ERR_BAD_ARG;
}

const double* field_ptr(const lbm_handle* h, lbm_field which)
{
    switch (which) {
    case LBM_FIELD_PHI: return h->b.phi;
    case LBM_FIELD_RHO: return h->b.rho;
    case LBM_FIELD_U: return h->b.u;
    case LBM_FIELD_V: return h->b.v;
    case LBM_FIELD_W: return h->b.w;
    case LBM_FIELD_P: return h->b.p;
    }
    return nullptr;
}

lbm_status load_common(lbm_handle* h, const double* const src[6], cudaMemcpyKind kind)
{
    const size_t bytes = static_cast<size_t>(h->geom.n) * sizeof(double);
    cudaStream_t st = h->stream;
    if (h->precision == LBM_PRECISION_FP64) {
        double* dst[6] = {h->b.phi, h->b.rho, h->b.u, h->b.v, h->b.w, h->b.p};
        for (int i = 0; i < 6; ++i) {
            if (src[i]) LBM_CUDA(h, cudaMemcpyAsync(dst[i], src[i], bytes, kind, st));
            else LBM_CUDA(h, cudaMemsetAsync(dst[i], 0, bytes, st));
        }
        LBM_CUDA(h, cudaMemsetAsync(h->b.p_prev, 0, bytes, st));
        // h0 of the first solve: the CPU object's h, all zero after initializeArrays.
        LBM_CUDA(h, cudaMemsetAsync(h->b.h[1], 0, 15 * bytes, st));
    } else {
        const lbm_status s = mixed_load(st, h->mb, h->geom, h->phys, src, kind);
        if (s != LBM_OK) return fail(h, s, "mixed load failed");
    }
    LBM_CUDA(h, cudaStreamSynchronize(st));
    h->first_step = true;
    h->h_loaded = true;
    h->fcur = 0;
    return LBM_OK;
}

void default_ghosts(lbm_handle* h)
{
    // Ghost planes of a fresh CPU Inamuro: rho_G, fei_min, 0 (CPU/Inamuro.cpp:518-524).
    const size_t plane = static_cast<size_t>(h->geom.lx) * h->geom.ly;
    h->ghost.assign(6 * 2 * plane, 0.0);
    std::fill(h->ghost.begin(), h->ghost.begin() + 2 * plane, h->prm.fei_min);          // phi
    std::fill(h->ghost.begin() + 2 * plane, h->ghost.begin() + 4 * plane, h->prm.rho_G);  // rho
}

}  // namespace

namespace lbm {

lbm_status fp64_view(lbm_handle* h, Fp64View* out)
{
    if (check_handle(h) != LBM_OK || !out || h->precision != LBM_PRECISION_FP64) return LBM_ERR_BAD_ARG;
    out->geom = h->geom;
    out->phys = h->phys;
    out->L = h->L;
    out->stream = h->stream;
    out->f = h->b.f[h->fcur];
    out->gpop = h->b.g[h->fcur];
    double* m[6] = {h->b.phi, h->b.rho, h->b.u, h->b.v, h->b.w, h->b.p};
    for (int i = 0; i < 6; ++i) out->macro[i] = m[i];
    out->h_last = h->b.h[h->h_last];
    return LBM_OK;
}

lbm_status fp64_restore(lbm_handle* h, const double* f, const double* gpop, const double* const macro[6])
{
    if (check_handle(h) != LBM_OK || h->precision != LBM_PRECISION_FP64 || !f || !gpop) return LBM_ERR_BAD_ARG;
    const size_t bytes = static_cast<size_t>(h->geom.n) * sizeof(double);
    cudaStream_t st = h->stream;
    LBM_CUDA(h, cudaMemcpyAsync(h->b.f[h->fcur], f, 15 * bytes, cudaMemcpyDeviceToDevice, st));
    LBM_CUDA(h, cudaMemcpyAsync(h->b.g[h->fcur], gpop, 15 * bytes, cudaMemcpyDeviceToDevice, st));
    double* m[6] = {h->b.phi, h->b.rho, h->b.u, h->b.v, h->b.w, h->b.p};
    for (int i = 0; i < 6; ++i) {
        if (!macro[i]) return LBM_ERR_BAD_ARG;
        LBM_CUDA(h, cudaMemcpyAsync(m[i], macro[i], bytes, cudaMemcpyDeviceToDevice, st));
    }
    LBM_CUDA(h, cudaStreamSynchronize(st));
    h->first_step = false;
    h->h_loaded = false;
    return LBM_OK;
}

lbm_status box_info(lbm_handle* h, BoxInfo* out)
{
    if (check_handle(h) != LBM_OK || !out) return LBM_ERR_BAD_ARG;
    out->geom = h->geom;
    out->phys = h->phys;
    out->L = h->L;
    out->stream = h->stream;
    out->precision = h->precision;
    return LBM_OK;
}

size_t box_state_bytes(const lbm_handle* h)
{
    if (h->precision == LBM_PRECISION_FP64) return 36 * static_cast<size_t>(h->geom.n) * sizeof(double);
    return mixed_state_bytes(h->geom);
}

lbm_status box_save_state(lbm_handle* h, void* dst)
{
    if (check_handle(h) != LBM_OK || !dst) return LBM_ERR_BAD_ARG;
    cudaStream_t st = h->stream;
    if (h->precision != LBM_PRECISION_FP64) {
        const lbm_status s = mixed_save_state(st, h->mb, h->geom, h->fcur, dst);
        return s == LBM_OK ? LBM_OK : fail(h, s, "state save failed");
    }
    const size_t n = static_cast<size_t>(h->geom.n);
    const size_t bytes = n * sizeof(double);
    double* d = static_cast<double*>(dst);
    LBM_CUDA(h, cudaMemcpyAsync(d, h->b.f[h->fcur], 15 * bytes, cudaMemcpyDeviceToDevice, st));
    LBM_CUDA(h, cudaMemcpyAsync(d + 15 * n, h->b.g[h->fcur], 15 * bytes, cudaMemcpyDeviceToDevice, st));
    double* m[6] = {h->b.phi, h->b.rho, h->b.u, h->b.v, h->b.w, h->b.p};
    for (int i = 0; i < 6; ++i)
        LBM_CUDA(h, cudaMemcpyAsync(d + (30 + i) * n, m[i], bytes, cudaMemcpyDeviceToDevice, st));
    return LBM_OK;
}

lbm_status box_restore_state(lbm_handle* h, const void* src)
{
    if (check_handle(h) != LBM_OK || !src) return LBM_ERR_BAD_ARG;
    if (h->precision == LBM_PRECISION_FP64) {
        const size_t n = static_cast<size_t>(h->geom.n);
        const double* d = static_cast<const double*>(src);
        const double* m[6];
        for (int i = 0; i < 6; ++i) m[i] = d + (30 + i) * n;
        return fp64_restore(h, d, d + 15 * n, m);
    }
    const lbm_status s = mixed_restore_state(h->stream, h->mb, h->geom, h->fcur, src);
    if (s != LBM_OK) return fail(h, s, "state restore failed");
    LBM_CUDA(h, cudaStreamSynchronize(h->stream));
    h->first_step = false;
    h->h_loaded = false;
    return LBM_OK;
}

lbm_status box_export(lbm_handle* h, double* macro6, double* h15)
{
    if (check_handle(h) != LBM_OK || !macro6) return LBM_ERR_BAD_ARG;
    cudaStream_t st = h->stream;
    const size_t n = static_cast<size_t>(h->geom.n);
    if (h->precision != LBM_PRECISION_FP64) {
        const lbm_status s = mixed_export(st, h->mb, h->geom, h->h_last, macro6, h15);
        return s == LBM_OK ? LBM_OK : fail(h, s, "state export failed");
    }
    double* m[6] = {h->b.phi, h->b.rho, h->b.u, h->b.v, h->b.w, h->b.p};
    for (int i = 0; i < 6; ++i)
        LBM_CUDA(h, cudaMemcpyAsync(macro6 + i * n, m[i], n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (h15)
        LBM_CUDA(h, cudaMemcpyAsync(h15, h->b.h[h->h_last], 15 * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return LBM_OK;
}

}  // namespace lbm

extern "C" {

int lbm_abi_version(void) { return LBM_B200_ABI_VERSION; }

const char* lbm_status_string(lbm_status s)
{
    switch (s) {
    case LBM_OK: return "ok";
    case LBM_ERR_CUDA: return "CUDA error";
    case LBM_ERR_NONFINITE: return "non-finite value";
    case LBM_ERR_POISSON_BUDGET: return "Poisson sweep limit reached";
    case LBM_ERR_BAD_ARG: return "bad argument";
    case LBM_ERR_OOM: return "out of device memory";
    case LBM_ERR_IO: return "I/O error";
    case LBM_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case LBM_ERR_OVERFLOW: return "counter overflow";
    }
    return "unknown status";
}

const char* lbm_last_error(const lbm_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

lbm_status lbm_create(const lbm_params* prm, lbm_precision precision, int device, lbm_handle** out)
{
    if (!prm || !out) return LBM_ERR_BAD_ARG;
    *out = nullptr;
    if (prm->lx < 2 || prm->ly < 1 || prm->lz < 1 || prm->lz > 65535) return LBM_ERR_BAD_ARG;
    if (!(prm->rho_L != prm->rho_G) || !(prm->tauf > 0.0) || !(prm->taug > 0.0)) return LBM_ERR_BAD_ARG;
    if (precision != LBM_PRECISION_FP64 && precision != LBM_PRECISION_MIXED) return LBM_ERR_BAD_ARG;
    int ndev = 0;
    const cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev <= 0 || device < 0 || device >= ndev) {
        cudaGetLastError();
        g_create_error = std::string("no usable CUDA device: cudaGetDeviceCount -> ") + cudaGetErrorString(ce) +
                         ", " + std::to_string(ndev) + " device(s), requested " + std::to_string(device);
        return LBM_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop{};
    const cudaError_t pe = cudaGetDeviceProperties(&prop, device);
    if (pe != cudaSuccess || prop.major != 10) {
        g_create_error = std::string("device ") + std::to_string(device) + " is not sm_100 (" +
                         (pe == cudaSuccess ? std::string(prop.name) + ", sm_" + std::to_string(prop.major) +
                                                  std::to_string(prop.minor)
                                            : std::string(cudaGetErrorString(pe))) + ")";
        return LBM_ERR_NO_DEVICE;
    }
    const cudaError_t se = cudaSetDevice(device);
    if (se != cudaSuccess) {
        g_create_error = std::string("cudaSetDevice: ") + cudaGetErrorString(se);
        return LBM_ERR_NO_DEVICE;
    }

    lbm_handle* h = new lbm_handle();
    h->prm = *prm;
    h->precision = precision;
    h->device = device;
    h->geom.lx = prm->lx;
    h->geom.ly = prm->ly;
    h->geom.lz = prm->lz;
    h->geom.periodic_x = prm->periodic_x ? 1 : 0;
    h->geom.n = static_cast<long long>(prm->lx) * prm->ly * prm->lz;
    h->phys = make_phys(*prm);
    const int bx = pick_bx(prm->lx);
    h->L = make_launch(prm->lx, prm->ly, prm->lz, bx, 256 / bx);
    lbm_status st = LBM_OK;
    auto bail = [&](lbm_status s) {
        free_all(h);
        delete h;
        return s;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(LBM_ERR_CUDA);
    for (auto& e : h->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(LBM_ERR_CUDA);
    if (cudaMalloc(&h->ds, sizeof(DevState)) != cudaSuccess) return bail(LBM_ERR_OOM);
    if (cudaMallocHost(&h->ds_host, sizeof(DevState)) != cudaSuccess) return bail(LBM_ERR_OOM);
    if (cudaMalloc(&h->stats_part, sizeof(double) * kStatsTerms * stats_blocks(h->geom.n)) != cudaSuccess ||
        cudaMalloc(&h->stats_dev, 7 * sizeof(lbm_field_stats)) != cudaSuccess)
        return bail(LBM_ERR_OOM);
    std::memset(h->ds_host, 0, sizeof(DevState));
    if (precision == LBM_PRECISION_FP64) st = alloc_fp64(h);
    else st = mixed_alloc(h->mb, h->geom, h->L);
    if (st != LBM_OK) return bail(st);
    if (precision == LBM_PRECISION_FP64) {
        // Two-sweep temporal blocking where the tile divides the box; the z
        // run length can be tuned (0 disables) through LBM_SWEEP2_ZLEN.
        const char* env = std::getenv("LBM_SWEEP2_ZLEN");
        const int zlen = env ? std::atoi(env) : 0;
        h->fuse_zlen = (zlen > 0 && fp64::sweep2_prepare(h->geom)) ? zlen : 0;
        // z-marching collide where its tile divides the box (LBM_COLLIDE_ZLEN,
        // 0 disables).
        const char* cenv = std::getenv("LBM_COLLIDE_ZLEN");
        const int czlen = cenv ? std::atoi(cenv) : 16;
        h->collide_zlen = (czlen > 0 && fp64::collide_zm_prepare(h->geom)) ? czlen : 0;
    }
    default_ghosts(h);
    // Background state until the caller loads fields.
    const size_t n = static_cast<size_t>(h->geom.n);
    std::vector<double> phi(n), rho(n), z(n, 0.0);
    std::fill(phi.begin(), phi.end(), prm->fei_min);
    std::fill(rho.begin(), rho.end(), prm->rho_G);
    const double* src[6] = {phi.data(), rho.data(), z.data(), z.data(), z.data(), z.data()};
    st = load_common(h, src, cudaMemcpyHostToDevice);
    if (st != LBM_OK) return bail(st);
    *out = h;
    return LBM_OK;
}

void lbm_destroy(lbm_handle* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
}

lbm_status lbm_load_fields(lbm_handle* h, const double* phi, const double* rho, const double* u,
                           const double* v, const double* w, const double* p)
{
    if (check_handle(h) != LBM_OK || !phi || !rho || !u || !v || !w) return fail(h, LBM_ERR_BAD_ARG, "null field");
    cudaSetDevice(h->device);
    const double* src[6] = {phi, rho, u, v, w, p};
    default_ghosts(h);
    return load_common(h, src, cudaMemcpyHostToDevice);
}

lbm_status lbm_load_fields_device(lbm_handle* h, const double* phi, const double* rho,
                                  const double* u, const double* v, const double* w, const double* p)
{
    if (check_handle(h) != LBM_OK || !phi || !rho || !u || !v || !w) return fail(h, LBM_ERR_BAD_ARG, "null field");
    cudaSetDevice(h->device);
    const double* src[6] = {phi, rho, u, v, w, p};
    return load_common(h, src, cudaMemcpyDeviceToDevice);
}

lbm_status lbm_load_fields_ghosted(lbm_handle* h, const double* phi, const double* rho,
                                   const double* u, const double* v, const double* w,
                                   const double* p)
{
    if (check_handle(h) != LBM_OK || !phi || !rho || !u || !v || !w || !p) return fail(h, LBM_ERR_BAD_ARG, "null field");
    cudaSetDevice(h->device);
    const size_t plane = static_cast<size_t>(h->geom.lx) * h->geom.ly;
    const size_t n = static_cast<size_t>(h->geom.n);
    const double* gsrc[6] = {phi, rho, u, v, w, p};
    std::vector<double> phys(6 * n);
    h->ghost.assign(6 * 2 * plane, 0.0);
    for (int f = 0; f < 6; ++f) {
        std::memcpy(phys.data() + f * n, gsrc[f] + plane, n * sizeof(double));
        std::memcpy(h->ghost.data() + (2 * f) * plane, gsrc[f], plane * sizeof(double));
        std::memcpy(h->ghost.data() + (2 * f + 1) * plane, gsrc[f] + (h->geom.lz + 1) * plane,
                    plane * sizeof(double));
    }
    const double* src[6] = {phys.data(), phys.data() + n, phys.data() + 2 * n,
                            phys.data() + 3 * n, phys.data() + 4 * n, phys.data() + 5 * n};
    return load_common(h, src, cudaMemcpyHostToDevice);
}

lbm_status lbm_set_poisson(lbm_handle* h, const lbm_poisson_cfg* cfg)
{
    if (check_handle(h) != LBM_OK || !cfg) return fail(h, LBM_ERR_BAD_ARG, "null config");
    // Same validation as InamuroCUDA::setPoissonConvergence / setPoissonIterationLimit
    // (GPU/InamuroCUDA.cu:2582-2608); the dual test needs >= 2 sweeps per segment.
    if (cfg->check_interval <= 0) return fail(h, LBM_ERR_BAD_ARG, "poisson check interval must be positive");
    if (cfg->dual_residual < 0 || cfg->dual_residual > 2)
        return fail(h, LBM_ERR_BAD_ARG, "dual_residual must be 0, 1 or 2");
    if (cfg->dual_residual && cfg->check_interval < 2)
        return fail(h, LBM_ERR_BAD_ARG, "dual residual needs a check interval of at least 2");
    if (!(cfg->tolerance > 0.0)) return fail(h, LBM_ERR_BAD_ARG, "poisson tolerance must be positive");
    if (cfg->max_sweeps != 0 && cfg->max_sweeps % static_cast<uint64_t>(cfg->check_interval) != 0)
        return fail(h, LBM_ERR_BAD_ARG, "Poisson iteration limit must be a multiple of check interval");
    if (cfg->check_interval != h->pcfg.check_interval || (cfg->dual_residual != 0) != (h->pcfg.dual_residual != 0)) {
        for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second.first);
        h->graphs.clear();
    }
    h->pcfg = *cfg;
    return LBM_OK;
}

lbm_status lbm_set_poisson_form(lbm_handle* h, lbm_poisson_form form, double source_scale, double omega)
{
    if (check_handle(h) != LBM_OK) return LBM_ERR_BAD_ARG;
    if (form != LBM_POISSON_KINETIC && form != LBM_POISSON_SCALAR_JACOBI && form != LBM_POISSON_SCALAR_RB &&
        form != LBM_POISSON_ONEPASS && form != LBM_POISSON_KRYLOV && form != LBM_POISSON_VARCOEF_RB &&
        form != LBM_POISSON_REFINE)
        return fail(h, LBM_ERR_BAD_ARG, "unknown Poisson form");
    if (form == LBM_POISSON_REFINE && h->precision != LBM_PRECISION_MIXED)
        return fail(h, LBM_ERR_BAD_ARG, "the refinement form runs on the mixed-precision box only");
    if (form != LBM_POISSON_KINETIC && form != LBM_POISSON_REFINE && h->precision != LBM_PRECISION_FP64)
        return fail(h, LBM_ERR_BAD_ARG, "the scalar, one-pass and Krylov Poisson forms run in FP64 precision only");
    if (!std::isfinite(source_scale)) return fail(h, LBM_ERR_BAD_ARG, "scalar source scale must be finite");
    if (!(omega == 0.0 || (omega > 0.0 && omega < 2.0)))
        return fail(h, LBM_ERR_BAD_ARG, "SOR relaxation must be 0 (automatic) or in (0, 2)");
    const Geom& g = h->geom;
    const bool rb = form == LBM_POISSON_SCALAR_RB || form == LBM_POISSON_VARCOEF_RB;
    if (rb && (g.ly % 2 || g.lz % 2 || (g.periodic_x && g.lx % 2)))
        return fail(h, LBM_ERR_BAD_ARG, "the red-black forms need even extents along the periodic axes");
    double w = omega;
    if (rb && w == 0.0) {
        // Optimal SOR for the Jacobi iteration of the 14-neighbour stencil:
        // its slowest mode (wave number k) has rho_J = (10 cos k + 4) / 14.
        const double pi = 3.14159265358979323846;
        double k = std::min(2.0 * pi / g.ly, 2.0 * pi / g.lz);
        k = std::min(k, g.periodic_x ? 2.0 * pi / g.lx : pi / std::max(1, g.lx - 1));
        const double rj = (10.0 * std::cos(k) + 4.0) / 14.0;
        w = 2.0 / (1.0 + std::sqrt(std::max(0.0, 1.0 - rj * rj)));
    }
    if (form != h->pform || source_scale != h->scalar_scale || w != h->sor_omega) {
        for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second.first);
        h->graphs.clear();
    }
    h->pform = form;
    h->scalar_scale = source_scale;
    h->sor_omega = w;
    return LBM_OK;
}

lbm_status lbm_set_poisson_accel(lbm_handle* h, const lbm_poisson_accel* a)
{
    if (check_handle(h) != LBM_OK || !a) return fail(h, LBM_ERR_BAD_ARG, "null settings");
    // The reference setters' own checks (GPU/InamuroCUDA.cu:2488-2540).
    if (!(a->pressure_relax_scale > 0.0)) return fail(h, LBM_ERR_BAD_ARG, "pressure relaxation scale must be positive");
    if (!(a->fixed_point_relax > 0.0))
        return fail(h, LBM_ERR_BAD_ARG, "Poisson fixed-point relaxation must be positive");
    if (!(a->anderson_beta_max >= 0.0))
        return fail(h, LBM_ERR_BAD_ARG, "Poisson Anderson beta max must be non-negative");
    if (!(a->two_grid_strength >= 0.0))
        return fail(h, LBM_ERR_BAD_ARG, "Poisson two-grid strength must be non-negative");
    if (!std::isfinite(a->source_aware_scale)) return fail(h, LBM_ERR_BAD_ARG, "source-aware scale must be finite");
    if (a->krylov_degree < 0 || a->krylov_degree > 16)
        return fail(h, LBM_ERR_BAD_ARG, "Krylov polynomial degree must be in [0, 16]");
    if ((a->pressure_relax_scale != 1.0 || a->fixed_point_relax != 1.0 || a->anderson_m1 || a->two_grid ||
         a->source_aware_init || a->spatial_diagnostics) && h->precision != LBM_PRECISION_FP64)
        return fail(h, LBM_ERR_BAD_ARG, "the Poisson accelerators run in FP64 precision only");
    const bool init_changed = (a->source_aware_init != 0) != (h->paccel.source_aware_init != 0) ||
                              a->source_aware_scale != h->paccel.source_aware_scale ||
                              a->two_grid_strength != h->paccel.two_grid_strength;
    h->paccel = *a;
    if (init_changed) {
        for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second.first);
        h->graphs.clear();
    }
    return LBM_OK;
}

lbm_status lbm_get_poisson_accel(const lbm_handle* h, lbm_poisson_accel* out)
{
    if (!h || !out) return LBM_ERR_BAD_ARG;
    *out = h->paccel;
    return LBM_OK;
}

lbm_status lbm_get_poisson_form(const lbm_handle* h, lbm_poisson_form* form, double* source_scale, double* omega)
{
    if (!h) return LBM_ERR_BAD_ARG;
    if (form) *form = static_cast<lbm_poisson_form>(h->pform);
    if (source_scale) *source_scale = h->scalar_scale;
    if (omega) *omega = h->sor_omega;
    return LBM_OK;
}

lbm_status lbm_get_poisson(const lbm_handle* h, lbm_poisson_cfg* cfg)
{
    if (!h || !cfg) return LBM_ERR_BAD_ARG;
    *cfg = h->pcfg;
    return LBM_OK;
}

lbm_status lbm_step(lbm_handle* h, int n_steps, lbm_step_stats* stats)
{
    if (check_handle(h) != LBM_OK || n_steps < 0) return fail(h, LBM_ERR_BAD_ARG, "bad step count");
    cudaSetDevice(h->device);
    for (int i = 0; i < n_steps; ++i) {
        const lbm_status s = step_once(h, 0, stats ? stats + i : nullptr);
        if (s != LBM_OK) return s;
    }
    return LBM_OK;
}

lbm_status lbm_step_replay(lbm_handle* h, int n_steps, const uint64_t* sweeps, lbm_step_stats* stats)
{
    if (check_handle(h) != LBM_OK || n_steps < 0 || !sweeps) return fail(h, LBM_ERR_BAD_ARG, "bad replay");
    cudaSetDevice(h->device);
    for (int i = 0; i < n_steps; ++i) {
        if (sweeps[i] == 0 || sweeps[i] % static_cast<uint64_t>(h->pcfg.check_interval) != 0)
            return fail(h, LBM_ERR_BAD_ARG, "replay sweeps must be a positive multiple of the check interval");
        const lbm_status s = step_once(h, sweeps[i], stats ? stats + i : nullptr);
        if (s != LBM_OK) return s;
    }
    return LBM_OK;
}

lbm_status lbm_set_check_callback(lbm_handle* h, lbm_check_callback cb, void* user)
{
    if (check_handle(h) != LBM_OK) return LBM_ERR_BAD_ARG;
    h->check_cb = cb;
    h->check_user = user;
    return LBM_OK;
}

lbm_status lbm_download(lbm_handle* h, lbm_field which, double* host)
{
    if (check_handle(h) != LBM_OK || !host || which < LBM_FIELD_PHI || which > LBM_FIELD_P)
        return fail(h, LBM_ERR_BAD_ARG, "bad download");
    cudaSetDevice(h->device);
    const size_t bytes = static_cast<size_t>(h->geom.n) * sizeof(double);
    if (h->precision == LBM_PRECISION_FP64) {
        LBM_CUDA(h, cudaMemcpyAsync(host, field_ptr(h, which), bytes, cudaMemcpyDeviceToHost, h->stream));
    } else {
        const lbm_status s = mixed_download(h->stream, h->mb, h->geom, static_cast<int>(which), host);
        if (s != LBM_OK) return fail(h, s, "mixed download failed");
    }
    LBM_CUDA(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

lbm_status lbm_download_ghosted(lbm_handle* h, lbm_field which, double* host)
{
    if (check_handle(h) != LBM_OK || !host) return fail(h, LBM_ERR_BAD_ARG, "bad download");
    const size_t plane = static_cast<size_t>(h->geom.lx) * h->geom.ly;
    const lbm_status s = lbm_download(h, which, host + plane);
    if (s != LBM_OK) return s;
    const int f = static_cast<int>(which);
    std::memcpy(host, h->ghost.data() + (2 * f) * plane, plane * sizeof(double));
    std::memcpy(host + (h->geom.lz + 1) * plane, h->ghost.data() + (2 * f + 1) * plane,
                plane * sizeof(double));
    return LBM_OK;
}

lbm_status lbm_download_h(lbm_handle* h, double* host)
{
    if (check_handle(h) != LBM_OK || !host) return fail(h, LBM_ERR_BAD_ARG, "bad download");
    cudaSetDevice(h->device);
    const size_t n = static_cast<size_t>(h->geom.n);
    if (h->h_loaded && h->precision == LBM_PRECISION_FP64) {
        std::vector<double> soa(15 * n);
        LBM_CUDA(h, cudaMemcpyAsync(soa.data(), h->b.h[1], 15 * n * sizeof(double),
                                    cudaMemcpyDeviceToHost, h->stream));
        LBM_CUDA(h, cudaStreamSynchronize(h->stream));
        for (size_t c = 0; c < n; ++c)
            for (int q = 0; q < 15; ++q) host[c * 15 + q] = soa[q * n + c];
        return LBM_OK;
    }
    if (h->h_loaded) {
        std::fill(host, host + 15 * n, 0.0);
        return LBM_OK;
    }
    // After update_hh: h_q = p * E_q (CPU/Inamuro.cpp:825-840).
    std::vector<double> p(n);
    const lbm_status s = lbm_download(h, LBM_FIELD_P, p.data());
    if (s != LBM_OK) return s;
    for (size_t c = 0; c < n; ++c)
        for (int q = 0; q < 15; ++q) host[c * 15 + q] = p[c] * wE(q);
    return LBM_OK;
}

lbm_status lbm_field_device_ptr(lbm_handle* h, lbm_field which, const double** dev)
{
    if (check_handle(h) != LBM_OK || !dev || which < LBM_FIELD_PHI || which > LBM_FIELD_P)
        return fail(h, LBM_ERR_BAD_ARG, "bad field");
    if (h->precision != LBM_PRECISION_FP64) return fail(h, LBM_ERR_BAD_ARG, "device pointers are FP64-only");
    *dev = field_ptr(h, which);
    return LBM_OK;
}

lbm_status lbm_field_statistics(lbm_handle* h, lbm_field which, lbm_field_stats* out)
{
    if (check_handle(h) != LBM_OK || !out || which < LBM_FIELD_PHI || which > LBM_FIELD_P)
        return fail(h, LBM_ERR_BAD_ARG, "bad field statistics request");
    cudaSetDevice(h->device);
    cudaError_t e;
    if (h->precision == LBM_PRECISION_FP64) {
        e = field_stats<double>(h->stream, field_ptr(h, which), h->geom.n, h->stats_part, h->stats_dev);
    } else {
        const void* f = mixed_field_ptr(h->mb, static_cast<int>(which));
        e = (which == LBM_FIELD_P)
                ? field_stats<double>(h->stream, static_cast<const double*>(f), h->geom.n, h->stats_part, h->stats_dev)
                : field_stats<float>(h->stream, static_cast<const float*>(f), h->geom.n, h->stats_part, h->stats_dev);
    }
    if (e != cudaSuccess) return fail(h, LBM_ERR_CUDA, std::string("field statistics: ") + cudaGetErrorString(e));
    LBM_CUDA(h, cudaMemcpyAsync(out, h->stats_dev, sizeof(lbm_field_stats), cudaMemcpyDeviceToHost, h->stream));
    LBM_CUDA(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

lbm_status lbm_diagnostics_snapshot(lbm_handle* h, lbm_diagnostics* out)
{
    if (check_handle(h) != LBM_OK || !out) return fail(h, LBM_ERR_BAD_ARG, "bad diagnostics request");
    cudaSetDevice(h->device);
    cudaStream_t st = h->stream;
    const long long n = h->geom.n;
    lbm_field_stats* dst[7] = {&out->rho, &out->fei, &out->u, &out->v, &out->w, &out->velocity_magnitude, &out->p};
    // snapshot order -> field ids (velocity magnitude handled apart)
    const lbm_field ids[7] = {LBM_FIELD_RHO, LBM_FIELD_PHI, LBM_FIELD_U, LBM_FIELD_V, LBM_FIELD_W,
                              LBM_FIELD_U, LBM_FIELD_P};
    for (int k = 0; k < 7; ++k) {
        cudaError_t e;
        lbm_field_stats* res = h->stats_dev + k;
        if (h->precision == LBM_PRECISION_FP64) {
            e = (k == 5) ? velmag_stats<double>(st, h->b.u, h->b.v, h->b.w, n, h->stats_part, res)
                         : field_stats<double>(st, field_ptr(h, ids[k]), n, h->stats_part, res);
        } else if (k == 5) {
            e = velmag_stats<float>(st, h->mb.u, h->mb.v, h->mb.w, n, h->stats_part, res);
        } else {
            const void* f = mixed_field_ptr(h->mb, static_cast<int>(ids[k]));
            e = (ids[k] == LBM_FIELD_P) ? field_stats<double>(st, static_cast<const double*>(f), n, h->stats_part, res)
                                        : field_stats<float>(st, static_cast<const float*>(f), n, h->stats_part, res);
        }
        if (e != cudaSuccess) return fail(h, LBM_ERR_CUDA, std::string("diagnostics: ") + cudaGetErrorString(e));
    }
    lbm_field_stats host[7];
    LBM_CUDA(h, cudaMemcpyAsync(host, h->stats_dev, sizeof(host), cudaMemcpyDeviceToHost, st));
    LBM_CUDA(h, cudaStreamSynchronize(st));
    for (int k = 0; k < 7; ++k) *dst[k] = host[k];
    return LBM_OK;
}

lbm_status lbm_synchronize(lbm_handle* h)
{
    if (check_handle(h) != LBM_OK) return LBM_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    LBM_CUDA(h, cudaStreamSynchronize(h->stream));
    return LBM_OK;
}

lbm_status lbm_get_timing(const lbm_handle* h, lbm_timing* out)
{
    if (!h || !out) return LBM_ERR_BAD_ARG;
    *out = h->acc;
    return LBM_OK;
}

lbm_status lbm_reset_timing(lbm_handle* h)
{
    if (!h) return LBM_ERR_BAD_ARG;
    h->acc = lbm_timing{};
    return LBM_OK;
}

lbm_status lbm_set_timing(lbm_handle* h, int enabled)
{
    if (!h) return LBM_ERR_BAD_ARG;
    h->timing = enabled != 0;
    return LBM_OK;
}

}  // extern "C"
