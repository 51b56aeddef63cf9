// adjoint_run.cu -- gradients through whole FP64 time steps (lbm_adjoint_*).
//
// The forward run is an ordinary FP64 box (lbm_handle) stepped one step at a
// time; every checkpoint_interval steps its state (post-collision f and g,
// the six macro fields) is copied aside.  The reverse pass walks the
// intervals from the last: it restores the interval's checkpoint, recomputes
// the interval with the forward's sweep counts (bitwise the same states),
// keeping each step's macro fields and final Poisson h, then runs the steps'
// adjoints backwards.  One step (CPU/Inamuro.cpp:347-363) and its adjoint:
//
//   forward                                    reverse
//   F', G', s' = collide(F, G, X)              4. collide^T -> lam F, G, X
//   X* = moments(F', G')                       3. moments^T (added to lam F', G')
//   p' = poisson(s, rho') + mean(p)            2. adjoint solve -> lam s, lam rho'
//   u' = correct(u*, p', rho')                 1. correct^T -> lam p', lam rho'
//
// X = (phi, rho, u, v, w, p).  p enters the next step only through the
// gauge target (the mean of p, CPU/Inamuro.cpp:699-705) and the solve's
// starting guess, which the converged solve forgets: the mean of lam p' goes
// to lam p uniformly, the rest drives the adjoint solve.  The source
// projection s = (u_x - mean u_x) + v_y + w_z is linear.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/lbm_b200.h"
#include "adjoint.hpp"
#include "handle_internal.hpp"
#include "lbm_solver.cuh"

using namespace lbm;

namespace {

thread_local std::string g_adj_create_error;

}  // namespace

struct lbm_adjoint {
    lbm_params prm{};
    lbm_adjoint_cfg cfg{};
    int device = 0;
    lbm_handle* fwd = nullptr;
    BoxInfo view{};                     // geometry, physics, launch shape, stream of the forward box
    size_t state_bytes = 0;             // one saved forward state (box_state_bytes)
    long long n = 0;
    std::string err;
    int n_steps = 0;
    bool have_forward = false;
    std::vector<uint64_t> sweeps;       // per forward step
    std::vector<double*> ckpt;          // ckpt[k]: state after step k * interval (k >= 1), box_save_state
    double* init = nullptr;             // loaded macro fields (6 n)
    double* final_state = nullptr;      // macro fields after the last step (6 n)
    double* seg_macro = nullptr;        // (interval + 1) x 6 n
    double* seg_h = nullptr;            // interval x 15 n
    double* lpop[2][2] = {};            // [parity][f, g] adjoints of the populations, 15 n each
    double* lmac[2] = {};               // [parity] adjoints of the 6 macro fields, 6 n each
    double* y[2] = {};                  // adjoint Poisson iterates, 15 n each
    double* pi_prev = nullptr;
    double* scratch = nullptr;          // adj::kCollideScratch n
    double* ls = nullptr;
    double* lsrc = nullptr;             // dux, dvy, dwz adjoints, 3 n
    double* lkf = nullptr;
    double* part = nullptr;             // max(2 nblocks, kSumBlocks) partials
    double* part_host = nullptr;        // pinned copy
    size_t part_len = 0;
    double forward_ms = 0.0;
    uint64_t forward_sweeps = 0;
    int y_warm = -1;                    // y buffer holding the last converged adjoint iterate, -1: none
    std::vector<double*> bslot;         // binomial mode: checkpoint slots (state_bytes each), allocated on first use
    std::vector<int> bfree;             // free slot indices
    KrylovBuffers kb{};                 // cfg.krylov: BiCGSTAB work vectors
};

namespace {

lbm_status afail(lbm_adjoint* a, lbm_status s, const std::string& msg)
{
    if (a) a->err = msg;
    return s;
}

#define ADJ_CUDA(a, call)                                                                         \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return afail((a), e_ == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA,       \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

#define ADJ_TRY(a, call, what)                                                                    \
    do {                                                                                          \
        const lbm_status s_ = (call);                                                             \
        if (s_ != LBM_OK) {                                                                       \
            const char* t_ = lbm_last_error((a)->fwd);                                            \
            return afail((a), s_, std::string(what) + (t_ && *t_ ? std::string(": ") + t_ : "")); \
        }                                                                                         \
    } while (0)

double* dalloc(size_t count, cudaError_t* e)
{
    void* p = nullptr;
    *e = cudaMalloc(&p, count * sizeof(double));
    return *e == cudaSuccess ? static_cast<double*>(p) : nullptr;
}

void free_all(lbm_adjoint* a)
{
    for (double* p : a->ckpt) cudaFree(p);
    a->ckpt.clear();
    for (double* p : a->bslot) cudaFree(p);
    a->bslot.clear();
    double* kv[] = {a->kb.r, a->kb.r0, a->kb.p, a->kb.v, a->kb.s, a->kb.t, a->kb.part};
    for (double* p : kv) cudaFree(p);
    if (a->kb.host) cudaFreeHost(a->kb.host);
    a->kb = KrylovBuffers{};
    double* bufs[] = {a->init, a->final_state, a->seg_macro, a->seg_h, a->lpop[0][0], a->lpop[0][1],
                      a->lpop[1][0], a->lpop[1][1], a->lmac[0], a->lmac[1], a->y[0], a->y[1], a->pi_prev,
                      a->scratch, a->ls, a->lsrc, a->lkf, a->part};
    for (double* p : bufs) cudaFree(p);
    if (a->part_host) cudaFreeHost(a->part_host);
    if (a->fwd) lbm_destroy(a->fwd);
}

// Deterministic sum of a[0..n) (fixed device tree, then the host in order).
lbm_status dsum(lbm_adjoint* a, const double* v, long long n, double* out)
{
    cudaStream_t st = a->view.stream;
    adj::sum_partials(st, v, n, a->part);
    ADJ_CUDA(a, cudaMemcpyAsync(a->part_host, a->part, adj::kSumBlocks * sizeof(double), cudaMemcpyDeviceToHost,
                                st));
    ADJ_CUDA(a, cudaStreamSynchronize(st));
    double s = 0.0;
    for (int i = 0; i < adj::kSumBlocks; ++i) s += a->part_host[i];
    *out = s;
    return LBM_OK;
}

}  // namespace

namespace {

double* slot(double* base, long long n, int i) { return base + static_cast<long long>(i) * n; }

// Adjoint of one step X_n -> X_{n+1}.  On entry lpop[cur], lmac[cur] hold the
// adjoint of X_{n+1} (F', G' and the six macro fields); on return
// lpop[1-cur], lmac[1-cur] hold that of X_n and *kf has gained the step's
// dJ/dk_f.  xn, x1: macro fields of X_n and X_{n+1}; h1: the h the step's
// Poisson solve ended with.
lbm_status step_adjoint(lbm_adjoint* a, bool first, double* const xn, double* const x1, const double* h1, int cur,
                        uint64_t* adj_sweeps, double* kf)
{
    const Geom& g = a->view.geom;
    const Phys& P = a->view.phys;
    const Launch& L = a->view.L;
    cudaStream_t st = a->view.stream;
    const long long n = a->n;
    double* lm = a->lmac[cur];
    double* lf = a->lpop[cur][0];
    double* lg = a->lpop[cur][1];
    auto X1 = [&](int i) { return slot(x1, n, i); };
    auto XN = [&](int i) { return slot(xn, n, i); };
    auto LM = [&](int i) { return slot(lm, n, i); };
    // 1. velocity correction
    adj::correct_backward_add(st, L, g, X1(5), X1(1), LM(2), LM(3), LM(4), LM(5), LM(1));
    // 2. the gauge takes the mean of lam p; the rest drives the adjoint solve
    double sum_lp = 0.0;
    lbm_status s = dsum(a, LM(5), n, &sum_lp);
    if (s != LBM_OK) return s;
    const double mean_lp = sum_lp / static_cast<double>(n);
    adj::add_const(st, LM(5), n, -mean_lp);
    // Start from the previous reverse step's converged iterate (the adjoint
    // fields change little from one step to the next), else from y = lam p.
    int yc = 0;
    if (a->y_warm >= 0) {
        yc = a->y_warm;
    } else {
        adj::poisson_init(st, L, g, LM(5), a->y[0]);
    }
    uint64_t it = 0;
    if (a->cfg.krylov) {
        // BiCGSTAB on (I - B) y = lam_p, B = M^T o pull from x + c_q
        KrylovResult kr;
        const double tol = a->cfg.krylov_tolerance > 0.0 ? a->cfg.krylov_tolerance : 1e-10;
        const lbm_status ks = krylov::solve_adjoint(st, L, g, a->kb, a->y[yc], X1(1), LM(5), tol, a->cfg.max_sweeps, &kr);
        if (ks == LBM_ERR_POISSON_BUDGET)
            return afail(a, ks, "adjoint Poisson sweep limit reached without convergence");
        if (ks != LBM_OK) return afail(a, ks, "adjoint Krylov solve broke down or diverged");
        it = kr.matvecs;
    }
    adj::poisson_pi(st, L, g, a->y[yc], a->pi_prev);
    const int ci = a->cfg.check_interval;
    for (; !a->cfg.krylov;) {
        for (int i = 0; i < ci; ++i) {
            const bool check = i == ci - 1;
            adj::poisson_sweep(st, L, g, check, a->y[yc], a->y[1 - yc], X1(1), LM(5), a->pi_prev, a->part);
            yc = 1 - yc;
        }
        it += static_cast<uint64_t>(ci);
        ADJ_CUDA(a, cudaGetLastError());
        ADJ_CUDA(a, cudaMemcpyAsync(a->part_host, a->part, 2 * L.nblocks * sizeof(double), cudaMemcpyDeviceToHost,
                                    st));
        ADJ_CUDA(a, cudaStreamSynchronize(st));
        double d = 0.0, nrm = 0.0;
        for (long long b = 0; b < L.nblocks; ++b) d += a->part_host[b];
        for (long long b = 0; b < L.nblocks; ++b) nrm += a->part_host[L.nblocks + b];
        if (!std::isfinite(d) || !std::isfinite(nrm))
            return afail(a, LBM_ERR_NONFINITE, "adjoint Poisson iterate contains NaN/Inf");
        if (nrm == 0.0 || d < a->cfg.tolerance * nrm) break;
        if (a->cfg.max_sweeps && it >= a->cfg.max_sweeps)
            return afail(a, LBM_ERR_POISSON_BUDGET, "adjoint Poisson sweep limit reached without convergence");
    }
    *adj_sweeps += it;
    a->y_warm = yc;
    adj::poisson_final(st, L, g, a->y[yc], h1, X1(1), a->ls, LM(1));
    // 3. source projection
    double sum_ls = 0.0;
    s = dsum(a, a->ls, n, &sum_ls);
    if (s != LBM_OK) return s;
    double* ldux = slot(a->lsrc, n, 0);
    double* ldvy = slot(a->lsrc, n, 1);
    double* ldwz = slot(a->lsrc, n, 2);
    adj::prep_backward(st, L, g, a->ls, sum_ls / static_cast<double>(n), ldux, ldvy, ldwz);
    // 4. moments, added to the adjoints of F', G'
    adj::moments_backward_add(st, L, g, P, X1(0), LM(0), LM(1), LM(2), LM(3), LM(4), lf, lg);
    // 5. collide, into the adjoint of X_n
    const int nx = 1 - cur;
    double* ln = a->lmac[nx];
    adj::collide_backward(st, L, g, P, first, XN(0), XN(1), XN(2), XN(3), XN(4), lf, lg, ldux, ldvy, ldwz,
                          a->lpop[nx][0], a->lpop[nx][1], slot(ln, n, 0), slot(ln, n, 1), slot(ln, n, 2),
                          slot(ln, n, 3), slot(ln, n, 4), a->scratch, a->lkf);
    ADJ_CUDA(a, cudaMemsetAsync(slot(ln, n, 5), 0, n * sizeof(double), st));
    adj::add_const(st, slot(ln, n, 5), n, mean_lp);
    ADJ_CUDA(a, cudaGetLastError());
    double k = 0.0;
    s = dsum(a, a->lkf, n, &k);
    if (s != LBM_OK) return s;
    *kf += k;
    return LBM_OK;
}

// Restores the state at step s0 and recomputes steps s0+1 .. s1, keeping
// X_{s0} .. X_{s1} (macro fields) and each step's final h.
lbm_status recompute(lbm_adjoint* a, int s0, int s1)
{
    const long long n = a->n;
    const size_t fbytes = static_cast<size_t>(n) * sizeof(double);
    cudaStream_t st = a->view.stream;
    if (s0 == 0) {
        ADJ_TRY(a, lbm_load_fields_device(a->fwd, slot(a->init, n, 0), slot(a->init, n, 1), slot(a->init, n, 2),
                                          slot(a->init, n, 3), slot(a->init, n, 4), slot(a->init, n, 5)),
                "reload of the initial fields");
        ADJ_CUDA(a, cudaMemcpyAsync(a->seg_macro, a->init, 6 * fbytes, cudaMemcpyDeviceToDevice, st));
    } else {
        ADJ_TRY(a, box_restore_state(a->fwd, a->ckpt[s0 / a->cfg.checkpoint_interval - 1]), "checkpoint restore");
        ADJ_TRY(a, box_export(a->fwd, a->seg_macro, nullptr), "state export");
    }
    for (int k = s0; k < s1; ++k) {
        ADJ_TRY(a, lbm_step_replay(a->fwd, 1, &a->sweeps[k], nullptr), "recomputation step");
        ADJ_TRY(a, box_export(a->fwd, slot(a->seg_macro, 6 * n, k - s0 + 1), slot(a->seg_h, 15 * n, k - s0)),
                "state export");
    }
    ADJ_CUDA(a, cudaStreamSynchronize(st));
    return LBM_OK;
}

// ---- binomial checkpointing ------------------------------------------------
// Griewank's revolve schedule, recursive form: to reverse steps [a, b) from
// a stored state at a with c free slots, when b - a > 1 and c > 0 advance to
// m, store the state there, reverse [m, b) with c - 1 slots, free it and
// reverse [a, m) with c.  The stored base counts as a checkpoint, so with r
// the least repetition count with beta(c + 1, r) = C(c + 1 + r, c + 1) >= l
// (l = b - a) a split keeps every step within r recomputations when
// [m, b) stays within beta(c, r) and [a, m) within beta(c + 1, r - 1)
// (beta(c + 1, r) = beta(c, r) + beta(c + 1, r - 1)).  Within that interval
// the split point is the one of nine evenly spaced candidates whose
// estimated total is least, the estimate being the cost of always splitting
// at the interval's midpoint (memoised).  Against an exhaustive search over
// all splits (up to 400 steps, 2 to 25 slots) this is within 4 % of the
// fewest recomputed steps.  With no slot left, each step of [a, b) is
// reached from a in turn.  A leaf n restores the base state at a, advances
// to n, runs step n + 1 keeping X_n, X_{n+1} and its final h, and runs that
// step's adjoint.
double beta(int c, int r)
{
    double v = 1.0;
    for (int i = 1; i <= c; ++i) v = v * (r + i) / i;
    return v;
}

// Split interval [lo, hi] for l steps and c free slots.
void split_bounds(int l, int c, int* lo, int* hi)
{
    int r = 1;
    while (beta(c + 1, r) < l) ++r;
    const double right_cap = beta(c, r), left_cap = beta(c + 1, r - 1);
    int a = right_cap >= l ? 1 : static_cast<int>(l - right_cap);
    int b = left_cap >= l - 1 ? l - 1 : static_cast<int>(left_cap);
    a = std::max(1, std::min(a, l - 1));
    b = std::max(1, std::min(b, l - 1));
    if (a > b) b = a;
    *lo = a;
    *hi = b;
}

// Forward steps of the midpoint schedule (the split estimate), memoised.
struct SplitPlanner {
    std::unordered_map<uint64_t, uint64_t> memo;
    uint64_t mid_cost(int l, int c)
    {
        if (l <= 1) return 1;
        if (c <= 0) return static_cast<uint64_t>(l) * (l + 1) / 2;
        const uint64_t key = (static_cast<uint64_t>(l) << 20) | static_cast<uint64_t>(c);
        const auto it = memo.find(key);
        if (it != memo.end()) return it->second;
        int lo, hi;
        split_bounds(l, c, &lo, &hi);
        const int l1 = (lo + hi) / 2;
        const uint64_t v = static_cast<uint64_t>(l1) + mid_cost(l - l1, c - 1) + mid_cost(l1, c);
        memo[key] = v;
        return v;
    }
    int split(int l, int c)
    {
        int lo, hi;
        split_bounds(l, c, &lo, &hi);
        int best = lo;
        uint64_t best_cost = UINT64_MAX;
        for (int k = 0; k <= 8; ++k) {
            const int l1 = lo + (hi - lo) * k / 8;
            const uint64_t v = static_cast<uint64_t>(l1) + mid_cost(l - l1, c - 1) + mid_cost(l1, c);
            if (v < best_cost) {
                best_cost = v;
                best = l1;
            }
        }
        return best;
    }
};

template <class Ops>
lbm_status revolve(Ops& ops, SplitPlanner& plan, int a, int b, int c, int base)
{
    const int l = b - a;
    if (l == 1) return ops.leaf(a, a, base);
    if (c <= 0) {
        for (int n = b - 1; n >= a; --n) {
            const lbm_status s = ops.leaf(n, a, base);
            if (s != LBM_OK) return s;
        }
        return LBM_OK;
    }
    const int m = a + plan.split(l, c);
    int slot = -1;
    lbm_status s = ops.save_at(base, a, m, &slot);
    if (s != LBM_OK) return s;
    s = revolve(ops, plan, m, b, c - 1, slot);
    if (s != LBM_OK) return s;
    ops.release(slot);
    return revolve(ops, plan, a, m, c, base);
}

// Counts what a schedule does, without device work.
struct DryOps {
    uint64_t steps = 0;
    int live = 0, peak = 0;
    lbm_status leaf(int n, int a, int) { steps += static_cast<uint64_t>(n - a) + 1; return LBM_OK; }
    lbm_status save_at(int, int a, int m, int* slot)
    {
        steps += static_cast<uint64_t>(m - a);
        *slot = live++;
        peak = std::max(peak, live);
        return LBM_OK;
    }
    void release(int) { --live; }
};

lbm_status restore_state(lbm_adjoint* a, int base);
lbm_status advance(lbm_adjoint* a, int from, int to, uint64_t* counted);

// Device schedule: base -1 is the loaded state (step 0), else a slot.
struct GpuOps {
    lbm_adjoint* a;
    int cur = 0;
    double kf = 0.0;
    uint64_t adj_sweeps = 0, recomputed = 0;

    lbm_status leaf(int n, int from, int base)
    {
        lbm_status s = restore_state(a, base);
        if (s != LBM_OK) return s;
        s = advance(a, from, n, &recomputed);
        if (s != LBM_OK) return s;
        s = recompute_from_current(n);
        if (s != LBM_OK) return s;
        s = step_adjoint(a, n == 0, a->seg_macro, slot(a->seg_macro, 6 * a->n, 1), a->seg_h, cur, &adj_sweeps, &kf);
        cur = 1 - cur;
        return s;
    }

    // X_n (the box's current state) and step n + 1 into the one-step buffers.
    lbm_status recompute_from_current(int n)
    {
        const long long nn = a->n;
        cudaStream_t st = a->view.stream;
        ADJ_TRY(a, box_export(a->fwd, a->seg_macro, nullptr), "state export");
        ADJ_TRY(a, lbm_step_replay(a->fwd, 1, &a->sweeps[n], nullptr), "recomputation step");
        ++recomputed;
        ADJ_TRY(a, box_export(a->fwd, slot(a->seg_macro, 6 * nn, 1), a->seg_h), "state export");
        ADJ_CUDA(a, cudaStreamSynchronize(st));
        return LBM_OK;
    }

    lbm_status save_at(int base, int from, int m, int* out)
    {
        lbm_status s = restore_state(a, base);
        if (s != LBM_OK) return s;
        s = advance(a, from, m, &recomputed);
        if (s != LBM_OK) return s;
        int k;
        if (!a->bfree.empty()) {
            k = a->bfree.back();
            a->bfree.pop_back();
        } else {
            cudaError_t e = cudaSuccess;
            double* buf = dalloc(a->state_bytes / sizeof(double), &e);
            if (e != cudaSuccess) return afail(a, LBM_ERR_OOM, "binomial checkpoint allocation failed");
            a->bslot.push_back(buf);
            k = static_cast<int>(a->bslot.size()) - 1;
        }
        cudaStream_t st = a->view.stream;
        ADJ_TRY(a, box_save_state(a->fwd, a->bslot[k]), "checkpoint save");
        ADJ_CUDA(a, cudaStreamSynchronize(st));
        *out = k;
        return LBM_OK;
    }

    void release(int k) { a->bfree.push_back(k); }
};

lbm_status restore_state(lbm_adjoint* a, int base)
{
    const long long n = a->n;
    if (base < 0) {
        ADJ_TRY(a, lbm_load_fields_device(a->fwd, slot(a->init, n, 0), slot(a->init, n, 1), slot(a->init, n, 2),
                                          slot(a->init, n, 3), slot(a->init, n, 4), slot(a->init, n, 5)),
                "reload of the initial fields");
        return LBM_OK;
    }
    ADJ_TRY(a, box_restore_state(a->fwd, a->bslot[base]), "checkpoint restore");
    return LBM_OK;
}

lbm_status advance(lbm_adjoint* a, int from, int to, uint64_t* counted)
{
    for (int k = from; k < to; ++k) {
        ADJ_TRY(a, lbm_step_replay(a->fwd, 1, &a->sweeps[k], nullptr), "recomputation step");
        ++*counted;
    }
    return LBM_OK;
}

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

lbm_status lbm_adjoint_create(const lbm_params* p, int device, const lbm_adjoint_cfg* cfg, lbm_adjoint** out)
{
    g_adj_create_error.clear();
    if (!p || !cfg || !out) {
        g_adj_create_error = "null argument";
        return LBM_ERR_BAD_ARG;
    }
    *out = nullptr;
    if ((cfg->binomial_checkpoints == 0 && cfg->checkpoint_interval < 1) || cfg->binomial_checkpoints < 0 ||
        (cfg->precision != 0 && cfg->precision != 1) ||
        cfg->check_interval < 1 || !(cfg->tolerance > 0.0) ||
        (cfg->max_sweeps && cfg->max_sweeps % static_cast<uint64_t>(cfg->check_interval) != 0)) {
        g_adj_create_error = "adjoint settings: checkpoint_interval >= 1 (or binomial_checkpoints > 0), "
                             "check_interval >= 1, tolerance > 0, max_sweeps a multiple of check_interval";
        return LBM_ERR_BAD_ARG;
    }
    lbm_adjoint* a = new lbm_adjoint();
    a->prm = *p;
    a->cfg = *cfg;
    a->device = device;
    const lbm_precision prec = cfg->precision == 1 ? LBM_PRECISION_MIXED : LBM_PRECISION_FP64;
    lbm_status s = lbm_create(p, prec, device, &a->fwd);
    if (s != LBM_OK) {
        g_adj_create_error = std::string("forward box: ") + lbm_last_error(nullptr);
        delete a;
        return s;
    }
    s = box_info(a->fwd, &a->view);
    if (s != LBM_OK) {
        g_adj_create_error = "forward box info";
        free_all(a);
        delete a;
        return s;
    }
    a->state_bytes = box_state_bytes(a->fwd);
    const long long n = a->view.geom.n;
    a->n = n;
    const size_t K = cfg->binomial_checkpoints > 0 ? 1 : static_cast<size_t>(cfg->checkpoint_interval);
    if (cfg->krylov) {
        const size_t parts = 3 * static_cast<size_t>(std::max<long long>(a->view.L.nblocks, kKrylovBlocks));
        double** kv[] = {&a->kb.r, &a->kb.r0, &a->kb.p, &a->kb.v, &a->kb.s, &a->kb.t};
        cudaError_t ke = cudaSuccess;
        for (double** p : kv)
            if (ke == cudaSuccess) *p = dalloc(15 * static_cast<size_t>(n), &ke);
        if (ke == cudaSuccess) a->kb.part = dalloc(parts, &ke);
        if (ke == cudaSuccess) ke = cudaMallocHost(&a->kb.host, parts * sizeof(double));
        if (ke != cudaSuccess) {
            g_adj_create_error = std::string("Krylov buffers: ") + cudaGetErrorString(ke);
            free_all(a);
            delete a;
            return ke == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA;
        }
    }
    cudaError_t e = cudaSuccess;
    struct Req { double** dst; size_t count; };
    const Req reqs[] = {
        {&a->init, 6 * (size_t)n}, {&a->final_state, 6 * (size_t)n}, {&a->seg_macro, (K + 1) * 6 * (size_t)n},
        {&a->seg_h, K * 15 * (size_t)n}, {&a->lpop[0][0], 15 * (size_t)n}, {&a->lpop[0][1], 15 * (size_t)n},
        {&a->lpop[1][0], 15 * (size_t)n}, {&a->lpop[1][1], 15 * (size_t)n}, {&a->lmac[0], 6 * (size_t)n},
        {&a->lmac[1], 6 * (size_t)n}, {&a->y[0], 15 * (size_t)n}, {&a->y[1], 15 * (size_t)n},
        {&a->pi_prev, (size_t)n}, {&a->scratch, adj::kCollideScratch * (size_t)n}, {&a->ls, (size_t)n},
        {&a->lsrc, 3 * (size_t)n}, {&a->lkf, (size_t)n}};
    for (const Req& r : reqs) {
        *r.dst = dalloc(r.count, &e);
        if (e != cudaSuccess) break;
    }
    a->part_len = std::max<size_t>(2 * static_cast<size_t>(a->view.L.nblocks), adj::kSumBlocks);
    if (e == cudaSuccess) a->part = dalloc(a->part_len, &e);
    if (e == cudaSuccess) e = cudaMallocHost(&a->part_host, a->part_len * sizeof(double));
    if (e != cudaSuccess) {
        g_adj_create_error = std::string("adjoint buffers: ") + cudaGetErrorString(e);
        free_all(a);
        delete a;
        return e == cudaErrorMemoryAllocation ? LBM_ERR_OOM : LBM_ERR_CUDA;
    }
    *out = a;
    return LBM_OK;
}

void lbm_adjoint_destroy(lbm_adjoint* a)
{
    if (!a) return;
    cudaSetDevice(a->device);
    free_all(a);
    delete a;
}

lbm_status lbm_adjoint_set_poisson(lbm_adjoint* a, const lbm_poisson_cfg* cfg)
{
    if (!a) return LBM_ERR_BAD_ARG;
    ADJ_TRY(a, lbm_set_poisson(a->fwd, cfg), "forward Poisson settings");
    return LBM_OK;
}

lbm_status lbm_adjoint_forward(lbm_adjoint* a, const double* phi, const double* rho, const double* u,
                               const double* v, const double* w, const double* p, int n_steps,
                               const uint64_t* sweeps)
{
    if (!a) return LBM_ERR_BAD_ARG;
    if (!phi || !rho || !u || !v || !w || n_steps < 1) return afail(a, LBM_ERR_BAD_ARG, "null field or n_steps < 1");
    cudaSetDevice(a->device);
    const auto t0 = std::chrono::steady_clock::now();
    a->have_forward = false;
    const long long n = a->n;
    const size_t fbytes = static_cast<size_t>(n) * sizeof(double);
    cudaStream_t st = a->view.stream;
    const double* src[6] = {phi, rho, u, v, w, p};
    for (int i = 0; i < 6; ++i) {
        if (src[i]) ADJ_CUDA(a, cudaMemcpyAsync(slot(a->init, n, i), src[i], fbytes, cudaMemcpyHostToDevice, st));
        else ADJ_CUDA(a, cudaMemsetAsync(slot(a->init, n, i), 0, fbytes, st));
    }
    ADJ_CUDA(a, cudaStreamSynchronize(st));
    for (double* c : a->ckpt) cudaFree(c);
    a->ckpt.clear();
    const int K = a->cfg.binomial_checkpoints > 0 ? n_steps : a->cfg.checkpoint_interval;
    const int n_ckpt = (n_steps - 1) / K;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < n_ckpt; ++k) {
        double* c = dalloc(a->state_bytes / sizeof(double), &e);
        if (e != cudaSuccess) return afail(a, LBM_ERR_OOM, "checkpoint allocation failed");
        a->ckpt.push_back(c);
    }
    ADJ_TRY(a, lbm_load_fields_device(a->fwd, slot(a->init, n, 0), slot(a->init, n, 1), slot(a->init, n, 2),
                                      slot(a->init, n, 3), slot(a->init, n, 4), slot(a->init, n, 5)),
            "load");
    a->sweeps.assign(n_steps, 0);
    a->forward_sweeps = 0;
    for (int k = 0; k < n_steps; ++k) {
        lbm_step_stats stt{};
        if (sweeps) ADJ_TRY(a, lbm_step_replay(a->fwd, 1, &sweeps[k], &stt), "forward step");
        else ADJ_TRY(a, lbm_step(a->fwd, 1, &stt), "forward step");
        a->sweeps[k] = stt.iterations;
        a->forward_sweeps += stt.iterations;
        const int done = k + 1;
        if (done < n_steps && done % K == 0)
            ADJ_TRY(a, box_save_state(a->fwd, a->ckpt[done / K - 1]), "checkpoint save");
        else if (done == n_steps)
            ADJ_TRY(a, box_export(a->fwd, a->final_state, nullptr), "state export");
    }
    ADJ_CUDA(a, cudaStreamSynchronize(st));
    a->n_steps = n_steps;
    a->have_forward = true;
    a->forward_ms = ms_since(t0);
    return LBM_OK;
}

lbm_status lbm_adjoint_sweeps(const lbm_adjoint* a, uint64_t* out)
{
    if (!a || !out || !a->have_forward) return LBM_ERR_BAD_ARG;
    for (int k = 0; k < a->n_steps; ++k) out[k] = a->sweeps[k];
    return LBM_OK;
}

lbm_status lbm_adjoint_download(const lbm_adjoint* a, lbm_field which, double* host)
{
    if (!a || !host || !a->have_forward || which < LBM_FIELD_PHI || which > LBM_FIELD_P) return LBM_ERR_BAD_ARG;
    cudaSetDevice(a->device);
    const cudaError_t e = cudaMemcpy(host, a->final_state + static_cast<long long>(which) * a->n,
                                     static_cast<size_t>(a->n) * sizeof(double), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LBM_OK : LBM_ERR_CUDA;
}

lbm_status lbm_adjoint_backward(lbm_adjoint* a, const double* lam_phi, const double* lam_rho, const double* lam_u,
                                const double* lam_v, const double* lam_w, const double* lam_p, double* grad_phi,
                                double* grad_rho, double* grad_u, double* grad_v, double* grad_w, double* grad_p,
                                lbm_adjoint_stats* stats)
{
    if (!a) return LBM_ERR_BAD_ARG;
    if (!a->have_forward) return afail(a, LBM_ERR_BAD_ARG, "no forward run");
    cudaSetDevice(a->device);
    const auto t0 = std::chrono::steady_clock::now();
    const long long n = a->n;
    const size_t fbytes = static_cast<size_t>(n) * sizeof(double);
    cudaStream_t st = a->view.stream;
    int cur = 0;
    ADJ_CUDA(a, cudaMemsetAsync(a->lpop[cur][0], 0, 15 * fbytes, st));
    ADJ_CUDA(a, cudaMemsetAsync(a->lpop[cur][1], 0, 15 * fbytes, st));
    const double* lam[6] = {lam_phi, lam_rho, lam_u, lam_v, lam_w, lam_p};
    for (int i = 0; i < 6; ++i) {
        if (lam[i]) ADJ_CUDA(a, cudaMemcpyAsync(slot(a->lmac[cur], n, i), lam[i], fbytes, cudaMemcpyHostToDevice, st));
        else ADJ_CUDA(a, cudaMemsetAsync(slot(a->lmac[cur], n, i), 0, fbytes, st));
    }
    const int T = a->n_steps;
    const int K = a->cfg.binomial_checkpoints > 0 ? T : a->cfg.checkpoint_interval;
    const int n_seg = a->cfg.binomial_checkpoints > 0 ? 0 : (T + K - 1) / K;
    double kf = 0.0;
    uint64_t adj_sweeps = 0, recomputed = 0;
    a->y_warm = -1;
    if (a->cfg.binomial_checkpoints > 0) {
        a->bfree.clear();
        for (int k = static_cast<int>(a->bslot.size()) - 1; k >= 0; --k) a->bfree.push_back(k);
        GpuOps ops{a};
        ops.cur = cur;
        SplitPlanner plan;
        const lbm_status s = revolve(ops, plan, 0, T, a->cfg.binomial_checkpoints, -1);
        if (s != LBM_OK) return s;
        cur = ops.cur;
        kf = ops.kf;
        adj_sweeps = ops.adj_sweeps;
        recomputed = ops.recomputed;
    }
    for (int seg = n_seg - 1; seg >= 0; --seg) {
        const int s0 = seg * K;
        const int s1 = std::min(T, s0 + K);
        const lbm_status s = recompute(a, s0, s1);
        if (s != LBM_OK) return s;
        recomputed += static_cast<uint64_t>(s1 - s0);
        for (int n1 = s1; n1 > s0; --n1) {
            const int j = n1 - s0;
            const lbm_status s2 = step_adjoint(a, n1 == 1, slot(a->seg_macro, 6 * n, j - 1),
                                               slot(a->seg_macro, 6 * n, j), slot(a->seg_h, 15 * n, j - 1), cur,
                                               &adj_sweeps, &kf);
            if (s2 != LBM_OK) return s2;
            cur = 1 - cur;
        }
    }
    double* grads[6] = {grad_phi, grad_rho, grad_u, grad_v, grad_w, grad_p};
    for (int i = 0; i < 6; ++i)
        if (grads[i])
            ADJ_CUDA(a, cudaMemcpyAsync(grads[i], slot(a->lmac[cur], n, i), fbytes, cudaMemcpyDeviceToHost, st));
    ADJ_CUDA(a, cudaStreamSynchronize(st));
    if (stats) {
        stats->grad_kappa_f = kf;
        stats->forward_steps = static_cast<uint64_t>(T);
        stats->forward_sweeps = a->forward_sweeps;
        stats->recompute_steps = recomputed;
        stats->adjoint_sweeps = adj_sweeps;
        stats->forward_ms = a->forward_ms;
        stats->backward_ms = ms_since(t0);
    }
    return LBM_OK;
}

const char* lbm_adjoint_last_error(const lbm_adjoint* a) { return a ? a->err.c_str() : g_adj_create_error.c_str(); }

lbm_status lbm_adjoint_schedule(int n_steps, int checkpoints, uint64_t* recompute_steps, int* peak_checkpoints)
{
    if (n_steps < 1 || checkpoints < 0) return LBM_ERR_BAD_ARG;
    DryOps ops;
    SplitPlanner plan;
    revolve(ops, plan, 0, n_steps, checkpoints, -1);
    if (recompute_steps) *recompute_steps = ops.steps;
    if (peak_checkpoints) *peak_checkpoints = ops.peak;
    return LBM_OK;
}

}  // extern "C"
