// InamuroCUDA.hpp -- drop-in replacement of the reference's GPU class
// (GPU/InamuroCUDA.hpp:16-248 + GPU/InamuroCUDA.cu of UniBoy222/LBM) over the
// B200 C ABI (lbm_b200.h, liblbm_b200.so).
//
// Same class name, constructor and public methods, so the reference's
// unchanged GPU/main.cpp and GPU/Inamuro.{hpp,cpp} build against it: put this
// directory before the reference's GPU directory on the include path, link
// liblbm_b200.so instead of compiling InamuroCUDA.cu.  The reference's
// `friend class InamuroCUDA` (GPU/Inamuro.hpp:13) gives this class the same
// access to the CPU object's fields as the original.
//
// Header-only; errors are thrown like the reference throws: std::runtime_error
// for CUDA failures and non-finite values, std::invalid_argument for bad
// settings, std::overflow_error for counter overflow.
//
// Precision: FP64 with the reference's per-cell operation order (the
// default), or the mixed FP32/FP64 mode through the second constructor.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "Inamuro.hpp"
#include "lbm_b200.h"
#include "lbm_b200_diagnostics.hpp"

class InamuroCUDA
{
public:
    struct PoissonStepDiagnostics
    {
        std::uint64_t iterations = 0;
        double relative_error = 0.0;
        double pressure_l1_delta = 0.0;
        double pressure_l1_norm = 0.0;
        double fixed_point_h_l1 = 0.0;
        double fixed_point_h_scale = 0.0;
        double fixed_point_h_relative = 0.0;
        double fixed_point_p_l1 = 0.0;
        double fixed_point_p_scale = 0.0;
        double fixed_point_p_relative = 0.0;
        double fixed_point_relative = 0.0;
        double source_mean = 0.0;
        double source_abs_mean = 0.0;
        double projected_source_mean = 0.0;
        double pressure_gauge_target = 0.0;
        double pressure_gauge_max_shift = 0.0;
        bool fixed_point_evaluated = false;
        bool pressure_converged = false;
        bool fixed_point_converged = false;
        bool dual_residual_enabled = false;
        bool converged = false;
        int fallback_count = 0;
    };

    explicit InamuroCUDA(const Inamuro& cpuSolver) : InamuroCUDA(cpuSolver, LBM_PRECISION_FP64) {}

    InamuroCUDA(const Inamuro& cpuSolver, lbm_precision precision)
    {
        int nx = 0, ny = 0, nz = 0;
        cpuSolver.getGridSize(nx, ny, nz);
        lx_ = nx;
        ly_ = ny;
        lz_ = nz;
        lbm_params prm;
        lbm_params_default(&prm);
        prm.lx = nx;
        prm.ly = ny;
        prm.lz = nz;
        const auto& P = cpuSolver.params;   // friend access, as the reference does (.cu:1444-1456)
        prm.rho_L = P.rho_L;
        prm.rho_G = P.rho_G;
        prm.mu_L = P.mu_L;
        prm.mu_G = P.mu_G;
        prm.tauf = P.tauf;
        prm.taug = P.taug;
        prm.k_f = P.k_f;
        prm.k_g = P.k_g;
        prm.T = P.T;
        prm.a = P.a;
        prm.b = P.b;
        prm.fei_L = P.fei_L;
        prm.fei_G = P.fei_G;
        prm.fei_max = P.fei_max;
        prm.fei_min = P.fei_min;
        prm.DD = P.DD;
        if (lbm_abi_version() != LBM_B200_ABI_VERSION)
            throw std::runtime_error("InamuroCUDA: liblbm_b200 ABI " + std::to_string(lbm_abi_version()) +
                                     " does not match the header's ABI " +
                                     std::to_string(LBM_B200_ABI_VERSION) + "; rebuild against the library");
        check(lbm_create(&prm, precision, 0, &h_), "InamuroCUDA: device set-up");
        // initFromCPU (.cu:1628-1673): the ghosted macro fields of the CPU object.
        std::vector<double> buf[6];
        const std::vector<std::vector<std::vector<double>>>* src[6] = {
            &cpuSolver.fei, &cpuSolver.rho, &cpuSolver.u, &cpuSolver.v, &cpuSolver.w, &cpuSolver.p};
        for (int f = 0; f < 6; ++f) {
            buf[f].resize(static_cast<std::size_t>(lx_) * ly_ * (lz_ + 2));
            for (int z = 0; z < lz_ + 2; ++z)
                for (int y = 0; y < ly_; ++y)
                    for (int x = 0; x < lx_; ++x)
                        buf[f][(static_cast<std::size_t>(z) * ly_ + y) * lx_ + x] = (*src[f])[x][y][z];
        }
        check(lbm_load_fields_ghosted(h_, buf[0].data(), buf[1].data(), buf[2].data(), buf[3].data(),
                                      buf[4].data(), buf[5].data()),
              "InamuroCUDA: upload");
        syncCheckCallback();
        applyPoissonConfig();
    }

    InamuroCUDA(const InamuroCUDA&) = delete;
    InamuroCUDA& operator=(const InamuroCUDA&) = delete;
    InamuroCUDA(InamuroCUDA&& o) noexcept { *this = std::move(o); }
    InamuroCUDA& operator=(InamuroCUDA&& o) noexcept
    {
        if (this != &o) {
            release();
            h_ = o.h_;
            o.h_ = nullptr;
            lx_ = o.lx_; ly_ = o.ly_; lz_ = o.lz_;
            check_interval_ = o.check_interval_;
            tolerance_ = o.tolerance_;
            iteration_limit_ = o.iteration_limit_;
            dual_ = o.dual_;
            shadow_ = o.shadow_;
            fused_ = o.fused_;
            fused_boundary_ = o.fused_boundary_;
            scalar_ = o.scalar_;
            scalar_scale_ = o.scalar_scale_;
            onepass_ = o.onepass_;
            acc_ = o.acc_;
            diag_ = o.diag_;
            csv_ = o.csv_;
            syncCheckCallback();
        }
        return *this;
    }

    ~InamuroCUDA() { release(); }

    // One time step (performTimeStepGPU, GPU/InamuroCUDA.cu:2372-2442).
    void performTimeStepGPU()
    {
        // The reference's own guard (GPU/InamuroCUDA.cu:1846-1856).
        if ((dual_ || shadow_) && (fused_ || fused_boundary_ || scalar_ || onepass_ || acc_.anderson_m1 ||
                                   acc_.two_grid || acc_.source_aware_init || acc_.spatial_diagnostics ||
                                   acc_.pressure_relax_scale != 1.0 ||
                                   acc_.fixed_point_relax != 1.0))
            throw std::runtime_error(
                "fixed-point residual requires frozen split+split Poisson with unit relaxation and all "
                "accelerators disabled");
        lbm_step_stats st{};
        const lbm_status s = lbm_step(h_, 1, &st);
        if (s == LBM_ERR_BAD_ARG) throw std::invalid_argument(lbm_last_error(h_));
        if (s == LBM_ERR_OVERFLOW) throw std::overflow_error(lbm_last_error(h_));
        if (s != LBM_OK) throw std::runtime_error(lbm_last_error(h_));
        diag_.iterations = st.iterations;
        diag_.relative_error = st.relative_error;
        diag_.pressure_l1_delta = st.pressure_l1_delta;
        diag_.pressure_l1_norm = st.pressure_l1_norm;
        diag_.fixed_point_h_l1 = st.fixed_point_h_l1;
        diag_.fixed_point_h_scale = st.fixed_point_h_scale;
        diag_.fixed_point_h_relative = st.fixed_point_h_relative;
        diag_.fixed_point_p_l1 = st.fixed_point_p_l1;
        diag_.fixed_point_p_scale = st.fixed_point_p_scale;
        diag_.fixed_point_p_relative = st.fixed_point_p_relative;
        diag_.fixed_point_relative = st.fixed_point_relative;
        diag_.source_mean = st.source_mean;
        diag_.source_abs_mean = st.source_abs_mean;
        diag_.projected_source_mean = st.projected_source_mean;
        diag_.pressure_gauge_target = st.pressure_gauge_target;
        diag_.pressure_gauge_max_shift = st.pressure_gauge_max_shift;
        diag_.fixed_point_evaluated = st.fixed_point_evaluated != 0;
        diag_.pressure_converged = st.pressure_converged != 0;
        diag_.fixed_point_converged = st.fixed_point_converged != 0;
        diag_.dual_residual_enabled = st.dual_residual_enabled != 0;
        diag_.converged = st.converged != 0;
        diag_.fallback_count = st.converged ? 0 : 1;
    }

    // downloadFieldsToCPU (.cu:1675-1701): rho, phi, u, v, w, p with ghosts.
    void downloadFieldsToCPU(Inamuro& cpuSolver) const
    {
        std::vector<double> buf(static_cast<std::size_t>(lx_) * ly_ * (lz_ + 2));
        std::vector<std::vector<std::vector<double>>>* dst[6] = {
            &cpuSolver.fei, &cpuSolver.rho, &cpuSolver.u, &cpuSolver.v, &cpuSolver.w, &cpuSolver.p};
        for (int f = 0; f < 6; ++f) {
            check(lbm_download_ghosted(h_, static_cast<lbm_field>(f), buf.data()), "downloadFieldsToCPU");
            for (int z = 0; z < lz_ + 2; ++z)
                for (int y = 0; y < ly_; ++y)
                    for (int x = 0; x < lx_; ++x)
                        (*dst[f])[x][y][z] = buf[(static_cast<std::size_t>(z) * ly_ + y) * lx_ + x];
        }
    }

    void downloadHH(std::vector<double>& hh) const
    {
        hh.resize(static_cast<std::size_t>(lx_) * ly_ * lz_ * 15);
        check(lbm_download_h(h_, hh.data()), "downloadHH");
    }

    void synchronize() const { check(lbm_synchronize(h_), "synchronize"); }

    const PoissonStepDiagnostics& getLastPoissonDiagnostics() const { return diag_; }

    // ---- settings (GPU/InamuroCUDA.hpp:67-88) ----
    // The fused Poisson kernel and the fused boundary+pressure kernel of the
    // reference do the split form's arithmetic in fewer launches
    // (GPU/InamuroCUDA.cu:539-584, 732-778): the library's sweep is that form.
    void setUseFusedPoisson(bool e) { fused_ = e; }
    void setUseFusedBoundaryPressure(bool e) { fused_boundary_ = e; }
    // The scalar form (GPU/InamuroCUDA.cu:864-901): lbm_set_poisson_form.
    void setUseScalarPoisson(bool e)
    {
        scalar_ = e;
        applyPoissonForm();
    }
    void setScalarPoissonSourceScale(double scale)
    {
        scalar_scale_ = scale;
        applyPoissonForm();
    }
    // The one-pass form and the accelerators (GPU/InamuroCUDA.cu:780-1328,
    // 2161-2275): lbm_set_poisson_form / lbm_set_poisson_accel.
    void setUseOnePassPoisson(bool e)
    {
        onepass_ = e;
        applyPoissonForm();
    }
    void setUseSourceAwareHHInit(bool e)
    {
        lbm_poisson_accel a = acc_;
        a.source_aware_init = e ? 1 : 0;
        applyPoissonAccel(a, "setUseSourceAwareHHInit");
    }
    void setSourceAwareHHScale(double v)
    {
        lbm_poisson_accel a = acc_;
        a.source_aware_scale = v;
        applyPoissonAccel(a, "setSourceAwareHHScale");
    }
    void setPressureRelaxScale(double v)
    {
        lbm_poisson_accel a = acc_;
        a.pressure_relax_scale = v;
        applyPoissonAccel(a, "setPressureRelaxScale");
    }
    void setPoissonFixedPointRelax(double v)
    {
        lbm_poisson_accel a = acc_;
        a.fixed_point_relax = v;
        applyPoissonAccel(a, "setPoissonFixedPointRelax");
    }
    void setUsePoissonAndersonM1(bool e)
    {
        lbm_poisson_accel a = acc_;
        a.anderson_m1 = e ? 1 : 0;
        applyPoissonAccel(a, "setUsePoissonAndersonM1");
    }
    void setPoissonAndersonBetaMax(double v)
    {
        lbm_poisson_accel a = acc_;
        a.anderson_beta_max = v;
        applyPoissonAccel(a, "setPoissonAndersonBetaMax");
    }
    void setUsePoissonTwoGridCorrection(bool e)
    {
        lbm_poisson_accel a = acc_;
        a.two_grid = e ? 1 : 0;
        applyPoissonAccel(a, "setUsePoissonTwoGridCorrection");
    }
    void setPoissonTwoGridStrength(double v)
    {
        lbm_poisson_accel a = acc_;
        a.two_grid_strength = v;
        applyPoissonAccel(a, "setPoissonTwoGridStrength");
    }
    void setUsePoissonSpatialDiagnostics(bool e)
    {
        lbm_poisson_accel a = acc_;
        a.spatial_diagnostics = e ? 1 : 0;
        applyPoissonAccel(a, "setUsePoissonSpatialDiagnostics");
    }
    // Every Poisson segment already runs as a captured CUDA graph.
    void setUsePoissonGraph(bool) {}
    // Per-phase device timing is always collected.
    void setEnablePoissonDetailTiming(bool) {}
    // Reductions are always fixed-order (deterministic).
    void setUsePoissonDeterministicReductions(bool) {}
    void setEnablePoissonFixedPointShadow(bool e)
    {
        shadow_ = e;
        applyPoissonConfig();
    }
    void setUsePoissonDualResidual(bool e)
    {
        dual_ = e;
        if (e) shadow_ = true;
        applyPoissonConfig();
    }
    void setPoissonConvergence(int check_interval, double tolerance)
    {
        if (check_interval <= 0) throw std::invalid_argument("poisson check interval must be positive");
        if (!(tolerance > 0.0)) throw std::invalid_argument("poisson tolerance must be positive");
        if (iteration_limit_ != 0 && iteration_limit_ % static_cast<std::uint64_t>(check_interval) != 0)
            throw std::invalid_argument("Poisson iteration limit must be a multiple of check interval");
        check_interval_ = check_interval;
        tolerance_ = tolerance;
        applyPoissonConfig();
    }
    void setPoissonIterationLimit(std::uint64_t max_iterations)
    {
        if (max_iterations != 0 && max_iterations % static_cast<std::uint64_t>(check_interval_) != 0)
            throw std::invalid_argument("Poisson iteration limit must be a multiple of check interval");
        iteration_limit_ = max_iterations;
        applyPoissonConfig();
    }
    // Per-check CSV, same header and columns as GPU/InamuroCUDA.cu:2610-2682.
    void setPoissonDiagnosticsPath(const std::string& path)
    {
        csv_.open(path);
        syncCheckCallback();
    }

    void printPerformanceMetrics() const
    {
        lbm_timing t{};
        lbm_get_timing(h_, &t);
        if (t.steps == 0) {
            std::cout << "No performance data collected yet." << std::endl;
            return;
        }
        const double sites = static_cast<double>(lx_) * ly_ * lz_;
        const double n = static_cast<double>(t.steps);
        const double total = t.collide_ms + t.moments_ms + t.prep_ms + t.poisson_ms + t.correct_ms;
        std::cout << "\n========== GPU Performance Metrics (B200 sm_100a) ==========" << std::endl;
        std::cout << "Total time steps: " << t.steps << std::endl;
        std::cout << "Poisson convergence: check_interval=" << check_interval_ << ", tolerance=" << tolerance_
                  << ", dual-residual exit=" << (dual_ ? "enabled" : "disabled")
                  << ", fixed-point shadow=" << (shadow_ ? "enabled" : "disabled") << std::endl;
        std::cout << "poisson_iteration_limit=" << iteration_limit_
                  << (iteration_limit_ == 0 ? " (unbounded)" : "") << std::endl;
        std::cout << "\nAverage device time per step (ms):" << std::endl;
        std::cout << "  Collide+stream: " << t.collide_ms / n << std::endl;
        std::cout << "  Macro:          " << t.moments_ms / n << std::endl;
        std::cout << "  Source prep:    " << t.prep_ms / n << std::endl;
        std::cout << "  Poisson:        " << t.poisson_ms / n << std::endl;
        std::cout << "  Correction:     " << t.correct_ms / n << std::endl;
        std::cout << "  Poisson iters:  " << static_cast<double>(t.sweeps) / n << std::endl;
        std::cout << "  Total per step: " << total / n << std::endl;
        std::cout << "  MLUPS:          " << sites / (total / n * 1000.0) << std::endl;
        std::cout << "  MLUPS (sweeps counted): " << sites * (n + static_cast<double>(t.sweeps)) / (total * 1000.0)
                  << std::endl;
        std::cout << "=============================================================\n" << std::endl;
    }

    void printRooflineSummary() const
    {
        lbm_timing t{};
        lbm_get_timing(h_, &t);
        const double cells = static_cast<double>(lx_) * ly_ * lz_;
        std::cout << "\n========== Roofline (measured) ==========" << std::endl;
        std::cout << "Grid cells: " << cells << std::endl;
        if (t.sweep_kernels > 0) {
            const double ms = t.poisson_ms / static_cast<double>(t.sweep_kernels);
            std::cout << std::fixed << std::setprecision(2)
                      << "Kinetic sweep: " << ms * 1e3 << " us/launch, "
                      << 272.0 * cells / (ms * 1e-3) / 1e9 << " GB/s at 272 B/cell (FP64 model)" << std::endl;
        }
        std::cout << "=========================================\n" << std::endl;
    }

    void resetPerformanceMetrics() { lbm_reset_timing(h_); }

private:
    lbm_handle* h_ = nullptr;
    int lx_ = 0, ly_ = 0, lz_ = 0;
    int check_interval_ = 100;
    double tolerance_ = 1.0e-3;
    std::uint64_t iteration_limit_ = 0;
    bool dual_ = false;
    bool shadow_ = false;
    bool fused_ = false;
    bool fused_boundary_ = false;
    bool scalar_ = false;
    double scalar_scale_ = 2.0;
    bool onepass_ = false;
    lbm_poisson_accel acc_{1.0, 1.0, 0, 1.0, 0, 0.5, 0, 1.0, 0};
    PoissonStepDiagnostics diag_;
    lbm_b200::PoissonCsv csv_;   // per-check CSV (setPoissonDiagnosticsPath)

    void release()
    {
        if (h_) lbm_destroy(h_);
        h_ = nullptr;
    }

    void check(lbm_status s, const char* what) const
    {
        if (s == LBM_OK) return;
        const std::string msg = std::string(what) + ": " + lbm_status_string(s) + " " +
                                (h_ ? lbm_last_error(h_) : "");
        if (s == LBM_ERR_BAD_ARG) throw std::invalid_argument(msg);
        if (s == LBM_ERR_OVERFLOW) throw std::overflow_error(msg);
        throw std::runtime_error(msg);
    }


    void applyPoissonForm()
    {
        if (!h_) return;
        const lbm_poisson_form f =
            scalar_ ? LBM_POISSON_SCALAR_JACOBI : (onepass_ ? LBM_POISSON_ONEPASS : LBM_POISSON_KINETIC);
        check(lbm_set_poisson_form(h_, f, scalar_scale_, 0.0), "setPoissonForm");
    }

    // Invalid values throw as the reference's setters do and leave the settings unchanged.
    void applyPoissonAccel(const lbm_poisson_accel& a, const char* what)
    {
        if (h_) check(lbm_set_poisson_accel(h_, &a), what);
        acc_ = a;
    }

    void applyPoissonConfig()
    {
        if (!h_) return;
        lbm_poisson_cfg cfg{};
        cfg.check_interval = check_interval_;
        cfg.tolerance = tolerance_;
        cfg.dual_residual = dual_ ? 1 : (shadow_ ? 2 : 0);
        cfg.max_sweeps = iteration_limit_;
        cfg.fail_on_limit = 0;
        check(lbm_set_poisson(h_, &cfg), "Poisson configuration");
    }

    // The per-check callback only while a CSV is written: without one the
    // library runs the Poisson segments in its device-side loop.
    void syncCheckCallback()
    {
        if (h_) lbm_set_check_callback(h_, csv_.path().empty() ? nullptr : &InamuroCUDA::onCheck, this);
    }

    static void onCheck(void* user, const lbm_check_record* r)
    {
        lbm_b200::PoissonCsv::on_check(&static_cast<InamuroCUDA*>(user)->csv_, r);
    }
};
