// InamuroSolver.hpp -- drop-in replacement of the reference CPU tree's driver
// class (CPU/InamuroSolver.hpp:9-80, CPU/InamuroSolver.cpp) that advances
// the time steps on the B200 through liblbm_b200 (FP64, the reference's
// per-cell operation order).
//
// Same class name, constructor, run() and setSolverConfig() and the same
// params.in handling, so the reference's unchanged CPU/main.cpp builds
// against it: put this directory before the reference's CPU directory on the
// include path, compile CPU/Inamuro.cpp and CPU/common.cpp as usual (not
// CPU/InamuroSolver.cpp), and link liblbm_b200.so.
//
// The solver object derives from the reference's own CPU Inamuro, so the
// parameters, the initial droplets, the Tecplot writer and the output
// configuration are the reference's; only performTimeStep() runs on the GPU.
// The host copy of the fields is refreshed from the device just before the
// reference writes results.  step_diagnostics.csv is written each step from
// the device statistics (lbm_diagnostics_snapshot) with the reference's
// columns and number format.  Console output is a short per-output-step line
// (the reference's progress bars and timing banners are not reproduced).
#pragma once

#include <chrono>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Inamuro.hpp"
#include "lbm_b200.h"
#include "lbm_b200_diagnostics.hpp"

class InamuroSolver
{
public:
    // CPU/InamuroSolver.hpp:17-27: console and output switches, overridable by
    // key=value lines of params.in.
    struct SolverConfig
    {
        bool enable_timing = true;
        bool enable_progress = true;
        bool enable_tecplot_output = true;
        bool enable_debug_field_csv = false;
        bool enable_step_summary_csv = true;
        bool enable_basic_warnings = true;
        std::string output_dir = "out/";
        std::string step_summary_filename = "step_diagnostics.csv";
    };

    explicit InamuroSolver(const std::string& filename)
    {
        const auto t0 = std::chrono::steady_clock::now();
        inamuro_ = std::make_unique<GpuInamuro>(filename);
        init_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        loadConfiguration(filename);
        applyOutputConfiguration();
        openDiagnosticsFile();
    }

    ~InamuroSolver() { releaseDiagnosticsLock(); }

    InamuroSolver(const InamuroSolver&) = delete;
    InamuroSolver& operator=(const InamuroSolver&) = delete;

    void setSolverConfig(const SolverConfig& config)
    {
        config_ = config;
        applyOutputConfiguration();
    }

    // CPU/InamuroSolver.cpp:56-114: diagnostics of the initial state (step 0),
    // then for each step: results every output_frequency steps, the step,
    // its diagnostics row.
    void run()
    {
        recordStepDiagnostics(0, 0.0);
        if (config_.enable_timing)
            std::cout << ">>> initialisation " << init_ms_ << " ms (GPU: liblbm_b200)" << std::endl;
        double total_ms = 0.0;
        for (int t = 0; t < max_time_steps_; ++t) {
            if (output_frequency_ > 0 && t % output_frequency_ == 0) {
                std::cout << t << std::endl;
                inamuro_->writeResults(t);
            }
            const auto s0 = std::chrono::steady_clock::now();
            inamuro_->performTimeStep();
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s0).count();
            total_ms += ms;
            recordStepDiagnostics(t + 1, ms);
        }
        if (config_.enable_timing && max_time_steps_ > 0)
            std::cout << ">>> " << max_time_steps_ << " steps, " << total_ms / max_time_steps_ << " ms per step"
                      << std::endl;
    }

private:
    // The reference's CPU Inamuro with the time step replaced by the GPU step.
    class GpuInamuro : public Inamuro
    {
    public:
        explicit GpuInamuro(const std::string& filename) : Inamuro(filename)
        {
            if (lbm_abi_version() != LBM_B200_ABI_VERSION)
                throw std::runtime_error("InamuroSolver: liblbm_b200 ABI does not match the header; rebuild");
            lbm_params prm;
            lbm_params_default(&prm);
            prm.lx = lx;
            prm.ly = ly;
            prm.lz = lz;
            prm.rho_L = params.rho_L;
            prm.rho_G = params.rho_G;
            prm.mu_L = params.mu_L;
            prm.mu_G = params.mu_G;
            prm.tauf = params.tauf;
            prm.taug = params.taug;
            prm.k_f = params.k_f;
            prm.k_g = params.k_g;
            prm.T = params.T;
            prm.a = params.a;
            prm.b = params.b;
            prm.fei_L = params.fei_L;
            prm.fei_G = params.fei_G;
            prm.fei_max = params.fei_max;
            prm.fei_min = params.fei_min;
            prm.DD = params.DD;
            check(lbm_create(&prm, LBM_PRECISION_FP64, 0, &h_), "InamuroSolver: device set-up");
            std::vector<double> buf[6];
            Vector3D* src[6] = {&fei, &rho, &u, &v, &w, &p};
            for (int f = 0; f < 6; ++f) {
                buf[f].resize(static_cast<std::size_t>(lx) * ly * (lz + 2));
                for (int z = 0; z < lz + 2; ++z)
                    for (int y = 0; y < ly; ++y)
                        for (int x = 0; x < lx; ++x)
                            buf[f][(static_cast<std::size_t>(z) * ly + y) * lx + x] = (*src[f])[x][y][z];
            }
            check(lbm_load_fields_ghosted(h_, buf[0].data(), buf[1].data(), buf[2].data(), buf[3].data(),
                                          buf[4].data(), buf[5].data()),
                  "InamuroSolver: upload");
        }

        ~GpuInamuro() override
        {
            if (h_) lbm_destroy(h_);
        }

        GpuInamuro(const GpuInamuro&) = delete;
        GpuInamuro& operator=(const GpuInamuro&) = delete;

        // Inamuro::performTimeStep (CPU/Inamuro.cpp:347-363) on the device.
        void performTimeStep() override
        {
            lbm_step_stats st{};
            check(lbm_step(h_, 1, &st), "performTimeStep");
            auto& d = last_pressure_solve_diagnostics;
            d.pressure_solve_call_count += 1;
            d.prev_iteration_count = d.iteration_count;
            d.iteration_count = st.iterations;
            d.hit_max_iterations = st.converged == 0;
            d.pressure_solve_time_ms = st.device_ms;
            host_stale_ = true;
        }

        // The reference's writer, on fields refreshed from the device.
        void writeResults(int timeStep) override
        {
            download();
            Inamuro::writeResults(timeStep);
        }

        lbm_handle* handle() const { return h_; }

    private:
        void download()
        {
            if (!host_stale_) return;
            std::vector<double> buf(static_cast<std::size_t>(lx) * ly * (lz + 2));
            Vector3D* dst[6] = {&fei, &rho, &u, &v, &w, &p};
            for (int f = 0; f < 6; ++f) {
                check(lbm_download_ghosted(h_, static_cast<lbm_field>(f), buf.data()), "download");
                for (int z = 0; z < lz + 2; ++z)
                    for (int y = 0; y < ly; ++y)
                        for (int x = 0; x < lx; ++x)
                            (*dst[f])[x][y][z] = buf[(static_cast<std::size_t>(z) * ly + y) * lx + x];
            }
            host_stale_ = false;
        }

        void check(lbm_status s, const char* what) const
        {
            if (s == LBM_OK) return;
            const std::string msg = std::string(what) + ": " + (h_ ? lbm_last_error(h_) : lbm_last_error(nullptr));
            if (s == LBM_ERR_BAD_ARG) throw std::invalid_argument(msg);
            throw std::runtime_error(msg);
        }

        lbm_handle* h_ = nullptr;
        bool host_stale_ = false;
    };

    // CPU/InamuroSolver.cpp:116-219: line 3 = steps, line 4 = output
    // frequency, then key=value lines ('#' starts a comment).
    void loadConfiguration(const std::string& filename)
    {
        std::ifstream file(filename);
        if (!file) {
            std::cerr << "warning: cannot open " << filename << ", default solver settings" << std::endl;
            return;
        }
        std::string line;
        std::getline(file, line);
        std::getline(file, line);
        file >> max_time_steps_ >> output_frequency_;
        std::getline(file, line);
        while (std::getline(file, line)) {
            const std::size_t hash = line.find('#');
            if (hash != std::string::npos) line = line.substr(0, hash);
            const std::size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            const std::string key = trim(line.substr(0, eq));
            const std::string value = trim(line.substr(eq + 1));
            if (!key.empty()) setOption(key, value);
        }
    }

    static std::string trim(const std::string& s)
    {
        const std::size_t a = s.find_first_not_of(" \t\r\n");
        if (a == std::string::npos) return "";
        return s.substr(a, s.find_last_not_of(" \t\r\n") - a + 1);
    }

    void setOption(const std::string& key, const std::string& value)
    {
        const bool on = value == "1" || value == "true" || value == "TRUE" || value == "on" || value == "ON";
        if (key == "enable_timing") config_.enable_timing = on;
        else if (key == "enable_progress") config_.enable_progress = on;
        else if (key == "enable_tecplot_output") config_.enable_tecplot_output = on;
        else if (key == "enable_debug_field_csv") config_.enable_debug_field_csv = on;
        else if (key == "enable_step_summary_csv") config_.enable_step_summary_csv = on;
        else if (key == "enable_basic_warnings") config_.enable_basic_warnings = on;
        else if (key == "output_dir") config_.output_dir = value;
        else if (key == "step_summary_filename") config_.step_summary_filename = value;
    }

    void applyOutputConfiguration()
    {
        Inamuro::OutputConfig oc;
        oc.enable_tecplot = config_.enable_tecplot_output;
        oc.enable_debug_field_csv = config_.enable_debug_field_csv;
        oc.enable_step_summary_csv = config_.enable_step_summary_csv;
        oc.output_dir = config_.output_dir;
        oc.summary_filename = config_.step_summary_filename;
        inamuro_->setOutputConfig(oc);
    }

    // One writer per file: a lock directory beside it, as the reference does
    // (CPU/InamuroSolver.cpp:233-262); a second process writes no diagnostics.
    void openDiagnosticsFile()
    {
        if (!config_.enable_step_summary_csv) return;
        std::filesystem::create_directories(config_.output_dir);
        const std::filesystem::path path = std::filesystem::path(config_.output_dir) / config_.step_summary_filename;
        lock_dir_ = path;
        lock_dir_ += ".lock";
        std::error_code ec;
        if (!std::filesystem::create_directory(lock_dir_, ec)) {
            std::cerr << "warning: " << path << " is held by another run; no step diagnostics" << std::endl;
            lock_dir_.clear();
            return;
        }
        csv_ = std::make_unique<lbm_b200::StepDiagnosticsCsv>(path.string());
    }

    void releaseDiagnosticsLock()
    {
        csv_.reset();
        if (!lock_dir_.empty()) {
            std::error_code ec;
            std::filesystem::remove(lock_dir_, ec);
            lock_dir_.clear();
        }
    }

    void recordStepDiagnostics(int time_step, double step_ms)
    {
        if (!csv_) return;
        const auto& pd = inamuro_->last_pressure_solve_diagnostics;
        lbm_b200::PressureSolveColumns ps;
        ps.call_count = static_cast<uint64_t>(pd.pressure_solve_call_count);
        ps.prev_iterations = pd.prev_iteration_count;
        ps.iterations = pd.iteration_count;
        ps.hit_max_iterations = pd.hit_max_iterations;
        ps.solve_ms = pd.pressure_solve_time_ms;
        const lbm_diagnostics d = csv_->record(inamuro_->handle(), time_step, step_ms, ps);
        if (!config_.enable_basic_warnings) return;
        // CPU/InamuroSolver.cpp:339-370: first NaN/Inf and first negative density
        const lbm_field_stats* all[7] = {&d.rho, &d.fei, &d.u, &d.v, &d.w, &d.velocity_magnitude, &d.p};
        bool non_finite = false;
        for (const lbm_field_stats* f : all) non_finite = non_finite || f->nan_count > 0 || f->inf_count > 0;
        if (non_finite && !warned_non_finite_) {
            warned_non_finite_ = true;
            std::cerr << "\n[warning] step " << time_step << ": first NaN/Inf, see step_diagnostics.csv" << std::endl;
        }
        if (d.rho.min < 0.0 && !warned_negative_rho_) {
            warned_negative_rho_ = true;
            std::cerr << "\n[warning] step " << time_step << ": first negative density, rho_min=" << d.rho.min
                      << std::endl;
        }
    }

    std::unique_ptr<GpuInamuro> inamuro_;
    SolverConfig config_;
    int max_time_steps_ = 20;
    int output_frequency_ = 10;
    double init_ms_ = 0.0;
    std::unique_ptr<lbm_b200::StepDiagnosticsCsv> csv_;
    std::filesystem::path lock_dir_;
    bool warned_non_finite_ = false;
    bool warned_negative_rho_ = false;
};
