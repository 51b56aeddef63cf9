// lbm_b200_diagnostics.hpp -- the reference's per-step diagnostics file over
// the C ABI (lbm_diagnostics_snapshot), header-only C++.
//
// StepDiagnosticsCsv writes step_diagnostics.csv with the columns and number
// format of InamuroSolver (CPU/InamuroSolver.cpp:262-334): a header row, then
// one row per recorded step: time_step, the step's timing and pressure-solve
// counters, and min, max, mean, abs_max, nan_count, inf_count of rho, fei, u,
// v, w, the velocity magnitude and p (Inamuro::collectDiagnostics,
// CPU/Inamuro.cpp:412-507), computed on the device.
#pragma once

#include <cmath>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <stdexcept>
#include <string>

#include "lbm_b200.h"

namespace lbm_b200 {

// The pressure-solve columns of a row (Inamuro::PressureSolveDiagnostics).
struct PressureSolveColumns {
    uint64_t call_count = 0;        // pressure solves so far
    uint64_t prev_iterations = 0;   // sweeps of the previous solve
    uint64_t iterations = 0;        // sweeps of this solve
    bool hit_max_iterations = false;
    double solve_ms = 0.0;
};

class StepDiagnosticsCsv
{
public:
    explicit StepDiagnosticsCsv(const std::string& path) : out_(path)
    {
        if (!out_) throw std::runtime_error("cannot open diagnostics file " + path);
        out_ << std::scientific << std::setprecision(10);
        out_ << "time_step"
             << ",step_time_ms,pressure_solve_call_count,prev_pressure_iterations,pressure_iterations,"
                "pressure_hit_max_iter,pressure_solve_ms";
        static const char* names[7] = {"rho", "fei", "u", "v", "w", "vel_mag", "p"};
        for (const char* n : names)
            out_ << ',' << n << "_min," << n << "_max," << n << "_mean," << n << "_abs_max," << n << "_nan_count,"
                 << n << "_inf_count";
        out_ << '\n';
    }

    // One row for the handle's current fields; returns the statistics.  Time
    // step 0 (the initial state) writes zeros in the timing and solve
    // columns, as the reference.
    lbm_diagnostics record(lbm_handle* h, int time_step, double step_time_ms, const PressureSolveColumns& ps)
    {
        lbm_diagnostics d;
        const lbm_status s = lbm_diagnostics_snapshot(h, &d);
        if (s != LBM_OK) throw std::runtime_error(std::string("lbm_diagnostics_snapshot: ") + lbm_last_error(h));
        out_ << time_step;
        if (time_step == 0)
            out_ << ",0,0,0,0,0,0";
        else
            out_ << ',' << step_time_ms << ',' << ps.call_count << ',' << ps.prev_iterations << ',' << ps.iterations
                 << ',' << (ps.hit_max_iterations ? 1 : 0) << ',' << ps.solve_ms;
        const lbm_field_stats* st[7] = {&d.rho, &d.fei, &d.u, &d.v, &d.w, &d.velocity_magnitude, &d.p};
        for (const lbm_field_stats* f : st)
            out_ << ',' << f->min << ',' << f->max << ',' << f->mean << ',' << f->abs_max << ',' << f->nan_count << ','
                 << f->inf_count;
        out_ << '\n';
        out_.flush();
        return d;
    }

private:
    std::ofstream out_;
};

// The per-check Poisson CSV of the reference's GPU program
// (setPoissonDiagnosticsPath, GPU/InamuroCUDA.cu:2610-2682): its header and
// one row per convergence check, fed by lbm_set_check_callback.  Usable with
// any handle of the C ABI:
//   lbm_b200::PoissonCsv csv("poisson.csv");
//   lbm_set_check_callback(h, &lbm_b200::PoissonCsv::on_check, &csv);
// Columns that a check did not evaluate (NaN in the record) are left empty,
// as the reference leaves them.
class PoissonCsv {
public:
    PoissonCsv() = default;
    explicit PoissonCsv(const std::string& path) { open(path); }

    // Creates (truncates) the file and writes the header; "" disables.
    void open(const std::string& path)
    {
        path_ = path;
        if (path.empty()) return;
        std::ofstream out(path);
        if (!out) throw std::runtime_error("failed to open Poisson diagnostics CSV: " + path);
        out << "step,iteration,pressure_l1_delta,pressure_l1_norm,relative_error,"
            << "fixed_point_h_l1,fixed_point_h_scale,fixed_point_h_relative,"
            << "fixed_point_p_l1,fixed_point_p_scale,fixed_point_p_relative,"
            << "fixed_point_relative,fixed_point_evaluated,pressure_converged,fixed_point_converged,"
            << "dual_residual_enabled,converged,block_low_frequency_fraction,"
            << "block_size,block_count\n";
    }
    const std::string& path() const { return path_; }

    // Appends one check row.
    void append(const lbm_check_record& r) const
    {
        if (path_.empty()) return;
        std::ofstream out(path_, std::ios::app);
        if (!out) return;
        out << r.step << ',' << r.iteration << ',' << std::setprecision(17) << r.pressure_l1_delta << ','
            << r.pressure_l1_norm << ',' << r.relative_error << ',';
        const double opt[7] = {r.fixed_point_h_l1, r.fixed_point_h_scale, r.fixed_point_h_relative,
                               r.fixed_point_p_l1, r.fixed_point_p_scale, r.fixed_point_p_relative,
                               r.fixed_point_relative};
        for (double v : opt) {
            if (std::isfinite(v)) out << v;
            out << ',';
        }
        out << r.fixed_point_evaluated << ',' << r.pressure_converged << ',' << r.fixed_point_converged << ','
            << r.dual_residual_enabled << ',' << r.converged << ',';
        if (std::isfinite(r.block_low_frequency_fraction)) out << r.block_low_frequency_fraction;
        out << ',' << r.spatial_block_size << ',' << r.spatial_block_count << '\n';
    }

    // lbm_check_callback adaptor: user is the PoissonCsv.
    static void on_check(void* user, const lbm_check_record* r)
    {
        if (user && r) static_cast<const PoissonCsv*>(user)->append(*r);
    }

private:
    std::string path_;
};

}  // namespace lbm_b200
