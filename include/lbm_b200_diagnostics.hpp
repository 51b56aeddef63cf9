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

}  // namespace lbm_b200
