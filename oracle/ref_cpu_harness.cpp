// ref_cpu_harness.cpp -- drives the UNMODIFIED reference CPU solver
// (CPU/Inamuro.cpp + CPU/common.cpp of UniBoy222/LBM, compiled from their own
// sources by oracle/Makefile into oracle/_ref/) and dumps raw FP64 state.
//
// TEST INFRASTRUCTURE ONLY: it pins the oracle restatement (tests/golden) and
// is the timed reference CPU baseline of bench.py.  It is never linked into
// the product.
//
// The reference keeps function-local statics (CPU/Inamuro.cpp:150,254,627),
// so one process runs exactly one case.
//
// Modes
//   run:    --params F --steps S --out DIR [--init FIELDS.bin] [--dump-h]
//           Writes DIR/init.bin, DIR/step%04d.bin (phi rho u v w p, N doubles
//           each, x fastest, no ghost layers) and DIR/summary.txt
//           ("step sweeps ms" per line).
//   tecplot: --params F --tecplot DIR --init FIELDS.bin
//           Writes the reference's own Tecplot binary file of the loaded
//           fields (Inamuro::writeTecplotBinary, step 0) into DIR.
//   sample: --params F --sample-sweeps K --out DIR [--init FIELDS.bin] [--sample-reps R]
//           [--nonpoisson-reps M]
//           R times (default 1): times one non-Poisson step part (collision,
//           stream, bounce, moments; only in the first M reps, default all)
//           and K kinetic Poisson sweeps (collision_p, stream, bounce, getp)
//           on the box of F; writes DIR/sample.txt ("cells N", then
//           "rep i nonpoisson_ms sweeps_ms", nonpoisson_ms -1 where skipped).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <string>
#include <vector>
#include <array>
#include <cmath>

// The sweep pieces (collision_p, getp) are private members of the reference
// class; this translation unit alone sees them as protected so the harness
// subclass can time them.  The reference sources themselves are compiled as-is.
#define private protected
#include "Inamuro.hpp"
#undef private

namespace {

class Harness : public Inamuro {
public:
    explicit Harness(const std::string& params) : Inamuro(params) {}

    long cells() const { return static_cast<long>(lx) * ly * lz; }

    void loadFields(const std::vector<double>& buf)
    {
        const long N = cells();
        Vector3D* dst[6] = {&fei, &rho, &u, &v, &w, &p};
        for (int f = 0; f < 6; ++f)
            for (int z = 0; z < lz; ++z)
                for (int y = 0; y < ly; ++y)
                    for (int x = 0; x < lx; ++x)
                        (*dst[f])[x][y][z + 1] = buf[f * N + (static_cast<long>(z) * ly + y) * lx + x];
    }

    void dumpFields(const std::string& path) const
    {
        const long N = cells();
        std::vector<double> buf(6 * N);
        const Vector3D* src[6] = {&fei, &rho, &u, &v, &w, &p};
        for (int f = 0; f < 6; ++f)
            for (int z = 0; z < lz; ++z)
                for (int y = 0; y < ly; ++y)
                    for (int x = 0; x < lx; ++x)
                        buf[f * N + (static_cast<long>(z) * ly + y) * lx + x] = (*src[f])[x][y][z + 1];
        writeRaw(path, buf);
    }

    void dumpH(const std::string& path) const
    {
        const long N = cells();
        std::vector<double> buf(15 * N);
        for (int q = 0; q < 15; ++q)
            for (int z = 0; z < lz; ++z)
                for (int y = 0; y < ly; ++y)
                    for (int x = 0; x < lx; ++x)
                        buf[q * N + (static_cast<long>(z) * ly + y) * lx + x] = hh[q][x][y][z];
        writeRaw(path, buf);
    }

    void writeTecplot(const std::string& dir)
    {
        OutputConfig oc = getOutputConfig();
        oc.output_dir = dir + "/";
        setOutputConfig(oc);
        writeTecplotBinary(0);
    }

    std::uint64_t lastSweeps() const { return getLastPressureSolveDiagnostics().iteration_count; }

    // One non-Poisson part of performTimeStep (CPU/Inamuro.cpp:350-355).
    void nonPoissonPart()
    {
        collision();
        stream(ff);
        stream(gg);
        applyBoundaryConditions(ff);
        applyBoundaryConditions(gg);
        getMacro();
    }

    // One kinetic sweep of the Poisson loop (CPU/Inamuro.cpp:679-686).
    void sweep()
    {
        collision_p();
        stream(hh);
        applyBoundaryConditions(hh);
        getp();
    }

    static void writeRaw(const std::string& path, const std::vector<double>& buf)
    {
        std::ofstream out(path, std::ios::binary);
        if (!out) throw std::runtime_error("cannot write " + path);
        out.write(reinterpret_cast<const char*>(buf.data()), buf.size() * sizeof(double));
    }
};

std::vector<double> readRaw(const std::string& path, long count)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot read " + path);
    std::vector<double> buf(count);
    in.read(reinterpret_cast<char*>(buf.data()), count * sizeof(double));
    if (in.gcount() != static_cast<std::streamsize>(count * sizeof(double)))
        throw std::runtime_error("short read " + path);
    return buf;
}

}  // namespace

int main(int argc, char** argv)
{
    std::string params, out, init;
    int steps = 0;
    long sample_sweeps = -1;
    int sample_reps = 1;
    int nonpoisson_reps = -1;
    std::string tecplot_dir;
    bool dump_h = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
            return argv[++i];
        };
        if (a == "--params") params = val();
        else if (a == "--steps") steps = std::stoi(val());
        else if (a == "--out") out = val();
        else if (a == "--init") init = val();
        else if (a == "--sample-sweeps") sample_sweeps = std::stol(val());
        else if (a == "--sample-reps") sample_reps = std::stoi(val());
        else if (a == "--nonpoisson-reps") nonpoisson_reps = std::stoi(val());
        else if (a == "--tecplot") tecplot_dir = val();
        else if (a == "--dump-h") dump_h = true;
        else {
            std::cerr << "unknown argument " << a << "\n";
            return 2;
        }
    }
    if (!params.empty() && !tecplot_dir.empty()) {
        try {
            Harness h(params);
            if (!init.empty()) h.loadFields(readRaw(init, 6 * h.cells()));
            h.writeTecplot(tecplot_dir);
        } catch (const std::exception& e) {
            std::cerr << "ref_cpu_harness error: " << e.what() << "\n";
            return 1;
        }
        return 0;
    }
    if (params.empty() || out.empty()) {
        std::cerr << "usage: ref_cpu_harness --params F --out DIR (--steps S | --sample-sweeps K) [--init B]\n";
        return 2;
    }
    try {
        Harness h(params);
        if (!init.empty()) h.loadFields(readRaw(init, 6 * h.cells()));
        using clk = std::chrono::steady_clock;
        if (sample_sweeps >= 0) {
            std::ofstream s(out + "/sample.txt");
            s.precision(17);
            s << "cells " << h.cells() << "\n";
            for (int r = 0; r < sample_reps; ++r) {
                const bool np = nonpoisson_reps < 0 || r < nonpoisson_reps;
                const auto t0 = clk::now();
                if (np) h.nonPoissonPart();
                const auto t1 = clk::now();
                for (long k = 0; k < sample_sweeps; ++k) h.sweep();
                const auto t2 = clk::now();
                s << "rep " << r << " "
                  << (np ? std::chrono::duration<double, std::milli>(t1 - t0).count() : -1.0) << " "
                  << std::chrono::duration<double, std::milli>(t2 - t1).count() << "\n";
                s.flush();
            }
            return 0;
        }
        h.dumpFields(out + "/init.bin");
        std::ofstream summary(out + "/summary.txt");
        for (int s = 1; s <= steps; ++s) {
            const auto t0 = clk::now();
            h.performTimeStep();
            const auto t1 = clk::now();
            char name[64];
            std::snprintf(name, sizeof(name), "/step%04d.bin", s);
            h.dumpFields(out + name);
            if (dump_h) {
                std::snprintf(name, sizeof(name), "/h%04d.bin", s);
                h.dumpH(out + name);
            }
            summary << s << " " << h.lastSweeps() << " "
                    << std::chrono::duration<double, std::milli>(t1 - t0).count() << "\n";
            summary.flush();
        }
    } catch (const std::exception& e) {
        std::cerr << "ref_cpu_harness error: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
