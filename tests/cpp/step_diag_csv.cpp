// Writes step_diagnostics.csv for a small droplet box through
// lbm_b200_diagnostics.hpp (rows for steps 0, 1, 2) and dumps the final six
// fields as raw doubles, for tests/test_gpu_diagnostics.py.
//   step_diag_csv <out.csv> <fields.bin> <precision 0|1>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "lbm_b200.h"
#include "lbm_b200_diagnostics.hpp"

int main(int argc, char** argv)
{
    if (argc != 4) return 2;
    lbm_params p;
    lbm_params_default(&p);
    p.lx = 24;
    p.ly = 20;
    p.lz = 16;
    p.DD = 8.0;
    p.init_single_droplet = 1;
    p.init_tanh = 1;
    const size_t n = static_cast<size_t>(p.lx) * p.ly * p.lz;
    std::vector<double> f[6];
    for (auto& v : f) v.resize(n);
    if (lbm_init_droplets(&p, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(), f[5].data()) != LBM_OK)
        return 3;
    lbm_handle* h = nullptr;
    if (lbm_create(&p, static_cast<lbm_precision>(std::atoi(argv[3])), 0, &h) != LBM_OK) return 4;
    if (lbm_load_fields(h, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(), f[5].data()) != LBM_OK)
        return 5;
    lbm_poisson_cfg cfg = {100, 1e-3, 0, 60000, 1};
    lbm_set_poisson(h, &cfg);
    lbm_b200::StepDiagnosticsCsv csv(argv[1]);
    csv.record(h, 0, 0.0, {});
    uint64_t prev = 0;
    for (int s = 1; s <= 2; ++s) {
        lbm_step_stats st;
        if (lbm_step(h, 1, &st) != LBM_OK) return 6;
        lbm_b200::PressureSolveColumns ps;
        ps.call_count = static_cast<uint64_t>(s);
        ps.prev_iterations = prev;
        ps.iterations = st.iterations;
        ps.hit_max_iterations = st.converged == 0;
        ps.solve_ms = st.device_ms;
        csv.record(h, s, st.device_ms, ps);
        prev = st.iterations;
    }
    FILE* fo = std::fopen(argv[2], "wb");
    if (!fo) return 7;
    std::vector<double> buf(n);
    for (int k = 0; k < 6; ++k) {
        if (lbm_download(h, static_cast<lbm_field>(k), buf.data()) != LBM_OK) return 8;
        std::fwrite(buf.data(), sizeof(double), n, fo);
    }
    std::fclose(fo);
    lbm_destroy(h);
    return 0;
}
