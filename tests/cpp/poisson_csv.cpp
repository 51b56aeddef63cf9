// Writes a Poisson CSV of two synthetic check records through
// include/lbm_b200_diagnostics.hpp (lbm_b200::PoissonCsv), for
// tests/test_tecplot.py.   poisson_csv <out.csv>
#include <cmath>

#include "lbm_b200_diagnostics.hpp"

int main(int argc, char** argv)
{
    if (argc != 2) return 2;
    lbm_b200::PoissonCsv csv(argv[1]);
    lbm_check_record r{};
    r.step = 3;
    r.iteration = 200;
    r.pressure_l1_delta = 0.25;
    r.pressure_l1_norm = 4.0;
    r.relative_error = 0.0625;
    r.fixed_point_h_l1 = r.fixed_point_h_scale = r.fixed_point_h_relative = std::nan("");
    r.fixed_point_p_l1 = r.fixed_point_p_scale = r.fixed_point_p_relative = std::nan("");
    r.fixed_point_relative = std::nan("");
    r.block_low_frequency_fraction = std::nan("");
    lbm_b200::PoissonCsv::on_check(&csv, &r);
    r.iteration = 300;
    r.fixed_point_h_l1 = 1.5;
    r.fixed_point_relative = 0.5;
    r.fixed_point_evaluated = 1;
    r.converged = 1;
    r.pressure_converged = 1;
    r.block_low_frequency_fraction = 0.125;
    r.spatial_block_size = 4;
    r.spatial_block_count = 27;
    lbm_b200::PoissonCsv::on_check(&csv, &r);
    return 0;
}
