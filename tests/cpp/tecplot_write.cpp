// Writes the Tecplot binary file of six fields through
// include/lbm_b200_tecplot.hpp, for tests/test_tecplot.py.
//   tecplot_write <lx> <ly> <lz> <fields.bin: phi rho u v w p, n doubles each> <out.plt>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "lbm_b200_tecplot.hpp"

int main(int argc, char** argv)
{
    if (argc != 6) return 2;
    const int lx = std::atoi(argv[1]), ly = std::atoi(argv[2]), lz = std::atoi(argv[3]);
    const size_t n = static_cast<size_t>(lx) * ly * lz;
    std::vector<double> buf(6 * n);
    std::FILE* f = std::fopen(argv[4], "rb");
    if (!f || std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) return 3;
    std::fclose(f);
    const double* d = buf.data();
    return lbm_b200::write_tecplot_binary(argv[5], lx, ly, lz, d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, d + 5 * n)
               ? 0 : 4;
}
