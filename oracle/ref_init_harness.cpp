// ref_init_harness.cpp -- constructs the UNMODIFIED reference GPU-tree
// Inamuro (GPU/Inamuro.cpp + GPU/common.cpp of UniBoy222/LBM, compiled from
// their own sources by oracle/Makefile into oracle/_ref/) from a params file
// and dumps the initial macro fields.  It pins the params.in parser (both
// key=value styles) and the droplet initial condition (GPU/Inamuro.cpp:24-115,
// 491-566).
//
// TEST INFRASTRUCTURE ONLY.
//
// usage: ref_init_harness PARAMS OUT.bin
//   OUT.bin: phi rho u v w p, N doubles each, x fastest, no ghost layers,
//   followed by the six ghost planes z=0 and z=lz+1 of each field
//   (6 * 2 * lx*ly doubles), then 16 doubles of parsed parameters:
//   lx ly lz rho_L rho_G mu_L mu_G tauf taug k_f k_g T a b fei_L fei_G.
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "Inamuro.hpp"

namespace {
class Harness : public Inamuro {
public:
    explicit Harness(const std::string& params) : Inamuro(params) {}
    void dump(const std::string& path) const
    {
        const long N = static_cast<long>(lx) * ly * lz;
        const long plane = static_cast<long>(lx) * ly;
        std::vector<double> buf;
        buf.reserve(6 * N + 12 * plane + 16);
        const Vector3D* src[6] = {&fei, &rho, &u, &v, &w, &p};
        for (int f = 0; f < 6; ++f)
            for (int z = 0; z < lz; ++z)
                for (int y = 0; y < ly; ++y)
                    for (int x = 0; x < lx; ++x) buf.push_back((*src[f])[x][y][z + 1]);
        for (int f = 0; f < 6; ++f)
            for (int zg : {0, lz + 1})
                for (int y = 0; y < ly; ++y)
                    for (int x = 0; x < lx; ++x) buf.push_back((*src[f])[x][y][zg]);
        const double prm[16] = {double(lx), double(ly), double(lz), params.rho_L, params.rho_G,
                                params.mu_L, params.mu_G, params.tauf, params.taug,
                                params.k_f, params.k_g, params.T, params.a, params.b,
                                params.fei_L, params.fei_G};
        buf.insert(buf.end(), prm, prm + 16);
        std::ofstream out(path, std::ios::binary);
        out.write(reinterpret_cast<const char*>(buf.data()), buf.size() * sizeof(double));
    }
};
}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::cerr << "usage: ref_init_harness PARAMS OUT.bin\n";
        return 2;
    }
    Harness h(argv[1]);
    h.dump(argv[2]);
    return 0;
}
