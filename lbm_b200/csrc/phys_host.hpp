// phys_host.hpp -- host-side derivation of a box's physical constants from
// its lbm_params (shared by the single-box and the batched C ABI).
#pragma once

#include <cmath>

#include "../../include/lbm_b200.h"
#include "lbm_solver.cuh"

namespace lbm {

inline bool is_pow2(double t)
{
    if (!(t > 0.0) || !std::isfinite(t)) return false;
    int e = 0;
    return std::frexp(t, &e) == 0.5;
}

inline Phys make_phys(const lbm_params& p)
{
    Phys P{};
    P.rho_L = p.rho_L;
    P.rho_G = p.rho_G;
    P.mu_G = p.mu_G;
    P.mu_slope = (p.mu_L - p.mu_G) / (p.rho_L - p.rho_G);
    P.tauf = p.tauf;
    P.taug = p.taug;
    P.k_f = p.k_f;
    P.k_g = p.k_g;
    P.T = p.T;
    P.a = p.a;
    P.b = p.b;
    P.fei_L = p.fei_L;
    P.fei_G = p.fei_G;
    P.fei_avg = (p.fei_L + p.fei_G) / 2.0;
    P.dfei = p.fei_L - p.fei_G;
    P.half_drho = (p.rho_L - p.rho_G) / 2.0;
    P.visc = 1.5 * (p.taug - 0.5) * 2.0;
    P.tauf_pow2 = is_pow2(p.tauf);
    P.taug_pow2 = is_pow2(p.taug);
    P.inv_tauf = 1.0 / p.tauf;
    P.inv_taug = 1.0 / p.taug;
    return P;
}

}  // namespace lbm
