// params.cpp -- params.in parser and droplet initial condition (host only).
//
// Format (kept because it is the drop-in contract):
//   14 whitespace-separated positional entries, normally one group per line
//   (CPU/Inamuro.cpp:38-53):
//     lx ly lz | period | t_max | Nwri | rho_L rho_G | tauf taug | mu_L mu_G |
//     k_f k_g | T | a | b | fei_max fei_min | fei_L fei_G | DD
//   then any number of key=value items.  Whitespace tokens containing '=' set
//   the initial-condition keys of the GPU tree (GPU/Inamuro.cpp:56-103); the
//   CPU tree's line-wise output switches (enable_*=, output_dir=,
//   step_summary_filename=, '#' comments; CPU/InamuroSolver.cpp:143-218) are
//   accepted and ignored here, since they steer file output, not the step.
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "../../include/lbm_b200.h"

extern "C" void lbm_params_default(lbm_params* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    // Inamuro(int nx = 48, int ny = 96, int nz = 128), GPU/Inamuro.hpp:81
    o->lx = 48; o->ly = 96; o->lz = 128;
    // Parameters defaults, GPU/Inamuro.hpp:38-67
    o->period = 1;
    o->t_max = 20;   // InamuroSolver::max_time_steps, CPU/InamuroSolver.hpp:49
    o->nwri = 10;    // InamuroSolver::output_frequency, CPU/InamuroSolver.hpp:50
    o->rho_L = 50.0; o->rho_G = 1.0;
    o->mu_L = 0.008; o->mu_G = 0.00016;
    o->tauf = 1.0; o->taug = 1.0;
    o->k_f = 0.5; o->k_g = 0.0005;
    o->fei_L = 0.092; o->fei_G = 0.015;
    o->fei_max = 0.09714; o->fei_min = 0.01134;
    o->DD = 32.0;
    o->T = 0.035; o->a = 1.0; o->b = 6.7;
    o->init_single_droplet = 0;
    o->init_tanh = 0;
    o->init_velocity = 0.035;
    o->interface_width = 2.0;
    o->init_center_x = -1.0; o->init_center_y = -1.0; o->init_center_z = -1.0;
    o->init_separation = -1.0;
    o->init_offset_x = 0.0;
    o->periodic_x = 0;
}

namespace {

bool parse_double(const std::string& s, double& out)
{
    if (s.empty()) return false;
    char* end = nullptr;
    out = std::strtod(s.c_str(), &end);
    return end && *end == '\0';
}

}  // namespace

extern "C" lbm_status lbm_params_load(const char* path, lbm_params* o)
{
    if (!path || !o) return LBM_ERR_BAD_ARG;
    lbm_params_default(o);
    std::ifstream file(path);
    if (!file.is_open()) return LBM_ERR_IO;
    int lx, ly, lz, period, t_max, nwri;
    double v[16];
    if (!(file >> lx >> ly >> lz >> period >> t_max >> nwri)) return LBM_ERR_BAD_ARG;
    for (double& x : v)
        if (!(file >> x)) return LBM_ERR_BAD_ARG;
    o->lx = lx; o->ly = ly; o->lz = lz;
    o->period = period; o->t_max = t_max; o->nwri = nwri;
    o->rho_L = v[0]; o->rho_G = v[1];
    o->tauf = v[2]; o->taug = v[3];
    o->mu_L = v[4]; o->mu_G = v[5];
    o->k_f = v[6]; o->k_g = v[7];
    o->T = v[8]; o->a = v[9]; o->b = v[10];
    o->fei_max = v[11]; o->fei_min = v[12];
    o->fei_L = v[13]; o->fei_G = v[14];
    o->DD = v[15];
    // Everything after DD is scanned as whitespace tokens.
    std::string token;
    while (file >> token) {
        const std::size_t pos = token.find('=');
        if (pos == std::string::npos) continue;
        const std::string key = token.substr(0, pos);
        const std::string value = token.substr(pos + 1);
        double d = 0.0;
        auto num = [&](double& dst) -> bool {
            if (!parse_double(value, d)) return false;
            dst = d;
            return true;
        };
        if (key == "init_mode") {
            // Unknown modes fall back to two_droplets (GPU/Inamuro.cpp:550-554).
            o->init_single_droplet = (value == "single_droplet") ? 1 : 0;
        } else if (key == "init_profile") {
            // Unknown profiles fall back to sharp (GPU/Inamuro.cpp:534-538).
            o->init_tanh = (value == "tanh") ? 1 : 0;
        } else if (key == "init_velocity") {
            if (!num(o->init_velocity)) return LBM_ERR_BAD_ARG;
        } else if (key == "interface_width") {
            if (!num(o->interface_width)) return LBM_ERR_BAD_ARG;
        } else if (key == "init_center_x") {
            if (!num(o->init_center_x)) return LBM_ERR_BAD_ARG;
        } else if (key == "init_center_y") {
            if (!num(o->init_center_y)) return LBM_ERR_BAD_ARG;
        } else if (key == "init_center_z") {
            if (!num(o->init_center_z)) return LBM_ERR_BAD_ARG;
        } else if (key == "init_separation") {
            if (!num(o->init_separation)) return LBM_ERR_BAD_ARG;
        } else if (key == "init_offset_x") {
            if (!num(o->init_offset_x)) return LBM_ERR_BAD_ARG;
        } else if (key == "boundary_x") {
            // Not a reference key: periodic x instead of the slip walls.
            if (value == "periodic") o->periodic_x = 1;
            else if (value == "slip") o->periodic_x = 0;
            else return LBM_ERR_BAD_ARG;
        }
        // Any other key (the CPU tree's output switches) is ignored.
    }
    if (o->lx < 2 || o->ly < 1 || o->lz < 1) return LBM_ERR_BAD_ARG;
    return LBM_OK;
}

namespace {

// place_droplet of GPU/Inamuro.cpp:499-533: liquid fraction from a sharp or
// tanh profile; a cell takes the droplet's values only where this raises phi.
void place_droplet(const lbm_params& p, double cx, double cy, double cz, double vz,
                   double* phi, double* rho, double* w)
{
    const double radius = p.DD / 2.0;
    const bool use_tanh = p.init_tanh != 0;
    const double iw = (p.interface_width > 0.0) ? p.interface_width : 2.0;
    const long plane = static_cast<long>(p.lx) * p.ly;
    for (int x = 0; x < p.lx; ++x)
        for (int y = 0; y < p.ly; ++y)
            for (int z = 1; z < p.lz + 1; ++z) {
                const double dx = x - cx;
                const double dy = y - cy;
                const double dz = (z - 1) - cz;
                const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                double frac = 0.0;
                if (use_tanh)
                    frac = 0.5 * (1.0 - std::tanh((r - radius) / iw));
                else if (r < radius)
                    frac = 1.0;
                if (frac > 0.0) {
                    const long c = static_cast<long>(z - 1) * plane + static_cast<long>(y) * p.lx + x;
                    const double local = p.fei_min + frac * (p.fei_max - p.fei_min);
                    if (local > phi[c]) {
                        phi[c] = local;
                        rho[c] = p.rho_G + frac * (p.rho_L - p.rho_G);
                        w[c] = vz * frac;
                    }
                }
            }
}

}  // namespace

extern "C" lbm_status lbm_init_droplets(const lbm_params* p, double* phi, double* rho,
                                        double* u, double* v, double* w, double* pr)
{
    if (!p || !phi || !rho || !u || !v || !w || !pr) return LBM_ERR_BAD_ARG;
    if (p->lx < 2 || p->ly < 1 || p->lz < 1) return LBM_ERR_BAD_ARG;
    const long n = static_cast<long>(p->lx) * p->ly * p->lz;
    // Background of initializeArrays (CPU/Inamuro.cpp:518-524).
    for (long i = 0; i < n; ++i) {
        phi[i] = p->fei_min;
        rho[i] = p->rho_G;
        u[i] = v[i] = w[i] = pr[i] = 0.0;
    }
    // GPU/Inamuro.cpp:540-565
    const double cy_default = p->ly / 2.0;
    const double cz_default = p->lz / 2.0;
    if (p->init_single_droplet) {
        const double cx = (p->init_center_x >= 0.0) ? p->init_center_x : p->lx / 2.0;
        const double cy = (p->init_center_y >= 0.0) ? p->init_center_y : cy_default;
        const double cz = (p->init_center_z >= 0.0) ? p->init_center_z : cz_default;
        place_droplet(*p, cx, cy, cz, p->init_velocity, phi, rho, w);
        return LBM_OK;
    }
    const double cx = (p->init_center_x >= 0.0) ? p->init_center_x : 0.0;
    const double cy = (p->init_center_y >= 0.0) ? p->init_center_y : cy_default;
    const double sep = (p->init_separation >= 0.0) ? p->init_separation : p->DD;
    const double cx1 = cx - 0.5 * p->init_offset_x;
    const double cx2 = cx + 0.5 * p->init_offset_x;
    const double cz1 = (p->init_center_z >= 0.0) ? p->init_center_z + sep : cz_default + sep;
    const double cz2 = (p->init_center_z >= 0.0) ? p->init_center_z - sep : cz_default - sep;
    place_droplet(*p, cx1, cy, cz1, -p->init_velocity, phi, rho, w);
    place_droplet(*p, cx2, cy, cz2, p->init_velocity, phi, rho, w);
    return LBM_OK;
}
