// Dot-product test of the per-node reverse (cfd_cavity_b200/csrc/node_ad.h):
// <J v, w> computed by forward-mode dual numbers through node_forward must
// equal <v, J^T w> computed by node_reverse, for random inputs, random input
// directions v and random output adjoints w.  Built by the tests with g++.
#include <cmath>
#include <cstdint>
#include <random>

#include "../../cfd_cavity_b200/csrc/node_ad.h"

struct D {
    double v, d;
    D(double x = 0.0, double dx = 0.0) : v(x), d(dx) {}
};
static D operator+(D a, D b) { return D(a.v + b.v, a.d + b.d); }
static D operator-(D a, D b) { return D(a.v - b.v, a.d - b.d); }
static D operator-(D a) { return D(-a.v, -a.d); }
static D operator*(D a, D b) { return D(a.v * b.v, a.d * b.v + a.v * b.d); }
static D operator/(D a, D b) { return D(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
namespace cav {
namespace ad {
template <>
D sqrt_<D>(D x) {
    double s = std::sqrt(x.v);
    return D(s, s > 0 ? x.d / (2.0 * s) : 0.0);
}
}  // namespace ad
}  // namespace cav

extern "C" int node_ad_check(int trials, uint32_t seed, int wall_mode, int zero_pi, double* max_rel) {
    using namespace cav::ad;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    double worst = 0.0;
    for (int t = 0; t < trials; ++t) {
        NodeScal<double> c{1e-4 * (1 + U(rng)), 0.01 * (1.5 + U(rng)), 0.013 * (1.5 + U(rng)),
                           1.5 / (0.53 + 0.02 * U(rng)), 1.0 / 0.9, 3.0 / 16.0, (t % 3 == 0) ? 0.0 : 1.0};
        NodeScal<D> cd{D(c.beta), D(c.nu), D(c.alpha), D(c.c1), D(c.inv_pr_t), D(c.lambda), D(c.q2)};
        const bool wall = wall_mode == 2 ? (t % 2 == 0) : wall_mode == 1;
        double h[9], g[9], vh[9], vg[9];
        const double u0x = 0.05 * U(rng), u0y = 0.05 * U(rng), rho = 1.0 + 0.01 * U(rng), T0 = 0.4 * U(rng);
        for (int i = 0; i < 9; ++i) {
            double eu = cx(i) * u0x + cy(i) * u0y;
            double feq = wd(i) * rho * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * (u0x * u0x + u0y * u0y));
            h[i] = feq - wd(i) + (zero_pi ? 0.0 : 1e-3 * U(rng));
            g[i] = wd(i) * T0 * (1 + 3 * eu) + 1e-3 * U(rng);
            vh[i] = U(rng);
            vg[i] = U(rng);
        }
        if (zero_pi) {  // f exactly at equilibrium of (rho, u): pi_neq = 0
            for (int i = 0; i < 9; ++i) {
                double eu = cx(i) * u0x + cy(i) * u0y;
                h[i] = wd(i) * (rho - 1.0) + wd(i) * rho * (3 * eu + 4.5 * eu * eu - 1.5 * (u0x * u0x + u0y * u0y));
            }
        }
        const double fyp = 1e-4 * U(rng), cs = 0.1 + 0.02 * U(rng);
        const double vfyp = U(rng), vcs = U(rng);
        double af[9], ag[9];
        for (int i = 0; i < 9; ++i) {
            af[i] = U(rng);
            ag[i] = U(rng);
        }
        const double afy = U(rng), at = U(rng);
        // tangent-linear
        D hd[9], gd[9], hod[9], god[9];
        for (int i = 0; i < 9; ++i) {
            hd[i] = D(h[i], vh[i]);
            gd[i] = D(g[i], vg[i]);
        }
        D td;
        D fyd = node_forward<D>(hd, gd, D(fyp, vfyp), wall, D(cs, vcs), cd, hod, god, &td);
        double jv = fyd.d * afy + td.d * at;
        for (int i = 0; i < 9; ++i) jv += hod[i].d * af[i] + god[i].d * ag[i];
        // adjoint
        double ah[9], agi[9], afyp;
        double bcs = node_reverse<double>(h, g, fyp, wall, cs, c, af, ag, afy, at, ah, agi, &afyp);
        double vjt = vfyp * afyp + vcs * bcs;
        for (int i = 0; i < 9; ++i) vjt += vh[i] * ah[i] + vg[i] * agi[i];
        double rel = std::fabs(jv - vjt) / std::fmax(std::fabs(jv), 1e-30);
        if (rel > worst) worst = rel;
    }
    *max_rel = worst;
    return 0;
}
