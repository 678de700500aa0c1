// tangent.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// FP64 tangent-linear oracle: the templated restatement of the reference
// solver (cavity_oracle.hpp) instantiated on forward-mode dual numbers.  One
// run gives J and its directional derivative dJ . v for a direction v in
// (hot-wall theta profile, Cs), where J is the mean hot-wall Nusselt number
// (src/uniform/post.rs:68-78) over the states after s steps, s in [ws, N].
#include <cmath>

#include "cavity_oracle.h"
#include "cavity_oracle.hpp"

namespace orc {

struct Dual {
    double v, d;
    Dual(double x = 0.0, double dx = 0.0) : v(x), d(dx) {}
};
inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) { return Dual(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
inline Dual operator+(double a, Dual b) { return Dual(a) + b; }
inline Dual operator+(Dual a, double b) { return a + Dual(b); }
inline Dual operator-(double a, Dual b) { return Dual(a) - b; }
inline Dual operator-(Dual a, double b) { return a - Dual(b); }
inline Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
inline Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
inline Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
inline Dual operator/(double a, Dual b) { return Dual(a) / b; }
inline double val(Dual x) { return x.v; }
// sqrt(pi:pi) at pi = 0 takes the derivative 0 (the same subgradient the
// device adjoint uses).
inline Dual dsqrt(Dual x) {
    double s = std::sqrt(x.v);
    return Dual(s, s > 0.0 ? x.d / (2.0 * s) : 0.0);
}

}  // namespace orc

extern "C" int orc_tl_nusselt(const orc_params* cp, int64_t n_steps, int64_t ws, const double* dtheta, double dcs,
                              double* J, double* dJ) {
    using orc::Dual;
    orc::Params p;
    p.nx = cp->nx;
    p.ny = cp->ny;
    p.ra = cp->ra;
    p.pr = cp->pr;
    p.cs = cp->cs;
    p.pr_t = cp->pr_t;
    p.utarget = cp->utarget;
    p.seed = cp->seed;
    p.jobs = cp->jobs;
    p.alpha_mult = cp->alpha_mult;
    p.nu_start_mult = cp->nu_start_mult;
    p.has_nu_override = cp->has_nu_override;
    p.nu_override = cp->nu_override;
    p.init_mode = cp->init_mode;
    p.noise_amp = cp->noise_amp;
    p.geq_order = cp->geq_order;
    p.t_hot_profile = cp->t_hot_profile;
    p.t_cold = cp->t_cold;
    orc::Solver<Dual> s;
    s.init(p);
    if (s.error) return s.error;
    orc::RowPool* pool = nullptr;
    if (p.jobs > 1) {
        pool = new orc::RowPool(p.jobs);
        s.pool = pool;
    }
    for (int iy = 0; iy < p.ny; ++iy) s.t_hot[iy].d = dtheta ? dtheta[iy] : 0.0;
    s.cs.d = dcs;
    Dual acc(0.0, 0.0);
    for (int64_t t = 1; t <= n_steps; ++t) {
        s.step();
        if (t >= ws) acc = acc + s.nusselt_hot();
    }
    const double nw = double(n_steps - ws + 1);
    *J = acc.v / nw;
    *dJ = acc.d / nw;
    delete pool;
    return 0;
}
