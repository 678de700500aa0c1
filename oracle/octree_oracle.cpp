// octree_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// FP64 restatement of the reference's block-refined (octree) cavity solver,
// molecular and dynamic mixed-scale SGS paths: src/octree/grid.rs (tables),
// src/octree/interface.rs (coarse <-> fine transfers), src/octree/lbm.rs,
// src/octree/cavity.rs (per-level physics, block-aware streaming and
// boundary conditions, diagnostics) and src/octree/solver.rs (CavitySolver::
// new, init_cavity, step_cavity, noise_stats), src/octree/smag.rs (the
// dynamic model, shared with the uniform restatement: dynamic_sgs_grid).
// Same arithmetic conventions and parity status as cavity_oracle.hpp.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "cavity_oracle.h"
#include "cavity_oracle.hpp"

namespace orc {
namespace oct {

using Pop = std::array<double, Q>;

// LbmLevel, src/octree/lbm.rs:19-53.
struct Level {
    int nx = 0, ny = 0;
    std::vector<Pop> f, g;
    std::vector<double> rho, ux, uy, temp;
    void alloc(int x, int y) {
        nx = x;
        ny = y;
        f.assign(size_t(x) * y, Pop{});
        g.assign(size_t(x) * y, Pop{});
        rho.assign(size_t(x) * y, 0.0);
        ux.assign(size_t(x) * y, 0.0);
        uy.assign(size_t(x) * y, 0.0);
        temp.assign(size_t(x) * y, 0.0);
    }
};

// RelaxTimes::from_nu_alpha, src/octree/lbm.rs:90-98.
struct Relax {
    double tp, tm, tt;
    static Relax from(double nu, double al) {
        Relax r;
        r.tp = 0.5 + 3.0 * nu;
        r.tm = 0.5 + LAMBDA_TRT / (r.tp - 0.5);
        r.tt = 0.5 + 3.0 * al;
        return r;
    }
};

struct Xi {
    double even, odd, th;
};

// rescaling_factors_multilevel, src/octree/interface.rs:112-131.
static Xi xi_multilevel(const Relax& c, const Relax& f, int substeps, bool odd_exact) {
    const double dt = 1.0 / double(substeps);
    Xi x;
    x.even = dt * f.tp / c.tp;
    x.odd = odd_exact ? dt * f.tm / c.tm : dt;
    x.th = dt * f.tt / c.tt;
    return x;
}

struct GhostE {
    int k;
    int kc[4];
    double w[4];
};
struct CoinE {
    int kc;
    int kf[9];
    double w[9];
};

// bilinear_stencil, src/octree/grid.rs:218-229 (clamped base).
static void bilinear(double x, double y, int nx0, int ny0, int kc[4], double w[4]) {
    long ix = (long)std::floor(x), iy = (long)std::floor(y);
    ix = std::min<long>(std::max<long>(ix, 0), nx0 - 2);
    iy = std::min<long>(std::max<long>(iy, 0), ny0 - 2);
    double fx = x - double(ix), fy = y - double(iy);
    kc[0] = int(iy * nx0 + ix);
    w[0] = (1.0 - fx) * (1.0 - fy);
    kc[1] = int(iy * nx0 + ix + 1);
    w[1] = fx * (1.0 - fy);
    kc[2] = int((iy + 1) * nx0 + ix);
    w[2] = (1.0 - fx) * fy;
    kc[3] = int((iy + 1) * nx0 + ix + 1);
    w[3] = fx * fy;
}

// OctreeGrid::build, src/octree/grid.rs:103-204.
struct Grid {
    int nx0, ny0, bx0, by0, bx1, by1, nx1, ny1;
    std::vector<GhostE> ghosts;
    std::vector<CoinE> coin;
    void build(int nx0_, int ny0_, int bx0_, int by0_, int bx1_, int by1_, bool wl, bool wr, bool wb, bool wt) {
        nx0 = nx0_;
        ny0 = ny0_;
        bx0 = bx0_;
        by0 = by0_;
        bx1 = bx1_;
        by1 = by1_;
        const int fw = bx1 - bx0, fh = by1 - by0;
        nx1 = 2 * fw + 3;
        ny1 = 2 * fh + 3;
        ghosts.clear();
        coin.clear();
        for (int b = 0; b < ny1; ++b)
            for (int a = 0; a < nx1; ++a)
                if (a == 0 || b == 0 || a == nx1 - 1 || b == ny1 - 1) {
                    GhostE e;
                    e.k = b * nx1 + a;
                    bilinear(double(bx0) - 0.5 + 0.5 * a, double(by0) - 0.5 + 0.5 * b, nx0, ny0, e.kc, e.w);
                    ghosts.push_back(e);
                }
        for (int cy = by0; cy < by1; ++cy)
            for (int cx = bx0; cx < bx1; ++cx) {
                if (cx == 0 || cx + 1 == nx0 || cy == 0 || cy + 1 == ny0) continue;
                if ((wl && cx == bx0) || (wr && cx + 1 == bx1) || (wb && cy == by0) || (wt && cy + 1 == by1)) continue;
                const int a = 2 * (cx - bx0) + 1, b = 2 * (cy - by0) + 1;
                const double ww[3] = {0.25, 0.5, 0.25};
                CoinE e;
                e.kc = cy * nx0 + cx;
                int idx = 0;
                for (int jb = 0; jb < 3; ++jb)
                    for (int ja = 0; ja < 3; ++ja) {
                        e.kf[idx] = (b + jb - 1) * nx1 + (a + ja - 1);
                        e.w[idx] = ww[ja] * ww[jb];
                        ++idx;
                    }
                coin.push_back(e);
            }
    }
};

// split_odd_even / rescale_fneq / rescale_fneq_inverse, interface.rs:68-102.
static Pop rescale(const Pop& fneq, const Xi& xi) {
    Pop out;
    for (int i = 0; i < Q; ++i) {
        const int o = OPP[i];
        const double even = 0.5 * (fneq[i] + fneq[o]);
        const double odd = 0.5 * (fneq[i] - fneq[o]);
        out[i] = xi.even * even + xi.odd * odd;
    }
    return out;
}
static Pop rescale_inv(const Pop& fneq, const Xi& xi) {
    Pop out;
    for (int i = 0; i < Q; ++i) {
        const int o = OPP[i];
        const double even = 0.5 * (fneq[i] + fneq[o]);
        const double odd = 0.5 * (fneq[i] - fneq[o]);
        out[i] = even / xi.even + odd / xi.odd;
    }
    return out;
}

// coarse_to_fine, interface.rs:137-170, then refresh_moments :209-227.
static void coarse_to_fine(const Grid& gr, const Level& c, Level& f, const Xi& xi, int geq_order) {
    for (const GhostE& gh : gr.ghosts) {
        double rho = 0, ux = 0, uy = 0, t = 0;
        for (int s = 0; s < 4; ++s) {
            rho += gh.w[s] * c.rho[gh.kc[s]];
            ux += gh.w[s] * c.ux[gh.kc[s]];
            uy += gh.w[s] * c.uy[gh.kc[s]];
            t += gh.w[s] * c.temp[gh.kc[s]];
        }
        Pop fn{}, gn{};
        for (int i = 0; i < Q; ++i)
            for (int s = 0; s < 4; ++s) {
                const int k = gh.kc[s];
                fn[i] += gh.w[s] * (c.f[k][i] - feq<double>(i, c.rho[k], c.ux[k], c.uy[k]));
                gn[i] += gh.w[s] * (c.g[k][i] - geq<double>(i, c.temp[k], c.ux[k], c.uy[k], geq_order));
            }
        const Pop fr = rescale(fn, xi);
        for (int i = 0; i < Q; ++i) {
            f.f[gh.k][i] = feq<double>(i, rho, ux, uy) + fr[i];
            f.g[gh.k][i] = geq<double>(i, t, ux, uy, geq_order) + xi.th * gn[i];
        }
    }
    for (const GhostE& gh : gr.ghosts) {
        const int k = gh.k;
        double rho = 0, mx = 0, my = 0, t = 0;
        for (int i = 0; i < Q; ++i) {
            const double fi = f.f[k][i];
            rho += fi;
            mx += fi * double(CX[i]);
            my += fi * double(CY[i]);
            t += f.g[k][i];
        }
        f.rho[k] = rho;
        f.ux[k] = mx / rho;
        f.uy[k] = my / rho;
        f.temp[k] = t;
    }
}

// fine_to_coarse, interface.rs:175-206.
static void fine_to_coarse(const Grid& gr, const Level& f, Level& c, const Xi& xi, int geq_order) {
    for (const CoinE& ce : gr.coin) {
        double rho = 0, ux = 0, uy = 0, t = 0;
        for (int s = 0; s < 9; ++s) {
            rho += ce.w[s] * f.rho[ce.kf[s]];
            ux += ce.w[s] * f.ux[ce.kf[s]];
            uy += ce.w[s] * f.uy[ce.kf[s]];
            t += ce.w[s] * f.temp[ce.kf[s]];
        }
        Pop fa{}, ga{};
        for (int i = 0; i < Q; ++i)
            for (int s = 0; s < 9; ++s) {
                const int k = ce.kf[s];
                fa[i] += ce.w[s] * (f.f[k][i] - feq<double>(i, f.rho[k], f.ux[k], f.uy[k]));
                ga[i] += ce.w[s] * (f.g[k][i] - geq<double>(i, f.temp[k], f.ux[k], f.uy[k], geq_order));
            }
        const Pop fg = rescale_inv(fa, xi);
        for (int i = 0; i < Q; ++i) {
            c.f[ce.kc][i] = feq<double>(i, rho, ux, uy) + fg[i];
            c.g[ce.kc][i] = geq<double>(i, t, ux, uy, geq_order) + ga[i] / xi.th;
        }
    }
}

// refresh_moments_nodes, src/octree/solver.rs:1183-1206.
static void refresh_nodes(Level& l, const std::vector<int>& nodes) {
    for (int k : nodes) {
        double rho = 0, mx = 0, my = 0, t = 0;
        for (int i = 0; i < Q; ++i) {
            const double fi = l.f[k][i];
            rho += fi;
            mx += double(CX[i]) * fi;
            my += double(CY[i]) * fi;
            t += l.g[k][i];
        }
        l.rho[k] = rho;
        l.temp[k] = t;
        if (rho > std::numeric_limits<double>::epsilon()) {
            l.ux[k] = mx / rho;
            l.uy[k] = my / rho;
        } else {
            l.ux[k] = 0.0;
            l.uy[k] = 0.0;
        }
    }
}

// collide_node_cavity, src/octree/cavity.rs:70-150.  With nut / at (the
// dynamic model's per-node nu_t / alpha_t) the relaxation times are rebuilt
// per node (:100-110); without, the level's.
static void collide_node(Pop& fn, Pop& gn, double& fy_out, double r, double u, double v, double temp,
                         const Relax& tau_l, double beta, int geq_order, const double* nut = nullptr,
                         const double* at = nullptr) {
    const double fyv = r * beta * 1.0 * (temp - 0.0);
    fy_out = fyv;
    Pop feq_, geq_;
    for (int i = 0; i < Q; ++i) {
        feq_[i] = feq<double>(i, r, u, v);
        geq_[i] = geq<double>(i, temp, u, v, geq_order);
    }
    Relax tau = tau_l;
    if (nut && at) {
        tau.tp = 0.5 + 3.0 * (tau_l.tp - 0.5) / 3.0 + 3.0 * *nut;
        tau.tm = 0.5 + LAMBDA_TRT / (tau.tp - 0.5);
        tau.tt = 0.5 + 3.0 * (tau_l.tt - 0.5) / 3.0 + 3.0 * *at;
    }
    const double a_f = 0.5 * (1.0 / tau.tp + 1.0 / tau.tm);
    const double b_f = 0.5 * (1.0 / tau.tp - 1.0 / tau.tm);
    const double a_g = 1.0 / tau.tt;
    const double b_g = 0.0;
    Pop d_f, d_g;
    for (int i = 0; i < Q; ++i) {
        d_f[i] = fn[i] - feq_[i];
        d_g[i] = gn[i] - geq_[i];
    }
    for (int i = 0; i < Q; ++i) {
        const double cx = CX[i], cy = CY[i];
        const int o = OPP[i];
        const double ei_u = cx * u + cy * v;
        const double s_i = W[i] * ((cy - v) / CS2 + ei_u * cy / (CS2 * CS2)) * fyv;
        const double s_minus = W[i] * (cy / CS2) * fyv;
        const double s_plus = s_i - s_minus;
        fn[i] = fn[i] + (-a_f * d_f[i] - b_f * d_f[o] + (1.0 - 0.5 / tau.tm) * s_minus +
                         (1.0 - 0.5 / tau.tp) * s_plus);
    }
    for (int i = 0; i < Q; ++i) gn[i] = gn[i] + (-a_g * d_g[i] - b_g * d_g[OPP[i]]);
}

// collide_cavity, cavity.rs:167-245.
static void collide_level(Level& l, const Relax& tau, double beta, std::vector<double>& fy, bool interior,
                          int geq_order, const std::vector<double>* nut = nullptr,
                          const std::vector<double>* at = nullptr) {
    const int x0 = interior ? 1 : 0, x1 = interior ? l.nx - 1 : l.nx;
    const int y0 = interior ? 1 : 0, y1 = interior ? l.ny - 1 : l.ny;
    for (int iy = y0; iy < y1; ++iy)
        for (int ix = x0; ix < x1; ++ix) {
            const int k = iy * l.nx + ix;
            collide_node(l.f[k], l.g[k], fy[k], l.rho[k], l.ux[k], l.uy[k], l.temp[k], tau, beta, geq_order,
                         nut ? &(*nut)[k] : nullptr, at ? &(*at)[k] : nullptr);
        }
}

// mean_field, src/octree/solver.rs:1176-1178 (sequential sum).
static double mean_field(const std::vector<double>& v) {
    double s = 0.0;
    for (double x : v) s += x;
    return s / double(v.size());
}

// update_macroscopic_guo, cavity.rs:252-325.
static void macro_guo(Level& l, const std::vector<double>& fy) {
    for (int k = 0; k < l.nx * l.ny; ++k) {
        double rho = 0, mx = 0, my = 0, t = 0;
        for (int i = 0; i < Q; ++i) {
            const double fi = l.f[k][i];
            rho += fi;
            mx += double(CX[i]) * fi;
            my += double(CY[i]) * fi;
            t += l.g[k][i];
        }
        l.rho[k] = rho;
        l.temp[k] = t;
        if (rho > std::numeric_limits<double>::epsilon()) {
            l.ux[k] = mx / rho;
            l.uy[k] = my / rho + 0.5 * fy[k] / rho;
        } else {
            l.ux[k] = 0.0;
            l.uy[k] = 0.0;
        }
    }
}

// stream (lbm.rs:152-180) and stream_cavity_block (cavity.rs:393-495).
static void stream_plain(Level& l) {
    const std::vector<Pop> fo = l.f, go = l.g;
    for (int iy = 0; iy < l.ny; ++iy)
        for (int ix = 0; ix < l.nx; ++ix) {
            const int k = iy * l.nx + ix;
            for (int i = 0; i < Q; ++i) {
                const int sx = ix - CX[i], sy = iy - CY[i];
                if (sx >= 0 && sx < l.nx && sy >= 0 && sy < l.ny) {
                    l.f[k][i] = fo[sy * l.nx + sx][i];
                    l.g[k][i] = go[sy * l.nx + sx][i];
                } else {
                    l.f[k][i] = fo[k][OPP[i]];
                    l.g[k][i] = go[k][i];
                }
            }
        }
}
static void stream_block(Level& l, bool wl, bool wr, bool wb, bool wt) {
    const std::vector<Pop> fo = l.f, go = l.g;
    const int nx = l.nx, ny = l.ny;
    for (int iy = 1; iy < ny - 1; ++iy)
        for (int ix = 1; ix < nx - 1; ++ix) {
            const int k = iy * nx + ix;
            for (int i = 0; i < Q; ++i) {
                const int sx = ix - CX[i], sy = iy - CY[i];
                const bool wall_src =
                    (sx == 0 && wl) || (sx == nx - 1 && wr) || (sy == 0 && wb) || (sy == ny - 1 && wt);
                if (wall_src) {
                    l.f[k][i] = fo[k][OPP[i]];
                    l.g[k][i] = go[k][i];
                } else {
                    l.f[k][i] = fo[sy * nx + sx][i];
                    l.g[k][i] = go[sy * nx + sx][i];
                }
            }
        }
}

// apply_thermal_boundary_conditions (cavity.rs:501-534) and the block
// variant (:543-605).
static void thermal_bc(Level& l, int geq_order) {
    const int nx = l.nx, ny = l.ny;
    for (int iy = 0; iy < ny; ++iy) {
        for (int i = 0; i < Q; ++i) l.g[iy * nx][i] = geq<double>(i, T_HOT, 0.0, 0.0, geq_order);
        for (int i = 0; i < Q; ++i) l.g[iy * nx + nx - 1][i] = geq<double>(i, T_COLD, 0.0, 0.0, geq_order);
    }
    for (int ix = 0; ix < nx; ++ix) {
        l.g[ix] = l.g[nx + ix];
        l.g[(ny - 1) * nx + ix] = l.g[(ny - 2) * nx + ix];
    }
}
static void thermal_bc_block(Level& l, bool hot, bool cold, int geq_order) {
    const int nx = l.nx, ny = l.ny;
    for (int iy = 0; iy < ny; ++iy) {
        if (hot)
            for (int i = 0; i < Q; ++i) l.g[iy * nx + 1][i] = geq<double>(i, T_HOT, 0.0, 0.0, geq_order);
        if (cold)
            for (int i = 0; i < Q; ++i) l.g[iy * nx + nx - 2][i] = geq<double>(i, T_COLD, 0.0, 0.0, geq_order);
    }
    for (int ix = 1; ix < nx - 1; ++ix) {
        l.g[nx + ix] = l.g[2 * nx + ix];
        l.g[(ny - 2) * nx + ix] = l.g[(ny - 3) * nx + ix];
    }
    for (int iy = 0; iy < ny; ++iy) {
        l.g[iy * nx] = l.g[iy * nx + 1];
        l.g[iy * nx + nx - 1] = l.g[iy * nx + nx - 2];
    }
    for (int ix = 0; ix < nx; ++ix) {
        l.g[ix] = l.g[nx + ix];
        l.g[(ny - 1) * nx + ix] = l.g[(ny - 2) * nx + ix];
    }
}

// enforce_wall_velocity (cavity.rs:609-626) and the block variant (:632-656).
static void noslip(Level& l) {
    for (int iy = 0; iy < l.ny; ++iy)
        for (int ix : {0, l.nx - 1}) l.ux[iy * l.nx + ix] = l.uy[iy * l.nx + ix] = 0.0;
    for (int iy : {0, l.ny - 1})
        for (int ix = 0; ix < l.nx; ++ix) l.ux[iy * l.nx + ix] = l.uy[iy * l.nx + ix] = 0.0;
}
static void noslip_block(Level& l, bool hot, bool cold) {
    for (int iy = 0; iy < l.ny; ++iy) {
        if (hot) l.ux[iy * l.nx + 1] = l.uy[iy * l.nx + 1] = 0.0;
        if (cold) l.ux[iy * l.nx + l.nx - 2] = l.uy[iy * l.nx + l.nx - 2] = 0.0;
    }
    for (int iy : {1, l.ny - 2})
        for (int ix = 0; ix < l.nx; ++ix) l.ux[iy * l.nx + ix] = l.uy[iy * l.nx + ix] = 0.0;
}

struct Sub {
    Grid grid;
    Level lvl;
    Relax tau;
    Xi xi_down;
    std::vector<double> fy;
    std::vector<double> nut, at;  // nu_t_pre / alpha_t_pre of the dynamic model
};
struct Block {
    Grid grid;
    Level fine;
    std::vector<double> fy;
    std::vector<double> nut, at;
    bool hot, cold;
    bool has_sub = false;
    Sub sub;
};

// CavitySolver (octree), src/octree/solver.rs:284-947.
struct Octree {
    int nx0, ny0, levels, geq_order = 2;
    Level coarse;
    std::vector<Block> blocks;
    Relax tau_c, tau_f;
    Xi xi;
    double nu, alpha, beta_c, beta_f, nu_start_mult;
    long spin_up, time_step = 0;
    std::vector<double> fy_c;
    int error = 0;
    bool odd_exact = false;
    // dynamic mixed-scale SGS (set_dynamic_sgs, src/octree/solver.rs:476-481)
    bool dynamic_smag = false;
    double smag_alpha = 0.5, nu_sm_min = -0.1, eta_test = 2.0;
    std::vector<double> nut_c, at_c;
    double cs_dyn_mean = 0.0, cs_dyn_max = 0.0, kappa_dyn_mean = 0.0, kappa_dyn_max = 0.0, nu_t_max = 0.0;

    void init(int nx0_, int ny0_, int blw, double ra, double pr, double utarget, uint64_t seed, bool odd_exact_,
              int levels_, double nu_start_mult_, int has_nu, double nu_over) {
        error = 0;
        if (blw < 2 || 2 * blw >= nx0_ || (levels_ != 2 && levels_ != 3) || ny0_ < 4) {
            error = 1;
            return;
        }
        nx0 = nx0_;
        ny0 = ny0_;
        levels = levels_;
        odd_exact = odd_exact_;
        const double lz = double(ny0 - 1);
        const double nu_cal = std::pow(utarget * std::sqrt(pr) * lz / (1.7 * std::sqrt(ra)), 2.0 / 3.0);
        nu = has_nu ? nu_over : std::fmax(nu_cal, 0.002);
        alpha = nu / pr;
        beta_c = ra * nu * alpha / (lz * lz * lz);
        beta_f = 0.5 * beta_c;
        tau_c = Relax::from(nu, alpha);
        tau_f = Relax::from(2.0 * nu, 2.0 * alpha);
        const Relax tau_s = Relax::from(4.0 * nu, 4.0 * alpha);
        xi = xi_multilevel(tau_c, tau_f, 2, odd_exact);
        const Xi xi_sub = xi_multilevel(tau_f, tau_s, 2, odd_exact);
        coarse.alloc(nx0, ny0);
        fy_c.assign(size_t(nx0) * ny0, 0.0);
        nut_c.assign(size_t(nx0) * ny0, 0.0);
        at_c.assign(size_t(nx0) * ny0, 0.0);
        blocks.clear();
        const int spec[2][4] = {{0, blw, 1, 0}, {nx0 - 1 - blw, nx0 - 1, 0, 1}};
        for (auto& sp : spec) {
            Block b;
            b.grid.build(nx0, ny0, sp[0], 0, sp[1], ny0 - 1, false, false, false, false);
            b.fine.alloc(b.grid.nx1, b.grid.ny1);
            b.fy.assign(size_t(b.grid.nx1) * b.grid.ny1, 0.0);
            b.nut.assign(size_t(b.grid.nx1) * b.grid.ny1, 0.0);
            b.at.assign(size_t(b.grid.nx1) * b.grid.ny1, 0.0);
            b.hot = sp[2];
            b.cold = sp[3];
            if (levels >= 3) {
                b.has_sub = true;
                const int sbx0 = b.hot ? 1 : b.grid.nx1 - 4, sbx1 = b.hot ? 3 : b.grid.nx1 - 2;
                b.sub.grid.build(b.grid.nx1, b.grid.ny1, sbx0, 1, sbx1, b.grid.ny1 - 2, true, false, true, false);
                b.sub.lvl.alloc(b.sub.grid.nx1, b.sub.grid.ny1);
                b.sub.tau = tau_s;
                b.sub.xi_down = xi_sub;
                b.sub.fy.assign(size_t(b.sub.grid.nx1) * b.sub.grid.ny1, 0.0);
                b.sub.nut.assign(size_t(b.sub.grid.nx1) * b.sub.grid.ny1, 0.0);
                b.sub.at.assign(size_t(b.sub.grid.nx1) * b.sub.grid.ny1, 0.0);
            }
            blocks.push_back(std::move(b));
        }
        nu_start_mult = std::max(nu_start_mult_, 1.0);
        spin_up = std::max<long>(ny0 / 10, 2000);
        time_step = 0;
        init_cavity(seed);
    }

    // init_cavity, src/octree/solver.rs:504-578.
    void init_cavity(uint64_t seed) {
        Rng rng(seed);
        for (int iy = 0; iy < ny0; ++iy)
            for (int ix = 0; ix < nx0; ++ix) {
                const int k = iy * nx0 + ix;
                const double xf = double(ix) / double(nx0 - 1);
                const double t_lin = T_HOT + (T_COLD - T_HOT) * xf;
                const double pert = 1.0e-3 * (2.0 * rng.next_f64() - 1.0);
                const double t = t_lin + pert;
                coarse.rho[k] = 1.0;
                coarse.ux[k] = 0.0;
                coarse.uy[k] = 0.0;
                coarse.temp[k] = t;
                for (int i = 0; i < Q; ++i) {
                    coarse.f[k][i] = feq<double>(i, 1.0, 0.0, 0.0);
                    coarse.g[k][i] = geq<double>(i, t, 0.0, 0.0, geq_order);
                }
            }
        auto interp_t = [&](double x, double y) {
            int kc[4];
            double w[4];
            bilinear(x, y, nx0, ny0, kc, w);
            double t = 0.0;
            for (int s = 0; s < 4; ++s) t += w[s] * coarse.temp[kc[s]];
            return t;
        };
        auto fill = [&](Level& l, int k, double t) {
            l.rho[k] = 1.0;
            l.ux[k] = 0.0;
            l.uy[k] = 0.0;
            l.temp[k] = t;
            for (int i = 0; i < Q; ++i) {
                l.f[k][i] = feq<double>(i, 1.0, 0.0, 0.0);
                l.g[k][i] = geq<double>(i, t, 0.0, 0.0, geq_order);
            }
        };
        for (Block& b : blocks) {
            for (int yb = 0; yb < b.grid.ny1; ++yb)
                for (int a = 0; a < b.grid.nx1; ++a)
                    fill(b.fine, yb * b.grid.nx1 + a,
                         interp_t(double(b.grid.bx0) - 0.5 + 0.5 * a, double(b.grid.by0) - 0.5 + 0.5 * yb));
            if (b.has_sub) {
                Grid& sg = b.sub.grid;
                for (int b2 = 0; b2 < sg.ny1; ++b2)
                    for (int a2 = 0; a2 < sg.nx1; ++a2) {
                        const double x = double(b.grid.bx0) - 0.5 + 0.5 * (double(sg.bx0) - 0.5 + 0.5 * a2);
                        const double y = double(b.grid.by0) - 0.5 + 0.5 * (double(sg.by0) - 0.5 + 0.5 * b2);
                        fill(b.sub.lvl, b2 * sg.nx1 + a2, interp_t(x, y));
                    }
            }
        }
    }

    // ramp_nu_alpha / ramp_beta_factor, src/octree/solver.rs:596-617.
    void ramp(long step, double& nu_eff, double& al_eff) const {
        if (nu_start_mult == 1.0) {
            nu_eff = nu;
            al_eff = alpha;
            return;
        }
        const double m = 1.0 + (nu_start_mult - 1.0) * std::exp(-double(step) / 1000.0);
        nu_eff = nu * m;
        al_eff = alpha * m;
    }
    double beta_factor(long step) const {
        if (nu_start_mult == 1.0 || step >= spin_up) return 1.0;
        return double(step) / double(spin_up);
    }

    void sub_step(Level& l, const Relax& tau, double beta, std::vector<double>& fy, bool hot, bool cold,
                  const std::vector<double>* nut = nullptr, const std::vector<double>* at = nullptr) {
        collide_level(l, tau, beta, fy, true, geq_order, nut, at);
        stream_block(l, hot, cold, true, true);
        thermal_bc_block(l, hot, cold, geq_order);
        macro_guo(l, fy);
        noslip_block(l, hot, cold);
    }

    // compute_dynamic_sgs_level (src/octree/smag.rs:144-416) of one level:
    // tau = tau_mol, nu / alpha in the level's lattice units.
    void dyn_level(const Level& l, double tau_mol, double nu_l, double al_l, std::vector<double>& nut,
                   std::vector<double>& at, bool stats) {
        DynSgs d = dynamic_sgs_grid(l.nx, l.ny, l.f, l.rho, l.ux, l.uy, l.temp, tau_mol, smag_alpha, eta_test, nu_l,
                                    al_l, nu_sm_min);
        nut = std::move(d.nu_t);
        at = std::move(d.alpha_t);
        if (stats) {
            cs_dyn_mean = d.cnu_mean;
            cs_dyn_max = d.cnu_max;
            kappa_dyn_mean = d.ck_mean;
            kappa_dyn_max = d.ck_max;
        }
    }

    // step_cavity, src/octree/solver.rs:647-947.
    void step() {
        double nu_eff, al_eff;
        ramp(time_step, nu_eff, al_eff);
        const Relax tc = Relax::from(nu_eff, al_eff);
        const Relax tf = Relax::from(2.0 * nu_eff, 2.0 * al_eff);
        const Relax ts = Relax::from(4.0 * nu_eff, 4.0 * al_eff);
        const bool dyn = dynamic_smag;
        if (dyn) {
            // L0 model before the L0 collision, then xi A from the mean
            // effective taus (L1's nu_t of the previous step) (:663-711)
            dyn_level(coarse, 0.5 + 3.0 * nu_eff, nu_eff, al_eff, nut_c, at_c, true);
            const double nt0 = mean_field(nut_c), at0 = mean_field(at_c);
            double nt1 = 0.0, at1 = 0.0;
            for (const Block& b : blocks) {
                nt1 += mean_field(b.nut);
                at1 += mean_field(b.at);
            }
            const double nb = double(blocks.size());
            const Relax tce = Relax::from(nu_eff + nt0, al_eff + at0);
            const Relax tfe = Relax::from(2.0 * nu_eff + nt1 / nb, 2.0 * al_eff + at1 / nb);
            xi = xi_multilevel(tce, tfe, 2, odd_exact);
        }
        const double br = beta_factor(time_step);
        collide_level(coarse, tc, beta_c * br, fy_c, false, geq_order, dyn ? &nut_c : nullptr,
                      dyn ? &at_c : nullptr);
        stream_plain(coarse);
        thermal_bc(coarse, geq_order);
        macro_guo(coarse, fy_c);
        noslip(coarse);
        for (Block& b : blocks) coarse_to_fine(b.grid, coarse, b.fine, xi, geq_order);
        const double bf = beta_f * br, bs = 0.25 * beta_c * br;
        const double tau_mol_l1 = 0.5 + 3.0 * 2.0 * nu_eff, tau_mol_l2 = 0.5 + 3.0 * 4.0 * nu_eff;
        for (Block& b : blocks) {
            if (dyn) dyn_level(b.fine, tau_mol_l1, 2.0 * nu_eff, 2.0 * al_eff, b.nut, b.at, false);
            sub_step(b.fine, tf, bf, b.fy, b.hot, b.cold, dyn ? &b.nut : nullptr, dyn ? &b.at : nullptr);
            if (b.has_sub) {
                if (dyn) {
                    // xi B from L1's fresh and L2's previous nu_t (:808-829)
                    const double nt1b = mean_field(b.nut), at1b = mean_field(b.at);
                    const double nt2 = mean_field(b.sub.nut), at2 = mean_field(b.sub.at);
                    const Relax t1e = Relax::from(2.0 * nu_eff + nt1b, 2.0 * al_eff + at1b);
                    const Relax t2e = Relax::from(4.0 * nu_eff + nt2, 4.0 * al_eff + at2);
                    b.sub.xi_down = xi_multilevel(t1e, t2e, 2, odd_exact);
                }
                coarse_to_fine(b.sub.grid, b.fine, b.sub.lvl, b.sub.xi_down, geq_order);
                for (int sp = 0; sp < 2; ++sp) {
                    if (dyn) dyn_level(b.sub.lvl, tau_mol_l2, 4.0 * nu_eff, 4.0 * al_eff, b.sub.nut, b.sub.at, false);
                    sub_step(b.sub.lvl, ts, bs, b.sub.fy, b.hot, b.cold, dyn ? &b.sub.nut : nullptr,
                             dyn ? &b.sub.at : nullptr);
                }
                fine_to_coarse(b.sub.grid, b.sub.lvl, b.fine, b.sub.xi_down, geq_order);
                std::vector<int> idx;
                for (const CoinE& c : b.sub.grid.coin) idx.push_back(c.kc);
                refresh_nodes(b.fine, idx);
            }
            // the second L1 model takes the unramped nu / alpha (:882-890)
            if (dyn) dyn_level(b.fine, tau_mol_l1, 2.0 * nu, 2.0 * alpha, b.nut, b.at, false);
            sub_step(b.fine, tf, bf, b.fy, b.hot, b.cold, dyn ? &b.nut : nullptr, dyn ? &b.at : nullptr);
            fine_to_coarse(b.grid, b.fine, coarse, xi, geq_order);
        }
        if (dyn) {
            double m = 0.0;
            for (double v : nut_c) m = std::fmax(m, std::fabs(v));
            for (const Block& b : blocks) {
                for (double v : b.nut) m = std::fmax(m, std::fabs(v));
                if (b.has_sub)
                    for (double v : b.sub.nut) m = std::fmax(m, std::fabs(v));
            }
            nu_t_max = m;
        }
        std::vector<int> idx;
        for (const Block& b : blocks)
            for (const CoinE& c : b.grid.coin) idx.push_back(c.kc);
        refresh_nodes(coarse, idx);
        time_step += 1;
    }

    Level* level(int i) {
        if (i == 0) return &coarse;
        if (i <= 2) return &blocks[i - 1].fine;
        if (levels >= 3 && i <= 4) return &blocks[i - 3].sub.lvl;
        return nullptr;
    }
};

}  // namespace oct
}  // namespace orc

using orc::oct::Octree;

extern "C" {

void* orc_oct_create(int32_t nx0, int32_t ny0, int32_t bl_width, double ra, double pr, double utarget,
                     uint64_t seed, int32_t odd_exact, int32_t levels, double nu_start_mult, int32_t has_nu,
                     double nu, int32_t* err) {
    Octree* o = new Octree;
    o->init(nx0, ny0, bl_width, ra, pr, utarget, seed, odd_exact != 0, levels, nu_start_mult, has_nu, nu);
    if (o->error) {
        if (err) *err = o->error;
        delete o;
        return nullptr;
    }
    if (err) *err = 0;
    return o;
}

void orc_oct_destroy(void* h) { delete static_cast<Octree*>(h); }

void orc_oct_step(void* h, int64_t n) {
    Octree* o = static_cast<Octree*>(h);
    for (int64_t i = 0; i < n; ++i) o->step();
}

// Level 0 = L0 (coarse), 1/2 = L1 hot/cold blocks, 3/4 = L2 hot/cold strips.
int32_t orc_oct_level_dims(void* h, int32_t level, int32_t* nx, int32_t* ny) {
    orc::oct::Level* l = static_cast<Octree*>(h)->level(level);
    if (!l) return 1;
    *nx = l->nx;
    *ny = l->ny;
    return 0;
}

int32_t orc_oct_get_level(void* h, int32_t level, double* rho, double* ux, double* uy, double* t, double* f,
                          double* g) {
    orc::oct::Level* l = static_cast<Octree*>(h)->level(level);
    if (!l) return 1;
    const size_t n = size_t(l->nx) * l->ny;
    if (rho) std::memcpy(rho, l->rho.data(), n * 8);
    if (ux) std::memcpy(ux, l->ux.data(), n * 8);
    if (uy) std::memcpy(uy, l->uy.data(), n * 8);
    if (t) std::memcpy(t, l->temp.data(), n * 8);
    if (f) std::memcpy(f, l->f.data(), n * 72);
    if (g) std::memcpy(g, l->g.data(), n * 72);
    return 0;
}

// set_from_snapshot's injection for one level (src/octree/solver.rs:1113-1153)
// followed by that level's no-slip; orc_oct_set_time_step(h, 0) completes a restart.
int32_t orc_oct_restart_level(void* h, int32_t level, const double* rho, const double* ux, const double* uy,
                              const double* t) {
    Octree* o = static_cast<Octree*>(h);
    orc::oct::Level* l = o->level(level);
    if (!l) return 1;
    const size_t n = size_t(l->nx) * l->ny;
    for (size_t k = 0; k < n; ++k) {
        l->rho[k] = rho[k];
        l->ux[k] = ux[k];
        l->uy[k] = uy[k];
        l->temp[k] = t[k];
        for (int i = 0; i < orc::Q; ++i) {
            l->f[k][i] = orc::feq<double>(i, rho[k], ux[k], uy[k]);
            l->g[k][i] = orc::geq<double>(i, t[k], ux[k], uy[k], o->geq_order);
        }
    }
    if (level == 0)
        orc::oct::noslip(*l);
    else
        orc::oct::noslip_block(*l, level == 1 || level == 3, level == 2 || level == 4);
    return 0;
}

void orc_oct_set_time_step(void* h, int64_t t) { static_cast<Octree*>(h)->time_step = t; }

// set_dynamic_sgs, src/octree/solver.rs:476-481 (no validation, as there).
void orc_oct_set_dynamic_sgs(void* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test) {
    Octree* o = static_cast<Octree*>(h);
    o->dynamic_smag = on != 0;
    o->smag_alpha = smag_alpha;
    o->nu_sm_min = nu_sm_min;
    o->eta_test = eta_test;
}

// out: cs_dyn_mean, cs_dyn_max, kappa_dyn_mean, kappa_dyn_max, nu_t_max,
// xi A (even, odd, th), xi B hot (even, odd, th), xi B cold (even, odd, th).
void orc_oct_dynamic_stats(void* h, double* out) {
    Octree* o = static_cast<Octree*>(h);
    out[0] = o->cs_dyn_mean;
    out[1] = o->cs_dyn_max;
    out[2] = o->kappa_dyn_mean;
    out[3] = o->kappa_dyn_max;
    out[4] = o->nu_t_max;
    out[5] = o->xi.even;
    out[6] = o->xi.odd;
    out[7] = o->xi.th;
    for (int b = 0; b < 2; ++b) {
        const bool l3 = o->levels >= 3;
        out[8 + 3 * b] = l3 ? o->blocks[b].sub.xi_down.even : 0.0;
        out[9 + 3 * b] = l3 ? o->blocks[b].sub.xi_down.odd : 0.0;
        out[10 + 3 * b] = l3 ? o->blocks[b].sub.xi_down.th : 0.0;
    }
}

// nu_t_pre and alpha_t_pre of a level (0 = L0, 1/2 = L1 hot/cold, 3/4 = L2).
int32_t orc_oct_get_nut(void* h, int32_t level, double* nut, double* at) {
    Octree* o = static_cast<Octree*>(h);
    const std::vector<double>* a = nullptr;
    const std::vector<double>* b = nullptr;
    if (level == 0) {
        a = &o->nut_c;
        b = &o->at_c;
    } else if (level == 1 || level == 2) {
        a = &o->blocks[level - 1].nut;
        b = &o->blocks[level - 1].at;
    } else if (o->levels >= 3 && (level == 3 || level == 4)) {
        a = &o->blocks[level - 3].sub.nut;
        b = &o->blocks[level - 3].sub.at;
    } else {
        return 1;
    }
    if (nut) std::memcpy(nut, a->data(), a->size() * 8);
    if (at) std::memcpy(at, b->data(), b->size() * 8);
    return 0;
}

// out: nu (L0 lattice), alpha, beta_c, tau+ L0, tau+ L1, tau+ L2, xi_even A,
// xi_odd A, xi_th A, xi_even B, time_step, coincident L0 count, ghost count.
void orc_oct_info(void* h, double* out) {
    Octree* o = static_cast<Octree*>(h);
    out[0] = o->nu;
    out[1] = o->alpha;
    out[2] = o->beta_c;
    out[3] = o->tau_c.tp;
    out[4] = o->tau_f.tp;
    out[5] = o->levels >= 3 ? o->blocks[0].sub.tau.tp : 0.0;
    out[6] = o->xi.even;
    out[7] = o->xi.odd;
    out[8] = o->xi.th;
    out[9] = o->levels >= 3 ? o->blocks[0].sub.xi_down.even : 0.0;
    out[10] = double(o->time_step);
    out[11] = double(o->blocks[0].grid.coin.size() + o->blocks[1].grid.coin.size());
    out[12] = double(o->blocks[0].grid.ghosts.size() + o->blocks[1].grid.ghosts.size());
}

// out: nusselt_hot, nusselt_hot_link0, nusselt_cold (cavity.rs:672-715, Lx
// scale), nusselt_hot_fine (:728-741), max_u over all levels (solver.rs:
// 1005-1016), mass (mean coarse rho), max|rho - rho_bar| all levels and at the
// interfaces (noise_stats, :954-1003), finite (1/0).
void orc_oct_diag(void* h, double* out) {
    Octree* o = static_cast<Octree*>(h);
    const orc::oct::Level& c = o->coarse;
    const int nx = c.nx, ny = c.ny;
    double sh = 0, s0 = 0, sc = 0;
    for (int iy = 0; iy < ny; ++iy) {
        sh += std::fabs(c.temp[iy * nx + 1] - c.temp[iy * nx + 2]);
        s0 += std::fabs(c.temp[iy * nx + 1] - c.temp[iy * nx]);
        sc += std::fabs(c.temp[iy * nx + nx - 2] - c.temp[iy * nx + nx - 3]);
    }
    const double lx = double(nx - 1);
    out[0] = sh / double(ny) * lx / orc::DELTA_T;
    out[1] = s0 / double(ny) * lx / orc::DELTA_T;
    out[2] = sc / double(ny) * lx / orc::DELTA_T;
    const orc::oct::Level& fh = o->blocks[0].fine;
    double sf = 0;
    for (int b = 1; b < fh.ny - 1; ++b) sf += std::fabs(fh.temp[b * fh.nx + 1] - fh.temp[b * fh.nx + 2]) * 2.0;
    out[3] = sf / double(fh.ny - 2) * lx / orc::DELTA_T;
    double mu = 0;
    bool fin = true;
    std::vector<const orc::oct::Level*> lv = {&o->coarse, &o->blocks[0].fine, &o->blocks[1].fine};
    if (o->levels >= 3) {
        lv.push_back(&o->blocks[0].sub.lvl);
        lv.push_back(&o->blocks[1].sub.lvl);
    }
    for (const auto* l : lv)
        for (size_t k = 0; k < l->rho.size(); ++k) {
            mu = std::fmax(mu, std::fmax(std::fabs(l->ux[k]), std::fabs(l->uy[k])));
            fin = fin && std::isfinite(l->rho[k]) && std::isfinite(l->ux[k]) && std::isfinite(l->uy[k]) &&
                  std::isfinite(l->temp[k]);
        }
    out[4] = mu;
    double rb = 0;
    for (double v : c.rho) rb += v;
    rb /= double(c.rho.size());
    out[5] = rb;
    double md = 0, mi = 0;
    for (const auto* l : lv)
        for (double v : l->rho) md = std::fmax(md, std::fabs(v - rb));
    for (const auto& b : o->blocks) {
        for (const auto& gh : b.grid.ghosts) mi = std::fmax(mi, std::fabs(b.fine.rho[gh.k] - rb));
        for (const auto& ce : b.grid.coin) mi = std::fmax(mi, std::fabs(c.rho[ce.kc] - rb));
        if (b.has_sub) {
            for (const auto& gh : b.sub.grid.ghosts) mi = std::fmax(mi, std::fabs(b.sub.lvl.rho[gh.k] - rb));
            for (const auto& ce : b.sub.grid.coin) mi = std::fmax(mi, std::fabs(b.fine.rho[ce.kc] - rb));
        }
    }
    out[6] = md;
    out[7] = mi;
    out[8] = fin ? 1.0 : 0.0;
}

}  // extern "C"
