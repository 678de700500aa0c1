// cavity_oracle.hpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// CPU FP64 restatement of the reference lattice-Boltzmann step for the 2D
// differentially heated cavity (bbrangeo/cfd_cavity, Rust crate `cavity_les`).
// It exists to check the CUDA product path; it is never linked into, loaded by
// or called from the product library.  Only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline / reference arm use it.
//
// Parity status.  The reference cannot be compiled in this environment (no
// cargo/rustc, and its arithmetic crate `oxiphysics-lbm 0.1.2` is not
// vendored).  This restatement is pinned by the reference's own known-answer
// tests (src/uniform/tests.rs), ported one by one into tests/, and by the
// reference's published Nusselt numbers (README.md:44-46).  Three pieces of
// crate arithmetic are NOT pinned by any reference test and are stated here
// as assumptions (each behind a switch where it matters):
//   * geq's velocity dependence (only sum_i geq = T is tested,
//     src/uniform/tests.rs:123-127): default quadratic, same form as feq with
//     rho -> T; `geq_order = 1` selects the linear form.
//   * the D2Q9 direction order (only "opp maps 1..4 onto 5..8" follows from
//     swap_opposite, src/uniform/solver.rs:938-946): c_{i+4} = -c_i.
//   * compute_turbulent_viscosity = (Cs*dx)^2*|S| and y_plus = y*u_tau/nu
//     (documented at src/uniform/solver.rs:1115-1117 and post.rs:189 only).
//
// Everything is templated on the scalar type so that the same code runs in
// plain double and in forward-mode dual numbers (tangent-linear oracle).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <type_traits>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// D2Q9 lattice (crate `oxiphysics_lbm::lattice`, used at
// src/uniform/solver.rs:10).  Order: rest, E, N, NE, NW, then the opposites
// W, S, SW, SE so that OPP[i] = i+4 for i in 1..4.
// ---------------------------------------------------------------------------
constexpr int Q = 9;
constexpr int CX[Q] = {0, 1, 0, 1, -1, -1, 0, -1, 1};
constexpr int CY[Q] = {0, 0, 1, 1, 1, 0, -1, -1, -1};
constexpr int OPP[Q] = {0, 5, 6, 7, 8, 1, 2, 3, 4};
constexpr double W[Q] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 36.0, 1.0 / 36.0,
                         1.0 / 9.0, 1.0 / 9.0, 1.0 / 36.0, 1.0 / 36.0};
constexpr double CS2 = 1.0 / 3.0;

// Wall temperatures, src/uniform/solver.rs:16-21.
constexpr double T_HOT = 0.5;
constexpr double T_COLD = -0.5;
constexpr double DELTA_T = T_HOT - T_COLD;
// TRT magic parameter, src/uniform/solver.rs:427.
constexpr double LAMBDA_TRT = 3.0 / 16.0;

// --- scalar helpers that also work for the dual type ----------------------
inline double val(double x) { return x; }
inline double dsqrt(double x) { return std::sqrt(x); }
inline double dpow(double a, double b) { return std::pow(a, b); }
inline double dabs(double x) { return std::fabs(x); }

// Equilibrium of the f populations.  The crate function is not vendored; its
// form is pinned by the restatement in the reference's Poiseuille test
// (src/uniform/tests.rs:308-316), reproduced here operation for operation.
template <class R>
inline R feq(int i, R rho, R ux, R uy) {
    R eu = double(CX[i]) * ux + double(CY[i]) * uy;
    R u2 = ux * ux + uy * uy;
    return W[i] * rho * (1.0 + eu / CS2 + eu * eu / (2.0 * CS2 * CS2) - u2 / (2.0 * CS2));
}

// Equilibrium of the g (temperature) populations.  Only sum_i geq = T is
// pinned (src/uniform/tests.rs:123-127); order 2 (default) uses the feq form
// with rho -> T, order 1 the linear advection-diffusion form.
template <class R>
inline R geq(int i, R t, R ux, R uy, int order) {
    R eu = double(CX[i]) * ux + double(CY[i]) * uy;
    if (order == 1) return W[i] * t * (1.0 + eu / CS2);
    R u2 = ux * ux + uy * uy;
    return W[i] * t * (1.0 + eu / CS2 + eu * eu / (2.0 * CS2 * CS2) - u2 / (2.0 * CS2));
}

// Boussinesq force, call site src/uniform/solver.rs:1084
// (boussinesq_force(rho, beta_eff, 1.0, temp, t_ref), gravity +1).
template <class R>
inline R boussinesq_force(R rho, double beta, R temp, double t_ref) {
    return rho * beta * 1.0 * (temp - t_ref);
}

// Dynamic model bounds (src/uniform/solver.rs:25, 31).
constexpr double C_DYN_MAX = 0.04;
constexpr double TAU_TRT_FLOOR = 0.505;

// lilly_coefficient, src/uniform/solver.rs:1250-1261: C = num / (2 den),
// 0 for a non-finite or non-positive denominator, clamped to [0, 0.04].
inline double lilly_coefficient(double num, double den) {
    if (!std::isfinite(den) || !std::isfinite(num) || den <= 0.0) return 0.0;
    const double c = 0.5 * num / den;
    if (!std::isfinite(c)) return 0.0;
    return c < 0.0 ? 0.0 : (c > C_DYN_MAX ? C_DYN_MAX : c);
}

// Rust's f64::max (returns the non-NaN operand).
inline double fmax_rs(double a, double b) { return std::fmax(a, b); }

// ---------------------------------------------------------------------------
// Construction parameters: the arguments of CavitySolver::new
// (src/uniform/solver.rs:108) plus the initial-field mode needed by the
// benchmark configurations and an optional hot-wall profile.
// ---------------------------------------------------------------------------
enum InitMode { INIT_LINEAR = 0, INIT_ZERO = 1 };

// ---------------------------------------------------------------------------
// Dynamic mixed-scale SGS model on one grid: compute_dynamic_sgs
// (src/uniform/solver.rs:562-828) and its per-level twin
// compute_dynamic_sgs_level (src/octree/smag.rs:144-416), which differ only
// in where tau comes from (tau_s of the collision, or 0.5 + 3 nu of the
// level).  Everything in lattice units of the grid (dx = 1), sequential sums.
// ---------------------------------------------------------------------------
struct DynSgs {
    std::vector<double> nu_t, alpha_t;
    double cnu_mean = 0.0, cnu_max = 0.0, ck_mean = 0.0, ck_max = 0.0;
};

// box_filter (src/uniform/solver.rs:1204-1227, src/octree/smag.rs:54-77):
// window of `width` nodes starting half_left = (width - 1) / 2 before the
// node, clamped at the walls.
inline std::vector<double> box_filter(const std::vector<double>& fld, int nx, int ny, int width) {
    std::vector<double> out(size_t(nx) * ny, 0.0);
    const int hl = (width - 1) / 2;
    for (int iy = 0; iy < ny; ++iy) {
        const int y0 = std::max(iy - hl, 0), y1 = std::min(iy + width - hl, ny);
        for (int ix = 0; ix < nx; ++ix) {
            const int x0 = std::max(ix - hl, 0), x1 = std::min(ix + width - hl, nx);
            double sum = 0.0;
            for (int yy = y0; yy < y1; ++yy)
                for (int xx = x0; xx < x1; ++xx) sum += fld[size_t(yy) * nx + xx];
            out[size_t(iy) * nx + ix] = sum / double((y1 - y0) * (x1 - x0));
        }
    }
    return out;
}
// ddx / ddy (src/uniform/solver.rs:1229-1245, src/octree/smag.rs:80-95):
// central differences, one-sided by clamping at the walls.
inline double ddx(const std::vector<double>& fld, int nx, int ix, int iy) {
    const int xm = ix == 0 ? 0 : ix - 1, xp = ix + 1 >= nx ? nx - 1 : ix + 1;
    return 0.5 * (fld[size_t(iy) * nx + xp] - fld[size_t(iy) * nx + xm]);
}
inline double ddy(const std::vector<double>& fld, int nx, int ny, int ix, int iy) {
    const int ym = iy == 0 ? 0 : iy - 1, yp = iy + 1 >= ny ? ny - 1 : iy + 1;
    return 0.5 * (fld[size_t(yp) * nx + ix] - fld[size_t(ym) * nx + ix]);
}

inline DynSgs dynamic_sgs_grid(int nx, int ny, const std::vector<std::array<double, Q>>& f,
                               const std::vector<double>& rho, const std::vector<double>& ux,
                               const std::vector<double>& uy, const std::vector<double>& T, double tau_s,
                               double alpha_exp, double eta_test, double nu_mol, double alpha_mol,
                               double nu_sm_min) {
    const int n = nx * ny;
    const double eta = std::max(eta_test, 1.0);
    const int width = std::max((int)std::llround(eta), 1);
    const double dx = 1.0, dtest = eta * dx, delta_t = DELTA_T;
    auto ubx = box_filter(ux, nx, ny, width), uby = box_filter(uy, nx, ny, width);
    auto tb = box_filter(T, nx, ny, width);
    std::vector<double> pxx(n), pxy(n), pyy(n), ptx(n), pty(n);
    for (int k = 0; k < n; ++k) {
        pxx[k] = ux[k] * ux[k];
        pxy[k] = ux[k] * uy[k];
        pyy[k] = uy[k] * uy[k];
        ptx[k] = ux[k] * T[k];
        pty[k] = uy[k] * T[k];
    }
    auto lbuxx = box_filter(pxx, nx, ny, width), lbuxy = box_filter(pxy, nx, ny, width);
    auto lbuyy = box_filter(pyy, nx, ny, width), lbutx = box_filter(ptx, nx, ny, width);
    auto lbuty = box_filter(pty, nx, ny, width);
    std::vector<double> shxx(n), shxy(n), shyy(n), smag_hat(n), sbxx(n), sbxy(n), sbyy(n), smag_bar(n),
        gtx(n), gty(n), gbx(n), gby(n), qsm_h(n), phi_h(n), tmag_hat(n), tmag_bar(n);
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
            const int k = iy * nx + ix;
            const double rho_k = rho[k], ux_k = ux[k], uy_k = uy[k], t_k = T[k];
            double pi_xx = 0.0, pi_xy = 0.0, pi_yy = 0.0;
            for (int i = 0; i < Q; ++i) {
                const double cx = CX[i], cy = CY[i];
                const double fneq = f[k][i] - feq<double>(i, rho_k, ux_k, uy_k);
                pi_xx += fneq * cx * cx;
                pi_xy += fneq * cx * cy;
                pi_yy += fneq * cy * cy;
            }
            const double rho_m = rho_k > 1e-12 ? rho_k : 1e-12;
            const double denom = 2.0 * CS2 * tau_s * rho_m;
            const double pi2 = pi_xx * pi_xx + 2.0 * pi_xy * pi_xy + pi_yy * pi_yy;
            shxx[k] = -pi_xx / denom;
            shxy[k] = -pi_xy / denom;
            shyy[k] = -pi_yy / denom;
            smag_hat[k] = std::sqrt(pi2) / denom;
            const double sxx = ddx(ubx, nx, ix, iy);
            const double syy = ddy(uby, nx, ny, ix, iy);
            const double sxy = 0.5 * (ddx(uby, nx, ix, iy) + ddy(ubx, nx, ny, ix, iy));
            sbxx[k] = sxx;
            sbxy[k] = sxy;
            sbyy[k] = syy;
            smag_bar[k] = std::sqrt(sxx * sxx + 2.0 * sxy * sxy + syy * syy);
            gtx[k] = ddx(T, nx, ix, iy);
            gty[k] = ddy(T, nx, ny, ix, iy);
            gbx[k] = ddx(tb, nx, ix, iy);
            gby[k] = ddy(tb, nx, ny, ix, iy);
            const double dux = ux_k - ubx[k], duy = uy_k - uby[k];
            const double du2 = dux * dux + duy * duy;
            qsm_h[k] = std::sqrt(0.5 * du2) / 2.0;
            const double dt_local = t_k - tb[k];
            phi_h[k] = 0.5 * std::fabs(dt_local) * std::sqrt(0.5 * du2);
            const double th_x = gtx[k] * shxx[k] + gty[k] * shxy[k];
            const double th_y = gtx[k] * shxy[k] + gty[k] * shyy[k];
            tmag_hat[k] = std::sqrt(2.0 * (th_x * th_x + th_y * th_y));
            const double tb_x = gbx[k] * sbxx[k] + gby[k] * sbxy[k];
            const double tb_y = gbx[k] * sbxy[k] + gby[k] * sbyy[k];
            tmag_bar[k] = std::sqrt(2.0 * (tb_x * tb_x + tb_y * tb_y));
        }
    auto qbar_h = box_filter(qsm_h, nx, ny, width), phibar_h = box_filter(phi_h, nx, ny, width);
    std::vector<double> num_v(n), den_v(n), num_k(n), den_k(n), nu_mix_grid(n), kap_mix_grid(n);
    for (int k = 0; k < n; ++k) {
        const double nu_mix_t =
            std::pow(dtest * dtest * smag_bar[k], alpha_exp) * std::pow(dtest * qbar_h[k], 1.0 - alpha_exp);
        const double nu_mix_g =
            std::pow(dx * dx * smag_hat[k], alpha_exp) * std::pow(dx * qsm_h[k], 1.0 - alpha_exp);
        const double kap_mix_t = std::pow(dtest * dtest * dtest / delta_t * tmag_bar[k], alpha_exp) *
                                 std::pow(dtest / delta_t * phibar_h[k], 1.0 - alpha_exp);
        const double kap_mix_g = std::pow(dx * dx * dx / delta_t * tmag_hat[k], alpha_exp) *
                                 std::pow(dx / delta_t * phi_h[k], 1.0 - alpha_exp);
        nu_mix_grid[k] = nu_mix_g;
        kap_mix_grid[k] = kap_mix_g;
        const double mxx = nu_mix_t * sbxx[k] - nu_mix_g * shxx[k];
        const double mxy = nu_mix_t * sbxy[k] - nu_mix_g * shxy[k];
        const double myy = nu_mix_t * sbyy[k] - nu_mix_g * shyy[k];
        const double mx = kap_mix_t * gbx[k] - kap_mix_g * gtx[k];
        const double my = kap_mix_t * gby[k] - kap_mix_g * gty[k];
        const double lxx = lbuxx[k] - ubx[k] * ubx[k];
        const double lxy = lbuxy[k] - ubx[k] * uby[k];
        const double lyy = lbuyy[k] - uby[k] * uby[k];
        const double lkk3 = (lxx + lyy) / 3.0;
        const double ldxx = lxx - lkk3, ldyy = lyy - lkk3;
        const double ljx = lbutx[k] - ubx[k] * tb[k];
        const double ljy = lbuty[k] - uby[k] * tb[k];
        num_v[k] = ldxx * mxx + 2.0 * lxy * mxy + ldyy * myy;
        den_v[k] = mxx * mxx + 2.0 * mxy * mxy + myy * myy;
        num_k[k] = ljx * mx + ljy * my;
        den_k[k] = mx * mx + my * my;
    }
    auto num_v_b = box_filter(num_v, nx, ny, width), den_v_b = box_filter(den_v, nx, ny, width);
    auto num_k_b = box_filter(num_k, nx, ny, width), den_k_b = box_filter(den_k, nx, ny, width);
    DynSgs d;
    d.nu_t.assign(n, 0.0);
    d.alpha_t.assign(n, 0.0);
    double cnu_sum = 0.0, cnu_max = 0.0, ck_sum = 0.0, ck_max = 0.0;
    const double margin = (TAU_TRT_FLOOR - 0.5) / 3.0;
    for (int k = 0; k < n; ++k) {
        const double cnu = lilly_coefficient(num_v_b[k], den_v_b[k]);
        const double ck = lilly_coefficient(num_k_b[k], den_k_b[k]);
        cnu_sum += cnu;
        if (cnu > cnu_max) cnu_max = cnu;
        ck_sum += ck;
        if (ck > ck_max) ck_max = ck;
        const double nt = cnu * nu_mix_grid[k];
        const double nu_t_min = fmax_rs(nu_sm_min * nu_mol, margin - nu_mol);
        d.nu_t[k] = nt < nu_t_min ? nu_t_min : nt;
        const double at = ck * kap_mix_grid[k];
        const double alpha_t_min = fmax_rs(nu_sm_min * alpha_mol, margin - alpha_mol);
        d.alpha_t[k] = at < alpha_t_min ? alpha_t_min : at;
    }
    d.cnu_mean = cnu_sum / double(n);
    d.cnu_max = cnu_max;
    d.ck_mean = ck_sum / double(n);
    d.ck_max = ck_max;
    return d;
}

struct Params {
    int nx = 64, ny = 256;
    double ra = 1e6, pr = 0.71, cs = 0.10, pr_t = 0.9, utarget = 0.02;
    uint64_t seed = 42;
    int jobs = 1;
    double alpha_mult = 1.0, nu_start_mult = 1.0;
    int has_nu_override = 0;
    double nu_override = 0.0;
    int init_mode = INIT_LINEAR;  // reference: linear theta + noise
    double noise_amp = 1.0e-3;    // reference: +-1e-3
    int geq_order = 2;
    const double* t_hot_profile = nullptr;  // [ny], replaces T_HOT at x = 0
    double t_cold = T_COLD;
};

// xorshift64*, src/uniform/rng.rs:5-31.
struct Rng {
    uint64_t state;
    explicit Rng(uint64_t seed) : state(seed | 1ull) {}
    uint64_t next_u64() {
        uint64_t x = state;
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        state = x;
        return x * 0x2545F4914F6CDD1Dull;
    }
    double next_f64() { return double(next_u64() >> 11) / double(1ull << 53); }
};

// Per-step scalars shared by every node (CollideCtx, src/uniform/solver.rs:1034-1043).
struct CollideCtx {
    double tau, beta_eff, t_ref, pr_t, nu, alpha, lambda_trt;
};

// Small persistent thread pool: row bands, one band per thread, like the
// reference's rayon row-band loops (src/uniform/solver.rs:462-511, 844-886).
class RowPool {
public:
    explicit RowPool(int jobs);
    ~RowPool();
    // Runs fn(y0, y1) on [0, ny) split into `jobs` contiguous bands.
    void run(int ny, const std::function<void(int, int)>& fn);
    int jobs() const { return jobs_; }

private:
    struct Impl;
    Impl* impl_;
    int jobs_;
};

// ---------------------------------------------------------------------------
// The solver: CavitySolver, src/uniform/solver.rs:35-104 (fixed-Cs path).
// ---------------------------------------------------------------------------
template <class R>
struct Solver {
    using Pop = std::array<R, Q>;
    int nx = 0, ny = 0;
    std::vector<Pop> f, g;  // AoS [k][9], k = iy*nx + ix (solver.rs:224-226)
    std::vector<R> rho, ux, uy, temperature, nu_t, fy_node;
    std::vector<R> t_hot;   // hot-wall temperature per row (T_HOT by default)
    R cs = 0.0;             // Smagorinsky constant (differentiable)
    double t_cold = T_COLD;
    double lz = 0, lx = 0, beta_eff = 0, nu = 0, alpha = 0, alpha_phys = 0, pr_t = 0;
    double tau = 0, tau_t = 0, t_ref = 0.0;
    double nu_start_mult = 1.0;
    long time_step = 0;
    long spin_up_steps = 0;
    int geq_order = 2;
    int error = 0;  // 0 ok, 1 arg, 2 tau
    RowPool* pool = nullptr;
    // dynamic mixed-scale SGS model (set_dynamic_sgs, src/uniform/solver.rs:215-220)
    bool dynamic_smag = false;
    double smag_alpha = 0.5, nu_sm_min = -0.1, eta_test = 2.0;
    std::vector<double> nu_t_pre, alpha_t_pre;  // empty when the model is off
    double cs_dyn_mean = 0.0, cs_dyn_max = 0.0, kappa_dyn_mean = 0.0, kappa_dyn_max = 0.0;

    int idx(int ix, int iy) const { return iy * nx + ix; }

    // CavitySolver::new, src/uniform/solver.rs:108-210.
    void init(const Params& p) {
        nx = p.nx;
        ny = p.ny;
        error = 0;
        if (nx < 4 || ny < 4) { error = 1; return; }
        lz = double(ny - 1);
        lx = double(nx - 1);
        const double c_scale = 1.7;
        double nu_cal = std::pow(p.utarget * std::sqrt(p.pr) * lz / (c_scale * std::sqrt(p.ra)), 2.0 / 3.0);
        if (p.has_nu_override) {
            double n = p.nu_override;
            if (!(n > 0.0 && std::isfinite(n))) { error = 1; return; }
            if (!(0.5 + 3.0 * n > 0.5005)) { error = 2; return; }
            nu = n;
        } else {
            nu = fmax_rs(nu_cal, 0.002);
        }
        alpha_phys = nu / p.pr;
        alpha = alpha_phys * p.alpha_mult;
        beta_eff = p.ra * nu * alpha_phys / (lz * lz * lz);
        tau = 0.5 + 3.0 * nu;
        tau_t = 0.5 + 3.0 * alpha;
        if (!p.has_nu_override && !(tau > 0.505)) { error = 2; return; }
        if (!(tau_t > 0.505)) { error = 2; return; }
        cs = p.cs;
        pr_t = p.pr_t;
        geq_order = p.geq_order;
        t_cold = p.t_cold;
        t_hot.assign(ny, R(T_HOT));
        if (p.t_hot_profile)
            for (int iy = 0; iy < ny; ++iy) t_hot[iy] = p.t_hot_profile[iy];
        const int n = nx * ny;
        f.assign(n, Pop{});
        g.assign(n, Pop{});
        rho.assign(n, R(0.0));
        ux.assign(n, R(0.0));
        uy.assign(n, R(0.0));
        temperature.assign(n, R(0.0));
        nu_t.assign(n, R(0.0));
        fy_node.assign(n, R(0.0));
        Rng rng(p.seed);
        // Initial fields, src/uniform/solver.rs:159-176.  INIT_ZERO replaces
        // the linear profile by theta = 0 (benchmark configurations).
        for (int iy = 0; iy < ny; ++iy) {
            for (int ix = 0; ix < nx; ++ix) {
                int k = iy * nx + ix;
                double xf = double(ix) / double(nx - 1);
                double t_lin = T_HOT + (T_COLD - T_HOT) * xf;
                double pert = p.noise_amp * (2.0 * rng.next_f64() - 1.0);
                double t = (p.init_mode == INIT_LINEAR) ? t_lin + pert : pert;
                temperature[k] = t;
                rho[k] = 1.0;
                ux[k] = 0.0;
                uy[k] = 0.0;
                for (int i = 0; i < Q; ++i) {
                    f[k][i] = feq<R>(i, R(1.0), R(0.0), R(0.0));
                    g[k][i] = geq<R>(i, R(t), R(0.0), R(0.0), geq_order);
                }
            }
        }
        time_step = 0;
        spin_up_steps = std::min<long>(std::max<long>(ny / 10, 200), 2000);
        nu_start_mult = std::max(p.nu_start_mult, 1.0);
    }

    // init_from_fields, src/uniform/solver.rs:232-262.
    void init_from_fields(const double* r, const double* u, const double* v, const double* t) {
        for (int k = 0; k < nx * ny; ++k) {
            rho[k] = r[k];
            ux[k] = u[k];
            uy[k] = v[k];
            temperature[k] = t[k];
            for (int i = 0; i < Q; ++i) {
                f[k][i] = feq<R>(i, rho[k], ux[k], uy[k]);
                g[k][i] = geq<R>(i, temperature[k], ux[k], uy[k], geq_order);
            }
        }
        enforce_wall_velocity();
        time_step = 0;
    }

    // ramp_nu_alpha, src/uniform/solver.rs:390-410.
    void ramp_nu_alpha(long step, double& nu_eff, double& alpha_eff) const {
        if (step < spin_up_steps) {
            double x = double(step) / double(spin_up_steps);
            double nu_start = nu * nu_start_mult;
            nu_eff = nu_start * std::pow(nu / nu_start, x);
            double alpha_start = alpha * nu_start_mult;
            alpha_eff = alpha_start * std::pow(alpha / alpha_start, x);
        } else {
            nu_eff = nu;
            alpha_eff = alpha;
        }
    }

    // Per-step scalars of collide, src/uniform/solver.rs:421-454.
    CollideCtx collide_ctx(long step) const {
        double beta = (step < spin_up_steps) ? beta_eff * (double(step) / double(spin_up_steps)) : beta_eff;
        double nu_eff, alpha_eff;
        ramp_nu_alpha(step, nu_eff, alpha_eff);
        CollideCtx c;
        c.tau = 0.5 + 3.0 * fmax_rs(nu_eff, 0.002 / 3.0);
        c.beta_eff = beta;
        c.t_ref = t_ref;
        c.pr_t = pr_t;
        c.nu = nu_eff;
        c.alpha = alpha_eff;
        c.lambda_trt = LAMBDA_TRT;
        return c;
    }

    // collide_node, src/uniform/solver.rs:1054-1185 (fixed-Cs branch).
    void collide_node(Pop& fn, Pop& gn, R& nu_t_out, R& fy_out, R r, R u, R v, R temp,
                      const CollideCtx& c, const double* nu_t_pre_k = nullptr,
                      const double* alpha_t_pre_k = nullptr) const {
        R fyv = boussinesq_force<R>(r, c.beta_eff, temp, c.t_ref);
        fy_out = fyv;
        Pop f_eq, g_eq;
        for (int i = 0; i < Q; ++i) {
            f_eq[i] = feq<R>(i, r, u, v);
            g_eq[i] = geq<R>(i, temp, u, v, geq_order);
        }
        R pi_xx = 0.0, pi_xy = 0.0, pi_yy = 0.0;
        for (int i = 0; i < Q; ++i) {
            double cx = CX[i], cy = CY[i];
            R fneq = fn[i] - f_eq[i];
            pi_xx = pi_xx + fneq * cx * cx;
            pi_xy = pi_xy + fneq * cx * cy;
            pi_yy = pi_yy + fneq * cy * cy;
        }
        R pi2 = pi_xx * pi_xx + 2.0 * pi_xy * pi_xy + pi_yy * pi_yy;
        R rho_m = (val(r) > 1e-12) ? r : R(1e-12);
        R s_mag = dsqrt(pi2) / (2.0 * CS2 * c.tau * rho_m);
        // compute_turbulent_viscosity(s_mag, cs) = (Cs*dx)^2*|S|, dx = 1.
        // dynamic mode: nu_t and alpha_t precomputed per node (solver.rs:1118-1139)
        R nut = nu_t_pre_k ? R(*nu_t_pre_k) : cs * cs * s_mag;
        nu_t_out = nut;
        R tau_plus = 0.5 + 3.0 * (c.nu + nut);
        R tau_minus = 0.5 + c.lambda_trt / (tau_plus - 0.5);
        R alpha_t = alpha_t_pre_k ? R(*alpha_t_pre_k) : nut / c.pr_t;
        R tau_t_plus = 0.5 + 3.0 * (c.alpha + alpha_t);
        R tau_t_minus = tau_t_plus;
        R a_f = 0.5 * (1.0 / tau_plus + 1.0 / tau_minus);
        R b_f = 0.5 * (1.0 / tau_plus - 1.0 / tau_minus);
        R a_g = 0.5 * (1.0 / tau_t_plus + 1.0 / tau_t_minus);
        R b_g = 0.5 * (1.0 / tau_t_plus - 1.0 / tau_t_minus);
        Pop d_f, d_g;
        for (int i = 0; i < Q; ++i) {
            d_f[i] = fn[i] - f_eq[i];
            d_g[i] = gn[i] - g_eq[i];
        }
        for (int i = 0; i < Q; ++i) {
            double cx = CX[i], cy = CY[i];
            int o = OPP[i];
            R ei_u = cx * u + cy * v;
            R s_i = W[i] * ((cy - v) / CS2 + ei_u * cy / (CS2 * CS2)) * fyv;
            R s_minus = W[i] * (cy / CS2) * fyv;
            R s_plus = s_i - s_minus;
            fn[i] = fn[i] + (-a_f * d_f[i] - b_f * d_f[o] + (1.0 - 0.5 / tau_minus) * s_minus +
                             (1.0 - 0.5 / tau_plus) * s_plus);
        }
        for (int i = 0; i < Q; ++i) {
            int o = OPP[i];
            gn[i] = gn[i] + (-a_g * d_g[i] - b_g * d_g[o]);
        }
    }

    template <class Fn>
    void rows(Fn&& fn) {
        if (pool && pool->jobs() > 1) pool->run(ny, [&](int y0, int y1) { fn(y0, y1); });
        else fn(0, ny);
    }

    // collide, src/uniform/solver.rs:421-540.
    void collide(long step) {
        CollideCtx c = collide_ctx(step);
        rows([&](int y0, int y1) {
            for (int iy = y0; iy < y1; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    int k = iy * nx + ix;
                    const bool dyn = !nu_t_pre.empty();
                    collide_node(f[k], g[k], nu_t[k], fy_node[k], rho[k], ux[k], uy[k], temperature[k], c,
                                 dyn ? &nu_t_pre[k] : nullptr, dyn ? &alpha_t_pre[k] : nullptr);
                }
        });
    }

    // stream, src/uniform/solver.rs:838-913 (pull, bounce-back for f, g kept
    // at out-of-domain sources until the thermal boundary conditions).
    std::vector<Pop> f_old, g_old;
    void stream() {
        f_old = f;
        g_old = g;
        rows([&](int y0, int y1) {
            for (int iy = y0; iy < y1; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    int k = iy * nx + ix;
                    for (int i = 0; i < Q; ++i) {
                        int sx = ix - CX[i], sy = iy - CY[i];
                        if (sx >= 0 && sx < nx && sy >= 0 && sy < ny) {
                            int src = sy * nx + sx;
                            f[k][i] = f_old[src][i];
                            g[k][i] = g_old[src][i];
                        } else {
                            f[k][i] = f_old[k][OPP[i]];
                            g[k][i] = g_old[k][i];
                        }
                    }
                }
        });
    }

    // apply_bounce_back / swap_opposite, src/uniform/solver.rs:920-946.
    void swap_opposite(int k) {
        for (int i = 1; i < 5; ++i) std::swap(f[k][i], f[k][OPP[i]]);
    }
    void apply_bounce_back() {
        for (int iy = 0; iy < ny; ++iy) {
            swap_opposite(iy * nx + 0);
            swap_opposite(iy * nx + nx - 1);
        }
        for (int ix = 0; ix < nx; ++ix) {
            swap_opposite(ix);
            swap_opposite((ny - 1) * nx + ix);
        }
    }

    // apply_thermal_boundary_conditions, src/uniform/solver.rs:951-988.
    void apply_thermal_boundary_conditions() {
        for (int iy = 0; iy < ny; ++iy) {
            int k = iy * nx;
            for (int i = 0; i < Q; ++i) g[k][i] = geq<R>(i, t_hot[iy], R(0.0), R(0.0), geq_order);
            k = iy * nx + (nx - 1);
            for (int i = 0; i < Q; ++i) g[k][i] = geq<R>(i, R(t_cold), R(0.0), R(0.0), geq_order);
        }
        for (int ix = 0; ix < nx; ++ix) {
            g[ix] = g[nx + ix];
            g[(ny - 1) * nx + ix] = g[(ny - 2) * nx + ix];
        }
    }

    // update_macroscopic, src/uniform/solver.rs:298-367 (Guo half-force
    // correction on u_y with the fy stored by the last collision).
    void update_macroscopic() {
        rows([&](int y0, int y1) {
            for (int iy = y0; iy < y1; ++iy)
                for (int ix = 0; ix < nx; ++ix) {
                    int k = iy * nx + ix;
                    R r = 0.0, un = 0.0, vn = 0.0, tn = 0.0;
                    for (int j = 0; j < Q; ++j) {
                        r = r + f[k][j];
                        un = un + double(CX[j]) * f[k][j];
                        vn = vn + double(CY[j]) * f[k][j];
                        tn = tn + g[k][j];
                    }
                    if (val(r) > std::numeric_limits<double>::epsilon()) {
                        un = un / r;
                        vn = vn / r;
                        vn = vn + 0.5 * fy_node[k] / r;
                    }
                    rho[k] = r;
                    ux[k] = un;
                    uy[k] = vn;
                    temperature[k] = tn;
                }
        });
    }

    // enforce_wall_velocity, src/uniform/solver.rs:992-1009.
    void enforce_wall_velocity() {
        for (int iy = 0; iy < ny; ++iy)
            for (int ix : {0, nx - 1}) {
                ux[iy * nx + ix] = 0.0;
                uy[iy * nx + ix] = 0.0;
            }
        for (int iy : {0, ny - 1})
            for (int ix = 0; ix < nx; ++ix) {
                ux[iy * nx + ix] = 0.0;
                uy[iy * nx + ix] = 0.0;
            }
    }

    // ---- dynamic mixed-scale SGS model, src/uniform/solver.rs:562-828 ------
    void compute_dynamic_sgs() {
        if constexpr (std::is_same<R, double>::value) {
            double nu_eff, alpha_eff;
            ramp_nu_alpha(time_step, nu_eff, alpha_eff);
            const double tau_s = 0.5 + 3.0 * fmax_rs(nu_eff, 0.002 / 3.0);
            const DynSgs d = dynamic_sgs_grid(nx, ny, f, rho, ux, uy, temperature, tau_s, smag_alpha, eta_test, nu,
                                              alpha, nu_sm_min);
            nu_t_pre = d.nu_t;
            alpha_t_pre = d.alpha_t;
            cs_dyn_mean = d.cnu_mean;
            cs_dyn_max = d.cnu_max;
            kappa_dyn_mean = d.ck_mean;
            kappa_dyn_max = d.ck_max;
        }
    }

    // step, src/uniform/solver.rs:279-293.
    void step() {
        if (dynamic_smag) compute_dynamic_sgs();
        collide(time_step);
        stream();
        apply_thermal_boundary_conditions();
        update_macroscopic();
        enforce_wall_velocity();
        time_step += 1;
    }

    // ---- diagnostics, src/uniform/post.rs -------------------------------
    // nusselt_hot, post.rs:68-78 (second link, height scale).
    R nusselt_hot() const {
        R sum = 0.0;
        for (int iy = 0; iy < ny; ++iy) sum = sum + dabs_r(temperature[idx(1, iy)] - temperature[idx(2, iy)]);
        return sum / double(ny) * lz / DELTA_T;
    }
    // nusselt_cold, post.rs:100-111.
    R nusselt_cold() const {
        R sum = 0.0;
        for (int iy = 0; iy < ny; ++iy)
            sum = sum + dabs_r(temperature[idx(nx - 2, iy)] - temperature[idx(nx - 3, iy)]);
        return sum / double(ny) * lz / DELTA_T;
    }
    // nusselt_hot_wall_link, post.rs:87-97 (first link).
    R nusselt_hot_wall_link() const {
        R sum = 0.0;
        for (int iy = 0; iy < ny; ++iy) sum = sum + dabs_r(temperature[idx(0, iy)] - temperature[idx(1, iy)]);
        return sum / double(ny) * lz / DELTA_T;
    }
    static R dabs_r(R x) { return val(x) < 0.0 ? R(-x) : x; }
};

}  // namespace orc
