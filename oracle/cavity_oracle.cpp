// cavity_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// C ABI over the templated FP64 restatement in cavity_oracle.hpp, plus the
// row-band thread pool that stands in for the reference's rayon loops when
// the oracle is timed as the CPU baseline.  Compiled with -ffp-contract=off
// so that, like Rust, no multiply-add is fused.
#include "cavity_oracle.h"

#include <atomic>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>

#include "cavity_oracle.hpp"

namespace orc {

struct RowPool::Impl {
    std::vector<std::thread> threads;
    std::mutex m;
    std::condition_variable cv_start, cv_done;
    const std::function<void(int, int)>* fn = nullptr;
    int ny = 0;
    long generation = 0;
    int pending = 0;
    bool stop = false;
};

static void band(int ny, int jobs, int t, int& y0, int& y1) {
    // Contiguous bands of rows, as rayon's par_chunks_mut(nx) over rows.
    y0 = int((long)ny * t / jobs);
    y1 = int((long)ny * (t + 1) / jobs);
}

RowPool::RowPool(int jobs) : impl_(new Impl), jobs_(jobs < 1 ? 1 : jobs) {
    for (int t = 1; t < jobs_; ++t) {
        impl_->threads.emplace_back([this, t]() {
            long seen = 0;
            for (;;) {
                const std::function<void(int, int)>* fn;
                int ny;
                {
                    std::unique_lock<std::mutex> lk(impl_->m);
                    impl_->cv_start.wait(lk, [&] { return impl_->stop || impl_->generation != seen; });
                    if (impl_->stop) return;
                    seen = impl_->generation;
                    fn = impl_->fn;
                    ny = impl_->ny;
                }
                int y0, y1;
                band(ny, jobs_, t, y0, y1);
                if (y1 > y0) (*fn)(y0, y1);
                {
                    std::lock_guard<std::mutex> lk(impl_->m);
                    if (--impl_->pending == 0) impl_->cv_done.notify_one();
                }
            }
        });
    }
}

RowPool::~RowPool() {
    {
        std::lock_guard<std::mutex> lk(impl_->m);
        impl_->stop = true;
    }
    impl_->cv_start.notify_all();
    for (auto& th : impl_->threads) th.join();
    delete impl_;
}

void RowPool::run(int ny, const std::function<void(int, int)>& fn) {
    {
        std::lock_guard<std::mutex> lk(impl_->m);
        impl_->fn = &fn;
        impl_->ny = ny;
        impl_->pending = jobs_ - 1;
        impl_->generation++;
    }
    impl_->cv_start.notify_all();
    int y0, y1;
    band(ny, jobs_, 0, y0, y1);
    if (y1 > y0) fn(y0, y1);
    std::unique_lock<std::mutex> lk(impl_->m);
    impl_->cv_done.wait(lk, [&] { return impl_->pending == 0; });
}

}  // namespace orc

using S = orc::Solver<double>;

struct OrcHandle {
    S s;
    orc::RowPool* pool = nullptr;
    ~OrcHandle() { delete pool; }
};

static OrcHandle* H(void* h) { return static_cast<OrcHandle*>(h); }

extern "C" {

void* orc_create(const orc_params* cp, int32_t* err) {
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
    OrcHandle* h = new OrcHandle;
    h->s.init(p);
    if (h->s.error) {
        if (err) *err = h->s.error;
        delete h;
        return nullptr;
    }
    if (p.jobs > 1) {
        h->pool = new orc::RowPool(p.jobs);
        h->s.pool = h->pool;
    }
    if (err) *err = 0;
    return h;
}

void orc_destroy(void* h) { delete H(h); }
void orc_step(void* h, int64_t n) {
    for (int64_t i = 0; i < n; ++i) H(h)->s.step();
}
// set_dynamic_sgs, src/uniform/solver.rs:215-220.
void orc_set_dynamic_sgs(void* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test) {
    auto& s = H(h)->s;
    s.dynamic_smag = on != 0;
    s.smag_alpha = smag_alpha;
    s.nu_sm_min = nu_sm_min;
    s.eta_test = eta_test;
    if (!s.dynamic_smag) {
        s.nu_t_pre.clear();
        s.alpha_t_pre.clear();
    }
}

// compute_dynamic_sgs alone (src/uniform/solver.rs:562-828) on the current state.
void orc_compute_dynamic_sgs(void* h) { H(h)->s.compute_dynamic_sgs(); }

// out4 = cs_dyn_mean, cs_dyn_max, kappa_dyn_mean, kappa_dyn_max; the per-node
// nu_t_pre / alpha_t_pre when the model has run (NULL to skip).
void orc_dynamic_stats(void* h, double* out4, double* nu_t_pre, double* alpha_t_pre) {
    auto& s = H(h)->s;
    out4[0] = s.cs_dyn_mean;
    out4[1] = s.cs_dyn_max;
    out4[2] = s.kappa_dyn_mean;
    out4[3] = s.kappa_dyn_max;
    const size_t n = size_t(s.nx) * s.ny;
    if (nu_t_pre && s.nu_t_pre.size() == n) std::memcpy(nu_t_pre, s.nu_t_pre.data(), n * 8);
    if (alpha_t_pre && s.alpha_t_pre.size() == n) std::memcpy(alpha_t_pre, s.alpha_t_pre.data(), n * 8);
}

// interpolate_field, src/uniform/snapshot.rs:102-131.
void orc_interpolate_field(const double* src, int64_t nx0, int64_t ny0, int64_t nx1, int64_t ny1, double* dst) {
    if (nx0 == nx1 && ny0 == ny1) {
        std::memcpy(dst, src, size_t(nx0 * ny0) * 8);
        return;
    }
    for (int64_t iy = 0; iy < ny1; ++iy) {
        const double vy = ny1 > 1 ? double(iy) / double(ny1 - 1) : 0.0;
        const double sy = vy * double(ny0 - 1);
        const int64_t y0 = (int64_t)std::floor(sy);
        const int64_t y1 = std::min<int64_t>(y0 + 1, ny0 - 1);
        const double wy = sy - double(y0);
        for (int64_t ix = 0; ix < nx1; ++ix) {
            const double vx = nx1 > 1 ? double(ix) / double(nx1 - 1) : 0.0;
            const double sx = vx * double(nx0 - 1);
            const int64_t x0 = (int64_t)std::floor(sx);
            const int64_t x1 = std::min<int64_t>(x0 + 1, nx0 - 1);
            const double wx = sx - double(x0);
            const double v00 = src[y0 * nx0 + x0], v10 = src[y0 * nx0 + x1];
            const double v01 = src[y1 * nx0 + x0], v11 = src[y1 * nx0 + x1];
            dst[iy * nx1 + ix] = v00 * (1.0 - wx) * (1.0 - wy) + v10 * wx * (1.0 - wy) + v01 * (1.0 - wx) * wy +
                                 v11 * wx * wy;
        }
    }
}

double orc_lilly_coefficient(double num, double den) { return orc::lilly_coefficient(num, den); }

// mixed_factor, src/uniform/solver.rs:1195-1202.
double orc_mixed_factor(double a, double b, double alpha) { return std::pow(a, alpha) * std::pow(b, 1.0 - alpha); }

void orc_collide(void* h, int64_t step) { H(h)->s.collide(step); }
void orc_stream(void* h) { H(h)->s.stream(); }
void orc_bounce_back(void* h) { H(h)->s.apply_bounce_back(); }
void orc_thermal_bc(void* h) { H(h)->s.apply_thermal_boundary_conditions(); }
void orc_macro(void* h) { H(h)->s.update_macroscopic(); }
void orc_noslip(void* h) { H(h)->s.enforce_wall_velocity(); }
void orc_set_time_step(void* h, int64_t t) { H(h)->s.time_step = t; }

void orc_init_from_fields(void* h, const double* rho, const double* ux, const double* uy, const double* t) {
    H(h)->s.init_from_fields(rho, ux, uy, t);
}

void orc_get_fields(void* h, double* rho, double* ux, double* uy, double* t, double* nu_t, double* fy) {
    S& s = H(h)->s;
    size_t n = size_t(s.nx) * s.ny;
    if (rho) std::memcpy(rho, s.rho.data(), n * 8);
    if (ux) std::memcpy(ux, s.ux.data(), n * 8);
    if (uy) std::memcpy(uy, s.uy.data(), n * 8);
    if (t) std::memcpy(t, s.temperature.data(), n * 8);
    if (nu_t) std::memcpy(nu_t, s.nu_t.data(), n * 8);
    if (fy) std::memcpy(fy, s.fy_node.data(), n * 8);
}

void orc_set_fields(void* h, const double* rho, const double* ux, const double* uy, const double* t,
                    const double* fy) {
    S& s = H(h)->s;
    size_t n = size_t(s.nx) * s.ny;
    if (rho) std::memcpy(s.rho.data(), rho, n * 8);
    if (ux) std::memcpy(s.ux.data(), ux, n * 8);
    if (uy) std::memcpy(s.uy.data(), uy, n * 8);
    if (t) std::memcpy(s.temperature.data(), t, n * 8);
    if (fy) std::memcpy(s.fy_node.data(), fy, n * 8);
}

void orc_get_pops(void* h, double* f, double* g) {
    S& s = H(h)->s;
    size_t n = size_t(s.nx) * s.ny;
    if (f) std::memcpy(f, s.f.data(), n * 9 * 8);
    if (g) std::memcpy(g, s.g.data(), n * 9 * 8);
}

void orc_set_pops(void* h, const double* f, const double* g) {
    S& s = H(h)->s;
    size_t n = size_t(s.nx) * s.ny;
    if (f) std::memcpy(s.f.data(), f, n * 9 * 8);
    if (g) std::memcpy(s.g.data(), g, n * 9 * 8);
}

void orc_info(void* h, double* out) {
    S& s = H(h)->s;
    out[0] = s.nu;
    out[1] = s.alpha;
    out[2] = s.alpha_phys;
    out[3] = s.beta_eff;
    out[4] = s.lz;
    out[5] = s.lx;
    out[6] = s.tau;
    out[7] = s.tau_t;
    out[8] = double(s.time_step);
    out[9] = double(s.spin_up_steps);
}

void orc_diag(void* h, double* out) {
    S& s = H(h)->s;
    const int nx = s.nx, ny = s.ny, n = nx * ny;
    out[0] = s.nusselt_hot();
    out[1] = s.nusselt_cold();
    out[2] = s.nusselt_hot_wall_link();
    // total_mass, src/uniform/solver.rs:1012-1014.
    double m = 0.0;
    for (int k = 0; k < n; ++k) m += s.rho[k];
    out[3] = m;
    // total_f_mass, src/uniform/solver.rs:1018-1020.
    double mf = 0.0;
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < 9; ++i) mf += s.f[k][i];
    out[4] = mf;
    // max |u| (src/main.rs:209-214), max |u_y| (post.rs:153-155), nu_t max (main.rs:172-175).
    double mu = 0.0, muy = 0.0, mnt = 0.0;
    for (int k = 0; k < n; ++k) {
        mu = std::fmax(mu, std::fmax(std::fabs(s.ux[k]), std::fabs(s.uy[k])));
        muy = std::fmax(muy, std::fabs(s.uy[k]));
        mnt = std::fmax(mnt, std::fabs(s.nu_t[k]));
    }
    out[5] = mu;
    out[6] = muy;
    out[7] = mnt;
    // check_finite, post.rs:406-411.
    bool fin = true;
    for (int k = 0; k < n && fin; ++k)
        fin = std::isfinite(s.temperature[k]) && std::isfinite(s.ux[k]) && std::isfinite(s.uy[k]) &&
              std::isfinite(s.rho[k]) && s.rho[k] > 0.0;
    out[8] = fin ? 1.0 : 0.0;
    // y_plus_hot, post.rs:182-199 (y_plus(y, u_tau, nu) = y*u_tau/nu).
    double sum = 0.0;
    for (int iy = 1; iy < ny - 1; ++iy) {
        double nu_eff = s.nu + s.nu_t[s.idx(1, iy)];
        double du = std::fabs(s.uy[s.idx(1, iy)] - s.uy[s.idx(0, iy)]);
        double tau_w = nu_eff * du;
        double u_tau = std::sqrt(std::fmax(tau_w, 0.0));
        sum += 0.5 * u_tau / s.nu;
    }
    out[9] = sum / double(ny - 2);
    // nusselt_volume, post.rs:117-134.
    double sv = 0.0;
    for (int iy = 1; iy < ny - 1; ++iy)
        for (int ix = 1; ix < nx - 1; ++ix) {
            int k = s.idx(ix, iy);
            sv += s.uy[k] * s.temperature[k];
        }
    double conv = sv / double((nx - 2) * (ny - 2));
    out[10] = 1.0 + conv * s.lz / orc::DELTA_T;
}

double orc_feq(int32_t i, double rho, double ux, double uy) { return orc::feq<double>(i, rho, ux, uy); }
double orc_geq(int32_t i, double t, double ux, double uy, int32_t order) {
    return orc::geq<double>(i, t, ux, uy, order);
}
double orc_weight(int32_t i) { return orc::W[i]; }
void orc_velocity(int32_t i, int32_t* cx, int32_t* cy) {
    *cx = orc::CX[i];
    *cy = orc::CY[i];
}
void orc_nusselt(void* h, double* hot, double* cold) {
    *hot = H(h)->s.nusselt_hot();
    *cold = H(h)->s.nusselt_cold();
}

struct OrcAvg {
    std::vector<double> sum_ux, sum_uy, sum_t, sum_nu_t, sum_uu;
    int64_t n = 0;
};

void* orc_avg_create(int64_t n) {
    OrcAvg* a = new OrcAvg;
    a->sum_ux.assign(n, 0.0);
    a->sum_uy.assign(n, 0.0);
    a->sum_t.assign(n, 0.0);
    a->sum_nu_t.assign(n, 0.0);
    a->sum_uu.assign(n, 0.0);
    return a;
}
void orc_avg_destroy(void* a) { delete static_cast<OrcAvg*>(a); }

// TimeAverager::accumulate, src/uniform/post.rs:37-49.
void orc_avg_accumulate(void* av, void* h) {
    OrcAvg* a = static_cast<OrcAvg*>(av);
    S& s = H(h)->s;
    size_t n = size_t(s.nx) * s.ny;
    for (size_t k = 0; k < n; ++k) {
        double ux = s.ux[k], uy = s.uy[k];
        a->sum_ux[k] += ux;
        a->sum_uy[k] += uy;
        a->sum_t[k] += s.temperature[k];
        a->sum_nu_t[k] += s.nu_t[k];
        a->sum_uu[k] += ux * ux + uy * uy;
    }
    a->n += 1;
}

// TimeAverager::means, src/uniform/post.rs:52-56.
int64_t orc_avg_means(void* av, double* ux, double* uy, double* t, double* nu_t, double* uu) {
    OrcAvg* a = static_cast<OrcAvg*>(av);
    double inv = 1.0 / double(a->n);
    for (size_t k = 0; k < a->sum_ux.size(); ++k) {
        if (ux) ux[k] = a->sum_ux[k] * inv;
        if (uy) uy[k] = a->sum_uy[k] * inv;
        if (t) t[k] = a->sum_t[k] * inv;
        if (nu_t) nu_t[k] = a->sum_nu_t[k] * inv;
        if (uu) uu[k] = a->sum_uu[k] * inv;
    }
    return a->n;
}

double orc_nusselt_from_mean(void* h, const double* t, int32_t hot) {
    S& s = H(h)->s;
    const int nx = s.nx, ny = s.ny;
    double sum = 0.0;
    for (int iy = 0; iy < ny; ++iy) {
        double grad = hot ? t[s.idx(1, iy)] - t[s.idx(2, iy)] : t[s.idx(nx - 3, iy)] - t[s.idx(nx - 2, iy)];
        sum += std::fabs(grad);
    }
    return (sum / double(ny)) * s.lz / orc::DELTA_T;
}

}  // extern "C"
