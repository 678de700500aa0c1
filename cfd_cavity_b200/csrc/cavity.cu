// cavity.cu -- the C ABI declared in include/cavity.h (host code only).
//
// Every entry point maps one CavitySolver method or field access of the
// reference (cited in include/cavity.h) onto a cav::Solver object; errors
// become status codes and a per-handle message instead of panics.
#include <map>
#include <mutex>

#include "batch.cuh"
#include "snapshot.cuh"
#include "solver.cuh"

using namespace cav;

namespace {
thread_local std::string g_create_error;
}  // namespace

struct cav_handle {
    std::unique_ptr<Solver> s;
};

struct cav_batch {
    std::unique_ptr<BatchBase> b;
};

namespace {

int fail(cav_handle* h, int code, const std::string& msg) {
    if (h && h->s) h->s->err = msg;
    else g_create_error = msg;
    return code;
}

template <class F>
int guarded(cav_handle* h, F&& fn) {
    if (!h || !h->s) return fail(nullptr, CAV_ERR_ARG, "null handle");
    try {
        cudaSetDevice(h->s->p.device);
        fn(*h->s);
        return CAV_OK;
    } catch (const CudaError& e) {
        return fail(h, CAV_ERR_CUDA, std::string(e.where) + ": " + cudaGetErrorString(e.e));
    } catch (const ArgError& e) {
        return fail(h, e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return fail(h, CAV_ERR_NOMEM, "host allocation failed");
    }
}

// CavitySolver::new (src/uniform/solver.rs:108-210) on the device: validates
// the parameters, derives the lattice units, allocates and uploads the
// initial state.  Throws ArgError / CudaError.  `shared` (may be null) is a
// stream the solver adopts instead of creating its own.
Solver* build_solver(const cav_params& p, cudaStream_t shared) {
    if (p.nx < 4 || p.ny < 4 || p.nx > 65536 || p.ny > 65536)
        throw ArgError{CAV_ERR_ARG, "nx and ny must be in [4, 65536]"};
    if (p.precision < CAV_PREC_F64 || p.precision > CAV_PREC_F16GSR) throw ArgError{CAV_ERR_ARG, "unknown precision"};
    if (p.geq_order != 1 && p.geq_order != 2) throw ArgError{CAV_ERR_ARG, "geq_order must be 1 or 2"};
    if (p.init_mode != CAV_INIT_LINEAR && p.init_mode != CAV_INIT_ZERO) throw ArgError{CAV_ERR_ARG, "unknown init_mode"};
    Units U = derive_units(p);
    std::unique_ptr<Solver> s(make_solver(p.precision));
    s->p = p;
    s->p.t_hot_profile = nullptr;
    s->U = U;
    s->spin_up = std::min<int64_t>(std::max<int64_t>(p.ny / 10, 200), 2000);
    s->nu_start_mult = std::fmax(p.nu_start_mult, 1.0);
    s->t_hot.assign(p.ny, 0.5);
    if (p.t_hot_profile)
        for (int i = 0; i < p.ny; ++i) s->t_hot[i] = p.t_hot_profile[i];
    s->pitch = (p.nx + 31) / 32 * 32;
    s->stream = shared;
    CK(cudaSetDevice(p.device));
    s->alloc();
    // Initial temperature, src/uniform/solver.rs:159-176 (row-major RNG order).
    std::vector<double> t0(size_t(p.nx) * p.ny);
    Rng rng(p.seed);
    for (int iy = 0; iy < p.ny; ++iy)
        for (int ix = 0; ix < p.nx; ++ix) {
            double xf = double(ix) / double(p.nx - 1);
            double t_lin = 0.5 + (-0.5 - 0.5) * xf;
            double pert = p.noise_amp * (2.0 * rng.next_f64() - 1.0);
            t0[size_t(iy) * p.nx + ix] = (p.init_mode == CAV_INIT_LINEAR) ? t_lin + pert : pert;
        }
    s->init_default(t0);
    return s.release();
}

}  // namespace

extern "C" {

const char* cav_version(void) { return "cfd_cavity_b200 0.1 (sm_100a)"; }

int cav_default_params(cav_params* p) {
    if (!p) return CAV_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->nx = 64;
    p->ny = 256;
    p->ra = 1.0e6;
    p->pr = 0.71;
    p->cs = 0.10;
    p->pr_t = 0.9;
    p->utarget = 0.02;
    p->seed = 42;
    p->jobs = 1;
    p->alpha_mult = 1.0;
    p->nu_start_mult = 1.0;
    p->has_nu_override = 0;
    p->nu_override = 0.0;
    p->init_mode = CAV_INIT_LINEAR;
    p->noise_amp = 1.0e-3;
    p->geq_order = 2;
    p->t_hot_profile = nullptr;
    p->t_cold = -0.5;
    p->precision = CAV_PREC_F64;
    p->device = 0;
    return CAV_OK;
}

int cav_create(const cav_params* pp, cav_handle** out) {
    if (!pp || !out) return fail(nullptr, CAV_ERR_ARG, "null argument");
    *out = nullptr;
    Solver* s = nullptr;
    try {
        s = build_solver(*pp, nullptr);
    } catch (const CudaError& e) {
        return fail(nullptr, e.e == cudaErrorMemoryAllocation ? CAV_ERR_NOMEM : CAV_ERR_CUDA,
                    std::string(e.where) + ": " + cudaGetErrorString(e.e));
    } catch (const ArgError& e) {
        return fail(nullptr, e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return fail(nullptr, CAV_ERR_NOMEM, "host allocation failed");
    }
    cav_handle* h = new cav_handle;
    h->s.reset(s);
    *out = h;
    return CAV_OK;
}

int cav_destroy(cav_handle* h) {
    if (!h) return CAV_ERR_ARG;
    if (h->s) cudaSetDevice(h->s->p.device);
    delete h;
    return CAV_OK;
}

const char* cav_last_error(const cav_handle* h) {
    if (h && h->s) return h->s->err.c_str();
    return g_create_error.c_str();
}

int cav_init_from_fields(cav_handle* h, const double* rho, const double* ux, const double* uy, const double* t) {
    if (!rho || !ux || !uy || !t) return fail(h, CAV_ERR_ARG, "init_from_fields: null field");
    return guarded(h, [&](Solver& s) { s.init_from_fields(rho, ux, uy, t); });
}

int cav_step(cav_handle* h, int64_t n) {
    if (n < 0) return fail(h, CAV_ERR_ARG, "negative step count");
    return guarded(h, [&](Solver& s) { s.step(n); });
}

int cav_get_fields(cav_handle* h, double* rho, double* ux, double* uy, double* t, double* nu_t, double* fy) {
    return guarded(h, [&](Solver& s) { s.get_fields(rho, ux, uy, t, nu_t, fy); });
}

int cav_set_fields(cav_handle* h, const double* rho, const double* ux, const double* uy, const double* t,
                   const double* fy) {
    return guarded(h, [&](Solver& s) { s.set_fields(rho, ux, uy, t, fy); });
}

int cav_get_populations(cav_handle* h, double* f, double* g) {
    return guarded(h, [&](Solver& s) { s.get_pops(f, g); });
}

int cav_set_populations(cav_handle* h, const double* f, const double* g) {
    return guarded(h, [&](Solver& s) { s.set_pops(f, g); });
}

int cav_get_info(cav_handle* h, cav_info* o) {
    if (!o) return fail(h, CAV_ERR_ARG, "null output");
    return guarded(h, [&](Solver& s) {
        o->nu = s.U.nu;
        o->alpha = s.U.alpha;
        o->alpha_phys = s.U.alpha_phys;
        o->beta_eff = s.U.beta_eff;
        o->lz = s.U.lz;
        o->lx = s.U.lx;
        o->tau = s.U.tau;
        o->tau_t = s.U.tau_t;
        o->time_step = s.time_step;
        o->spin_up_steps = s.spin_up;
        o->nx = s.p.nx;
        o->ny = s.p.ny;
        o->pitch = s.pitch;
        o->precision = s.p.precision;
    });
}

int cav_set_time_step(cav_handle* h, int64_t t) {
    if (t < 0) return fail(h, CAV_ERR_ARG, "negative time step");
    return guarded(h, [&](Solver& s) { s.time_step = t; });
}

int cav_diag(cav_handle* h, cav_diag_out* o) {
    if (!o) return fail(h, CAV_ERR_ARG, "null output");
    return guarded(h, [&](Solver& s) {
        double v[11];
        s.diag(v);
        o->nusselt_hot = v[0];
        o->nusselt_cold = v[1];
        o->nusselt_hot_wall_link = v[2];
        o->total_mass = v[3];
        o->total_f_mass = v[4];
        o->max_u = v[5];
        o->max_uy = v[6];
        o->nu_t_max = v[7];
        o->y_plus_hot = v[8];
        o->nusselt_volume = v[9];
        o->finite = v[10] == 0.0 ? 1 : 0;
    });
}

int cav_check_guards(cav_handle* h, double max_u_abort) {
    cav_diag_out d;
    int rc = cav_diag(h, &d);
    if (rc != CAV_OK) return rc;
    if (d.max_u > max_u_abort) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "max_u = %.5f above the %.2f guard", d.max_u, max_u_abort);
        return fail(h, CAV_ERR_MAXU, buf);
    }
    if (!d.finite) return fail(h, CAV_ERR_DIVERGED, "non-finite field (diverged)");
    return CAV_OK;
}

int cav_debug_phase(cav_handle* h, int32_t phase, int64_t step_arg) {
    return guarded(h, [&](Solver& s) { s.debug_phase(phase, step_arg); });
}

int cav_sample(cav_handle* h) {
    return guarded(h, [&](Solver& s) { s.sample(); });
}

int cav_reset_means(cav_handle* h) {
    return guarded(h, [&](Solver& s) { s.reset_means(); });
}

int cav_get_means(cav_handle* h, double* ux, double* uy, double* t, double* nu_t, double* uu, int64_t* n) {
    return guarded(h, [&](Solver& s) {
        int64_t c = s.get_means(ux, uy, t, nu_t, uu);
        if (n) *n = c;
    });
}

int cav_nusselt_from_mean(cav_handle* h, int32_t hot, double* out) {
    if (!out) return fail(h, CAV_ERR_ARG, "null output");
    return guarded(h, [&](Solver& s) {
        const int nx = s.p.nx, ny = s.p.ny;
        std::vector<double> t(size_t(nx) * ny);
        s.get_means(nullptr, nullptr, t.data(), nullptr, nullptr);
        double sum = 0.0;
        for (int iy = 0; iy < ny; ++iy) {
            const double* r = t.data() + size_t(iy) * nx;
            double grad = hot ? r[1] - r[2] : r[nx - 3] - r[nx - 2];
            sum += std::fabs(grad);
        }
        *out = (sum / double(ny)) * s.U.lz / 1.0;
    });
}

int cav_nu_accumulate(cav_handle* h, int32_t enable) {
    return guarded(h, [&](Solver& s) { s.nu_accumulate(enable != 0); });
}

int cav_nu_accumulated(cav_handle* h, double* hot, double* cold, int64_t* n) {
    return guarded(h, [&](Solver& s) { s.nu_accumulated(hot, cold, n); });
}

int cav_adjoint_run(cav_handle* h, const cav_adjoint_spec* spec, double* grad_theta, cav_adjoint_result* res) {
    if (!spec || !grad_theta || !res) return fail(h, CAV_ERR_ARG, "null argument");
    return guarded(h, [&](Solver& s) {
        double out[5];
        s.adjoint_run(spec->n_steps, spec->window_start, spec->checkpoint_every, grad_theta, out);
        res->objective = out[0];
        res->grad_cs = out[1];
        res->forward_ms = out[2];
        res->reverse_ms = out[3];
        res->checkpoints = int64_t(out[4]);
    });
}

int cav_sync(cav_handle* h) {
    return guarded(h, [&](Solver& s) { s.sync(); });
}

int cav_get_stream(cav_handle* h, void** stream) {
    if (!stream) return fail(h, CAV_ERR_ARG, "null output");
    return guarded(h, [&](Solver& s) { *stream = (void*)s.stream; });
}

int cav_set_step_kernel(cav_handle* h, int32_t kernel) {
    return guarded(h, [&](Solver& s) { s.set_step_kernel(kernel); });
}

int cav_get_step_kernel(cav_handle* h, int32_t* kernel) {
    if (!kernel) return fail(h, CAV_ERR_ARG, "null output");
    return guarded(h, [&](Solver& s) { *kernel = s.step_kernel(); });
}

int cav_snapshot_write_fields(const char* path, int64_t nx, int64_t ny, const double* rho, const double* ux,
                              const double* uy, const double* t) {
    if (!path || !rho || !ux || !uy || !t || nx < 1 || ny < 1) return fail(nullptr, CAV_ERR_ARG, "bad arguments");
    try {
        snap::write_cavsnap(path, nx, ny, rho, ux, uy, t);
    } catch (const ArgError& e) {
        return fail(nullptr, e.code, e.msg);
    }
    return CAV_OK;
}

int cav_snapshot_read_fields(const char* path, int64_t* nx, int64_t* ny, double* rho, double* ux, double* uy,
                             double* t) {
    if (!path || !nx || !ny) return fail(nullptr, CAV_ERR_ARG, "bad arguments");
    try {
        const snap::Fields F = snap::read_cavsnap(path);
        *nx = F.nx;
        *ny = F.ny;
        const size_t n = size_t(F.nx * F.ny);
        if (rho) std::memcpy(rho, F.rho.data(), n * 8);
        if (ux) std::memcpy(ux, F.ux.data(), n * 8);
        if (uy) std::memcpy(uy, F.uy.data(), n * 8);
        if (t) std::memcpy(t, F.t.data(), n * 8);
    } catch (const ArgError& e) {
        return fail(nullptr, e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return fail(nullptr, CAV_ERR_NOMEM, "host allocation failed");
    }
    return CAV_OK;
}

int cav_snapshot_write(cav_handle* h, const char* path) {
    if (!path) return fail(h, CAV_ERR_ARG, "null path");
    return guarded(h, [&](Solver& s) {
        const size_t n = size_t(s.p.nx) * s.p.ny;
        std::vector<double> r(n), u(n), v(n), t(n);
        s.get_fields(r.data(), u.data(), v.data(), t.data(), nullptr, nullptr);
        snap::write_cavsnap(path, s.p.nx, s.p.ny, r.data(), u.data(), v.data(), t.data());
    });
}

int cav_restart_from_snapshot(cav_handle* h, const char* path) {
    if (!path) return fail(h, CAV_ERR_ARG, "null path");
    return guarded(h, [&](Solver& s) {
        const snap::Fields F = snap::read_cavsnap(path);
        const int nx1 = s.p.nx, ny1 = s.p.ny;
        const size_t n0 = size_t(F.nx * F.ny), n1 = size_t(nx1) * ny1;
        // restart is not a hot path: temporary device buffers for the source
        // and the regridded fields
        struct Buf {
            double* p = nullptr;
            ~Buf() {
                if (p) cudaFree(p);
            }
        } src, dst;
        CK(cudaMalloc(&src.p, sizeof(double) * 4 * n0));
        CK(cudaMalloc(&dst.p, sizeof(double) * 4 * n1));
        const std::vector<double>* fs[4] = {&F.rho, &F.ux, &F.uy, &F.t};
        for (int q = 0; q < 4; ++q) {
            CK(cudaMemcpyAsync(src.p + q * n0, fs[q]->data(), sizeof(double) * n0, cudaMemcpyHostToDevice,
                               s.stream));
            if (F.nx == nx1 && F.ny == ny1) {
                CK(cudaMemcpyAsync(dst.p + q * n1, src.p + q * n0, sizeof(double) * n1, cudaMemcpyDeviceToDevice,
                                   s.stream));
            } else {
                const dim3 b(32, 4), g((nx1 + 31) / 32, (ny1 + 3) / 4);
                snap::k_regrid<<<g, b, 0, s.stream>>>(src.p + q * n0, int(F.nx), int(F.ny), dst.p + q * n1, nx1,
                                                      ny1);
                ++s.launches;
                CK(cudaGetLastError());
            }
        }
        s.init_from_device_fields(dst.p, dst.p + n1, dst.p + 2 * n1, dst.p + 3 * n1);
    });
}

int cav_set_dynamic_sgs(cav_handle* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test) {
    return guarded(h, [&](Solver& s) { s.set_dynamic_sgs(on != 0, smag_alpha, nu_sm_min, eta_test); });
}

int cav_dynamic_sgs_stats(cav_handle* h, double* out4) {
    if (!out4) return fail(h, CAV_ERR_ARG, "null output");
    return guarded(h, [&](Solver& s) { s.dynamic_stats(out4); });
}

int cav_launch_count(cav_handle* h, int64_t* n) {
    if (!n) return fail(h, CAV_ERR_ARG, "null output");
    return guarded(h, [&](Solver& s) { *n = s.launches; });
}

}  // extern "C"

namespace cav {
Solver* make_solver_f64();
Solver* make_solver_f32();
Solver* make_solver_f16();
Solver* make_solver_bf16();
Solver* make_solver_f16g();
Solver* make_solver_f16sr();
Solver* make_solver_bf16sr();
Solver* make_solver_f16gsr();

BatchBase* make_batch_f64();
BatchBase* make_batch_f32();
BatchBase* make_batch_f16();
BatchBase* make_batch_bf16();
BatchBase* make_batch_f16g();
BatchBase* make_batch_f16sr();
BatchBase* make_batch_bf16sr();
BatchBase* make_batch_f16gsr();

BatchBase* make_batch(int precision) {
    switch (precision) {
        case CAV_PREC_F64: return make_batch_f64();
        case CAV_PREC_F32: return make_batch_f32();
        case CAV_PREC_F16: return make_batch_f16();
        case CAV_PREC_BF16: return make_batch_bf16();
        case CAV_PREC_F16G: return make_batch_f16g();
        case CAV_PREC_F16SR: return make_batch_f16sr();
        case CAV_PREC_BF16SR: return make_batch_bf16sr();
        default: return make_batch_f16gsr();
    }
}

Solver* make_solver(int precision) {
    switch (precision) {
        case CAV_PREC_F64: return make_solver_f64();
        case CAV_PREC_F32: return make_solver_f32();
        case CAV_PREC_F16: return make_solver_f16();
        case CAV_PREC_BF16: return make_solver_bf16();
        case CAV_PREC_F16G: return make_solver_f16g();
        case CAV_PREC_F16SR: return make_solver_f16sr();
        case CAV_PREC_BF16SR: return make_solver_bf16sr();
        default: return make_solver_f16gsr();
    }
}
}  // namespace cav

// ---------------------------------------------------------------------------
// Batches.
// ---------------------------------------------------------------------------
namespace cav {
BatchBase* make_batch(int precision);
}

namespace {

std::mutex g_tune_mutex;
std::map<std::string, BatchTuning> g_tune_cache;  // grid class -> tuning chosen by the autotuner

// Grid class of a batch: storage format and the multiset of cavity sizes.
std::string grid_class(const BatchBase& b) {
    std::map<std::pair<int, int>, int> sizes;
    for (Solver* s : b.cavs) sizes[{s->p.nx, s->p.ny}] += 1;
    std::string key = "prec" + std::to_string(b.cavs[0]->p.precision);
    for (auto& kv : sizes)
        key += ":" + std::to_string(kv.first.first) + "x" + std::to_string(kv.first.second) + "*" +
               std::to_string(kv.second);
    return key;
}

BatchBase* build_batch(const cav_params* ps, int n) {
    if (n < 1) throw ArgError{CAV_ERR_ARG, "a batch needs at least one cavity"};
    for (int i = 1; i < n; ++i)
        if (ps[i].precision != ps[0].precision || ps[i].device != ps[0].device)
            throw ArgError{CAV_ERR_ARG, "all cavities of a batch share one precision and one device"};
    if (ps[0].precision < CAV_PREC_F64 || ps[0].precision > CAV_PREC_F16GSR)
        throw ArgError{CAV_ERR_ARG, "unknown precision"};
    CK(cudaSetDevice(ps[0].device));
    std::unique_ptr<BatchBase> b(make_batch(ps[0].precision));
    CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    for (int i = 0; i < n; ++i) b->cavs.push_back(build_solver(ps[i], b->stream));
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = g_tune_cache.find(grid_class(*b));
        if (it != g_tune_cache.end()) b->tun = it->second;
    }
    b->setup();
    return b.release();
}

int bfail(cav_batch* b, int code, const std::string& msg) {
    if (b && b->b) b->b->err = msg;
    else g_create_error = msg;
    return code;
}

template <class F>
int bguarded(cav_batch* b, F&& fn) {
    if (!b || !b->b) return bfail(nullptr, CAV_ERR_ARG, "null batch");
    try {
        cudaSetDevice(b->b->cavs[0]->p.device);
        fn(*b->b);
        return CAV_OK;
    } catch (const CudaError& e) {
        return bfail(b, CAV_ERR_CUDA, std::string(e.where) + ": " + cudaGetErrorString(e.e));
    } catch (const ArgError& e) {
        return bfail(b, e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return bfail(b, CAV_ERR_NOMEM, "host allocation failed");
    }
}

Solver* cavity_of(BatchBase& b, int32_t i) {
    if (i < 0 || i >= int32_t(b.cavs.size())) throw ArgError{CAV_ERR_ARG, "cavity index out of range"};
    return b.cavs[i];
}

}  // namespace

extern "C" {

int cav_batch_create(const cav_params* params, int32_t n, cav_batch** out) {
    if (!params || !out) return bfail(nullptr, CAV_ERR_ARG, "null argument");
    *out = nullptr;
    BatchBase* b = nullptr;
    try {
        b = build_batch(params, n);
    } catch (const CudaError& e) {
        return bfail(nullptr, e.e == cudaErrorMemoryAllocation ? CAV_ERR_NOMEM : CAV_ERR_CUDA,
                     std::string(e.where) + ": " + cudaGetErrorString(e.e));
    } catch (const ArgError& e) {
        return bfail(nullptr, e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return bfail(nullptr, CAV_ERR_NOMEM, "host allocation failed");
    }
    cav_batch* h = new cav_batch;
    h->b.reset(b);
    *out = h;
    return CAV_OK;
}

int cav_batch_destroy(cav_batch* b) {
    if (!b) return CAV_ERR_ARG;
    if (b->b) cudaSetDevice(b->b->cavs[0]->p.device);
    delete b;
    return CAV_OK;
}

const char* cav_batch_last_error(const cav_batch* b) {
    if (b && b->b) return b->b->err.c_str();
    return g_create_error.c_str();
}

int cav_batch_step(cav_batch* b, int64_t n) {
    if (n < 0) return bfail(b, CAV_ERR_ARG, "negative step count");
    return bguarded(b, [&](BatchBase& x) { x.step(n); });
}

int cav_batch_get_fields(cav_batch* b, int32_t i, double* rho, double* ux, double* uy, double* t, double* nu_t,
                         double* fy) {
    return bguarded(b, [&](BatchBase& x) { cavity_of(x, i)->get_fields(rho, ux, uy, t, nu_t, fy); });
}

int cav_batch_get_populations(cav_batch* b, int32_t i, double* f, double* g) {
    return bguarded(b, [&](BatchBase& x) { cavity_of(x, i)->get_pops(f, g); });
}

int cav_batch_diag(cav_batch* b, int32_t i, cav_diag_out* o) {
    if (!o) return bfail(b, CAV_ERR_ARG, "null output");
    return bguarded(b, [&](BatchBase& x) {
        double v[11];
        cavity_of(x, i)->diag(v);
        o->nusselt_hot = v[0];
        o->nusselt_cold = v[1];
        o->nusselt_hot_wall_link = v[2];
        o->total_mass = v[3];
        o->total_f_mass = v[4];
        o->max_u = v[5];
        o->max_uy = v[6];
        o->nu_t_max = v[7];
        o->y_plus_hot = v[8];
        o->nusselt_volume = v[9];
        o->finite = v[10] == 0.0 ? 1 : 0;
    });
}

int cav_batch_info(cav_batch* b, int32_t* n_cavities, int64_t* total_nodes, int64_t* time_step) {
    return bguarded(b, [&](BatchBase& x) {
        if (n_cavities) *n_cavities = int32_t(x.cavs.size());
        if (total_nodes) *total_nodes = x.total_nodes;
        if (time_step) *time_step = x.cavs[0]->time_step;
    });
}

int cav_batch_get_tuning(cav_batch* b, cav_batch_tuning* t) {
    if (!t) return bfail(b, CAV_ERR_ARG, "null output");
    return bguarded(b, [&](BatchBase& x) {
        t->rows_per_item = x.tun.rows_per_item;
        t->ctas_per_sm = x.tun.ctas_per_sm;
        t->kernel = x.tun.kernel;
    });
}

int cav_batch_set_tuning(cav_batch* b, const cav_batch_tuning* t) {
    if (!t) return bfail(b, CAV_ERR_ARG, "null tuning");
    return bguarded(b, [&](BatchBase& x) {
        BatchTuning bt;
        bt.rows_per_item = t->rows_per_item;
        bt.ctas_per_sm = t->ctas_per_sm;
        bt.kernel = t->kernel;
        x.set_tuning(bt);
    });
}

int cav_batch_autotune(cav_batch* b, int32_t trial_steps, cav_batch_tuning* chosen) {
    if (trial_steps < 1) return bfail(b, CAV_ERR_ARG, "trial_steps must be positive");
    return bguarded(b, [&](BatchBase& x) {
        // Trials run on a twin batch built from the same parameters, so the
        // state of this batch is untouched.
        std::vector<cav_params> ps;
        for (Solver* s : x.cavs) {
            cav_params p = s->p;
            p.t_hot_profile = s->t_hot.data();
            ps.push_back(p);
        }
        std::unique_ptr<BatchBase> twin(build_batch(ps.data(), int(ps.size())));
        // candidates: every kernel the format has, over the parameters that
        // kernel uses (BatchTuning): the persistent global-memory kernel over
        // tile heights and grid sizes, the shared-memory tile kernel over its
        // shapes and resident CTAs, the one-CTA-per-item kernels over item
        // heights
        const int prec = x.cavs[0]->p.precision;
        const bool p16 = prec >= CAV_PREC_F16;
        std::vector<BatchTuning> cand;
        auto add = [&](int k, int r, int c) {
            BatchTuning t;
            t.kernel = k;
            t.rows_per_item = r;
            t.ctas_per_sm = c;
            cand.push_back(t);
        };
        for (int r : {4, 8, 16})
            for (int c : {4, 8, 16}) add(0, r, c);
        for (int v : {1, 2})
            for (int c : {1, 2, 3, 4}) add(v, 4, c);
        for (int r : {1, 2, 4, 8}) add(3, r, 8);
        if (prec != CAV_PREC_F64)
            for (int r : {2, 4, 8}) add(4, r, 8);
        if (p16) {
            for (int r : {1, 2, 4, 8}) add(5, r, 8);
            for (int r : {4, 8})
                for (int c : {3, 4, 5}) add(6, r, c);
        }
        // each candidate timed three times (after its warm-up steps), the
        // median kept: one-off noise cannot pick the winner
        BatchTuning best = x.tun;
        double best_ms = 1e300;
        for (const BatchTuning& t : cand) {
            twin->set_tuning(t);
            double ms[3];
            for (double& m : ms) m = twin->time_steps(trial_steps);
            std::sort(ms, ms + 3);
            if (ms[1] < best_ms) {
                best_ms = ms[1];
                best = t;
            }
        }
        x.set_tuning(best);
        {
            std::lock_guard<std::mutex> lk(g_tune_mutex);
            g_tune_cache[grid_class(x)] = best;
        }
        if (chosen) {
            chosen->rows_per_item = best.rows_per_item;
            chosen->ctas_per_sm = best.ctas_per_sm;
            chosen->kernel = best.kernel;
        }
    });
}

int cav_batch_debug_stall_copies(cav_batch* b, int32_t on) {
    return bguarded(b, [&](BatchBase& x) { x.set_stall_copies(on != 0); });
}

int cav_batch_sync(cav_batch* b) {
    return bguarded(b, [&](BatchBase& x) { x.sync(); });
}

int cav_batch_get_stream(cav_batch* b, void** stream) {
    if (!stream) return bfail(b, CAV_ERR_ARG, "null output");
    return bguarded(b, [&](BatchBase& x) { *stream = (void*)x.stream; });
}

int cav_batch_launch_count(cav_batch* b, int64_t* n) {
    if (!n) return bfail(b, CAV_ERR_ARG, "null output");
    return bguarded(b, [&](BatchBase& x) { *n = x.launches; });
}

}  // extern "C"
