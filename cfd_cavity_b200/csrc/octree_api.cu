// octree_api.cu -- the cav_octree_* entry points of include/cavity.h (host
// code only): octree::solver::CavitySolver methods onto a cav::oct::Octree.
#include "octree.cuh"
#include "snapshot.cuh"

using namespace cav;
using namespace cav::oct;

namespace cav {
namespace oct {
Octree* make_octree_f64();
Octree* make_octree_f32();
Octree* make_octree_f32_f16();
Octree* make_octree_f32_f16g();
}  // namespace oct
}  // namespace cav

struct cav_octree {
    std::unique_ptr<Octree> o;
};

namespace {
thread_local std::string g_oct_create_error;

int ofail(cav_octree* h, int code, const std::string& msg) {
    if (h && h->o) h->o->err = msg;
    else g_oct_create_error = msg;
    return code;
}

template <class F>
int oguarded(cav_octree* h, F&& fn) {
    if (!h || !h->o) return ofail(nullptr, CAV_ERR_ARG, "null handle");
    try {
        cudaSetDevice(h->o->p.device);
        return fn(*h->o);
    } catch (const CudaError& e) {
        return ofail(h, CAV_ERR_CUDA, std::string(e.where) + ": " + cudaGetErrorString(e.e));
    } catch (const ArgError& e) {
        return ofail(h, e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return ofail(h, CAV_ERR_NOMEM, "host allocation failed");
    }
}
}  // namespace

extern "C" {

int cav_octree_default_params(cav_octree_params* p) {
    if (!p) return CAV_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    // cli.rs defaults of the octree mode: 256 x 1024 base, --bl-width 16, levels 2
    p->nx0 = 256;
    p->ny0 = 1024;
    p->bl_width = 16;
    p->ra = 1.0e6;
    p->pr = 0.71;
    p->utarget = 0.02;
    p->seed = 42;
    p->jobs = 1;
    p->odd_exact = 0;
    p->levels = 2;
    p->nu_start_mult = 1.0;
    p->precision = CAV_OCT_F64;
    p->device = 0;
    p->cs = 0.0;
    p->pr_t = 0.9;
    return CAV_OK;
}

int cav_octree_create(const cav_octree_params* p, cav_octree** out) {
    if (!p || !out) {
        g_oct_create_error = "null argument";
        return CAV_ERR_ARG;
    }
    *out = nullptr;
    std::unique_ptr<Octree> o;
    try {
        switch (p->precision) {
            case CAV_OCT_F64: o.reset(make_octree_f64()); break;
            case CAV_OCT_F32: o.reset(make_octree_f32()); break;
            case CAV_OCT_F32_F16: o.reset(make_octree_f32_f16()); break;
            case CAV_OCT_F32_F16G: o.reset(make_octree_f32_f16g()); break;
            default: g_oct_create_error = "unknown precision"; return CAV_ERR_ARG;
        }
        o->setup(*p);
    } catch (const CudaError& e) {
        g_oct_create_error = std::string(e.where) + ": " + cudaGetErrorString(e.e);
        return CAV_ERR_CUDA;
    } catch (const ArgError& e) {
        g_oct_create_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_oct_create_error = "host allocation failed";
        return CAV_ERR_NOMEM;
    }
    *out = new cav_octree{std::move(o)};
    return CAV_OK;
}

int cav_octree_destroy(cav_octree* h) {
    if (!h) return CAV_ERR_ARG;
    if (h->o) cudaSetDevice(h->o->p.device);
    delete h;
    return CAV_OK;
}

const char* cav_octree_last_error(const cav_octree* h) {
    if (!h || !h->o) return g_oct_create_error.c_str();
    return h->o->err.c_str();
}

int cav_octree_step(cav_octree* h, int64_t n) {
    if (n < 0) return ofail(h, CAV_ERR_ARG, "negative step count");
    return oguarded(h, [&](Octree& o) {
        o.step(n);
        return CAV_OK;
    });
}

int cav_octree_get_info(cav_octree* h, cav_octree_info* out) {
    if (!out) return ofail(h, CAV_ERR_ARG, "null output");
    return oguarded(h, [&](Octree& o) {
        std::memset(out, 0, sizeof(*out));
        out->nu = o.nu;
        out->alpha = o.alpha;
        out->beta_eff_coarse = o.beta_c;
        for (int l = 0; l < 3; ++l) out->tau_plus[l] = l < o.levels ? o.tau_p[l] : 0.0;
        out->xi_even = o.xiA[0];
        out->xi_odd = o.xiA[1];
        out->xi_thermal = o.xiA[2];
        if (o.levels == 3) {
            out->xi_even_sub = o.xiB[0];
            out->xi_odd_sub = o.xiB[1];
            out->xi_thermal_sub = o.xiB[2];
        }
        out->time_step = o.time_step;
        out->spin_up_steps = o.spin_up;
        out->levels = o.levels;
        out->precision = o.p.precision;
        out->nx[0] = o.nx0;
        out->ny[0] = o.ny0;
        out->nx[1] = out->nx[2] = o.nx1;
        out->ny[1] = out->ny[2] = o.ny1;
        if (o.levels == 3) {
            out->nx[3] = out->nx[4] = o.nx2;
            out->ny[3] = out->ny[4] = o.ny2;
        }
        int64_t tot = 0;
        for (int l = 0; l < 5; ++l) tot += int64_t(out->nx[l]) * out->ny[l];
        out->n_nodes_total = tot;
        out->n_ghosts = 2 * o.n_ghost;
        out->n_coincident = o.n_co0 + o.n_co1;
        out->n_ghosts_sub = o.levels == 3 ? 2 * o.n_ghost2 : 0;
        out->n_coincident_sub = o.levels == 3 ? o.n_co2_0 + o.n_co2_1 : 0;
        return CAV_OK;
    });
}

int cav_octree_get_level(cav_octree* h, int32_t level, double* rho, double* ux, double* uy, double* t, double* f,
                         double* g) {
    return oguarded(h, [&](Octree& o) {
        o.get_level(level, rho, ux, uy, t, f, g);
        return CAV_OK;
    });
}

int cav_octree_set_level(cav_octree* h, int32_t level, const double* rho, const double* ux, const double* uy,
                         const double* t, const double* f, const double* g) {
    return oguarded(h, [&](Octree& o) {
        o.set_level(level, rho, ux, uy, t, f, g);
        return CAV_OK;
    });
}

int cav_octree_restart_level(cav_octree* h, int32_t level, const double* rho, const double* ux, const double* uy,
                             const double* t) {
    if (!rho || !ux || !uy || !t) return ofail(h, CAV_ERR_ARG, "null field");
    return oguarded(h, [&](Octree& o) {
        o.restart_level(level, rho, ux, uy, t);
        return CAV_OK;
    });
}

int cav_octree_set_time_step(cav_octree* h, int64_t t) {
    return oguarded(h, [&](Octree& o) {
        o.set_time_step(t);
        return CAV_OK;
    });
}

int cav_octree_snapshot_write(cav_octree* h, const char* path, uint64_t step) {
    if (!path) return ofail(h, CAV_ERR_ARG, "null path");
    return oguarded(h, [&](Octree& o) {
        snap::Oct s;
        s.levels = uint32_t(o.levels);
        s.step = step;
        const int n_lv = o.levels == 3 ? 5 : 3;
        s.grids.resize(n_lv);
        for (int l = 0; l < n_lv; ++l) {
            snap::Fields& g = s.grids[l];
            g.nx = l == 0 ? o.nx0 : (l <= 2 ? o.nx1 : o.nx2);
            g.ny = l == 0 ? o.ny0 : (l <= 2 ? o.ny1 : o.ny2);
            const size_t n = size_t(g.nx * g.ny);
            g.rho.resize(n);
            g.ux.resize(n);
            g.uy.resize(n);
            g.t.resize(n);
            o.get_level(l, g.rho.data(), g.ux.data(), g.uy.data(), g.t.data(), nullptr, nullptr);
        }
        snap::write_octsnap(path, s);
        return CAV_OK;
    });
}

int cav_octree_restart_from_snapshot(cav_octree* h, const char* path) {
    if (!path) return ofail(h, CAV_ERR_ARG, "null path");
    return oguarded(h, [&](Octree& o) {
        const snap::Oct s = snap::read_octsnap(path);
        const int n_lv = o.levels == 3 ? 5 : 3;
        if (int(s.levels) != o.levels || int(s.grids.size()) != n_lv)
            throw ArgError{CAV_ERR_ARG, "octree restart: snapshot levels differ from the solver's"};
        for (int l = 0; l < n_lv; ++l) {
            const int64_t nx = l == 0 ? o.nx0 : (l <= 2 ? o.nx1 : o.nx2);
            const int64_t ny = l == 0 ? o.ny0 : (l <= 2 ? o.ny1 : o.ny2);
            if (s.grids[l].nx != nx || s.grids[l].ny != ny)
                throw ArgError{CAV_ERR_ARG, "octree restart: grid " + std::to_string(l) +
                                                " differs from the solver's (the same level layout is required)"};
        }
        for (int l = 0; l < n_lv; ++l) {
            const snap::Fields& g = s.grids[l];
            o.restart_level(l, g.rho.data(), g.ux.data(), g.uy.data(), g.t.data());
        }
        o.set_time_step(0);
        return CAV_OK;
    });
}

int cav_octree_couple(cav_octree* h, int32_t which) {
    return oguarded(h, [&](Octree& o) {
        o.debug_phase(which);
        return CAV_OK;
    });
}

int cav_octree_diag(cav_octree* h, cav_octree_diag_out* out) {
    if (!out) return ofail(h, CAV_ERR_ARG, "null output");
    return oguarded(h, [&](Octree& o) {
        double d[10];
        o.diag(d);
        out->nu_hot = d[0];
        out->nu_hot_link0 = d[1];
        out->nu_cold = d[2];
        out->nu_hot_fine = d[3];
        out->max_u = d[4];
        out->mass = d[5];
        out->max_rho_dev = d[6];
        out->max_rho_dev_ifaces = d[7];
        out->finite = d[8];
        out->y_plus_fine = d[9];
        return CAV_OK;
    });
}

int cav_octree_check_guards(cav_octree* h, double max_u_abort) {
    return oguarded(h, [&](Octree& o) {
        double d[10];
        o.diag(d);
        // check_guards (src/octree/solver.rs:1019-1038): max_u first, then finiteness
        if (d[4] > max_u_abort) {
            o.err = "max_u = " + std::to_string(d[4]) + " exceeds the guard " + std::to_string(max_u_abort);
            return int(CAV_ERR_MAXU);
        }
        if (d[8] != 1.0) {
            o.err = "divergence: non-finite values";
            return int(CAV_ERR_DIVERGED);
        }
        return int(CAV_OK);
    });
}

int cav_octree_sync(cav_octree* h) {
    return oguarded(h, [&](Octree& o) {
        o.sync();
        return CAV_OK;
    });
}

int cav_octree_get_stream(cav_octree* h, void** stream) {
    if (!stream) return ofail(h, CAV_ERR_ARG, "null output");
    return oguarded(h, [&](Octree& o) {
        *stream = (void*)o.stream;
        return CAV_OK;
    });
}

int cav_octree_launch_count(cav_octree* h, int64_t* n) {
    if (!n) return ofail(h, CAV_ERR_ARG, "null output");
    return oguarded(h, [&](Octree& o) {
        *n = o.launches;
        return CAV_OK;
    });
}

int cav_octree_set_level_kernel(cav_octree* h, int32_t kind) {
    return oguarded(h, [&](Octree& o) {
        o.set_level_kernel(kind);
        return CAV_OK;
    });
}

int cav_octree_get_level_kernel(cav_octree* h, int32_t* kind) {
    if (!kind) return ofail(h, CAV_ERR_ARG, "null output");
    return oguarded(h, [&](Octree& o) {
        *kind = o.get_level_kernel();
        return CAV_OK;
    });
}

int cav_octree_set_dynamic_sgs(cav_octree* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test) {
    return oguarded(h, [&](Octree& o) {
        o.set_dynamic_sgs(on != 0, smag_alpha, nu_sm_min, eta_test);
        return CAV_OK;
    });
}

int cav_octree_dynamic_stats(cav_octree* h, double* out14) {
    if (!out14) return ofail(h, CAV_ERR_ARG, "null output");
    return oguarded(h, [&](Octree& o) {
        o.dynamic_stats(out14);
        return CAV_OK;
    });
}

int cav_octree_get_nu_t(cav_octree* h, int32_t level, double* nu_t, double* alpha_t) {
    return oguarded(h, [&](Octree& o) {
        o.get_nut(level, nu_t, alpha_t);
        return CAV_OK;
    });
}

}  // extern "C"
