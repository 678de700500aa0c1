// solver.cuh -- the per-cavity solver object behind the C ABI.
//
// A Solver owns one cavity on one GPU: two population buffers (18 SoA planes
// each), the fields, the per-node Guo force and nu_t, and one CUDA stream.
// The state is held in one of two forms:
//   REF  post-stream populations + rho/u/T fields, i.e. exactly what the
//        reference's CavitySolver holds between step() calls
//        (src/uniform/solver.rs:35-104); produced by new(),
//        init_from_fields() and the debug phases;
//   PC   post-collision populations of the last collide, the form the fused
//        kernel streams from.
// step() runs one k_collide_ref (REF -> PC) if needed, then one k_fused per
// step, replaying a CUDA graph of GRAPH_STEPS fused steps once the spin-up
// ramps are over (all steps then share the same scalars).  Reading the
// state back runs k_materialize (PC -> REF) into the spare buffer.
//
// Impl<St> is instantiated once per storage format, each in its own
// translation unit (prec_*.cu): the FP64 one is compiled without fused
// multiply-add so that it reproduces the FP64 oracle bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cavity.h"
#include "diag.cuh"
#include "kernels.cuh"

namespace cav {

constexpr int GRAPH_STEPS = 64;  // even: a replay leaves the buffer parity unchanged
constexpr int BX = 32, BY = 4;
constexpr int DIAG_BLOCKS_MAX = 592;  // 4 x 148 SMs

// xorshift64* (src/uniform/rng.rs:5-31) for the initial temperature noise.
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed | 1ull) {}
    uint64_t next_u64() {
        uint64_t x = s;
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        s = x;
        return x * 0x2545F4914F6CDD1Dull;
    }
    double next_f64() { return double(next_u64() >> 11) / double(1ull << 53); }
};

struct CudaError {
    cudaError_t e;
    const char* where;
};

#define CK(call)                                               \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) throw CudaError{_e, #call};     \
    } while (0)

struct ArgError {
    int code;
    std::string msg;
};

// Lattice units of CavitySolver::new (src/uniform/solver.rs:123-154).
struct Units {
    double lz, lx, nu, alpha_phys, alpha, beta_eff, tau, tau_t;
};

inline Units derive_units(const cav_params& p) {
    Units u{};
    u.lz = double(p.ny - 1);
    u.lx = double(p.nx - 1);
    const double c_scale = 1.7;
    double nu_cal = std::pow(p.utarget * std::sqrt(p.pr) * u.lz / (c_scale * std::sqrt(p.ra)), 2.0 / 3.0);
    if (p.has_nu_override) {
        double n = p.nu_override;
        if (!(n > 0.0 && std::isfinite(n))) throw ArgError{CAV_ERR_ARG, "--nu must be > 0 and finite"};
        if (!(0.5 + 3.0 * n > 0.5005)) throw ArgError{CAV_ERR_TAU, "--nu too low: tau+ too close to 0.5"};
        u.nu = n;
    } else {
        u.nu = std::fmax(nu_cal, 0.002);
    }
    u.alpha_phys = u.nu / p.pr;
    u.alpha = u.alpha_phys * p.alpha_mult;
    u.beta_eff = p.ra * u.nu * u.alpha_phys / (u.lz * u.lz * u.lz);
    u.tau = 0.5 + 3.0 * u.nu;
    u.tau_t = 0.5 + 3.0 * u.alpha;
    if (!p.has_nu_override && !(u.tau > 0.505))
        throw ArgError{CAV_ERR_TAU, "tau too close to 0.5 (TRT floor: tau+ >= 0.506, nu >= 0.002)"};
    if (!(u.tau_t > 0.505)) throw ArgError{CAV_ERR_TAU, "tau_t too close to 0.5 (adjust alpha_mult)"};
    return u;
}

// Abstract solver; Impl<St> below holds the buffers of one storage format.
struct Solver {
    virtual ~Solver() = default;
    virtual void alloc() = 0;
    virtual void init_default(const std::vector<double>& t0) = 0;
    virtual void init_from_fields(const double* r, const double* u, const double* v, const double* t) = 0;
    virtual void step(int64_t n) = 0;
    virtual void get_fields(double* r, double* u, double* v, double* t, double* nut, double* fy) = 0;
    virtual void set_fields(const double* r, const double* u, const double* v, const double* t,
                            const double* fy) = 0;
    virtual void get_pops(double* f, double* g) = 0;
    virtual void set_pops(const double* f, const double* g) = 0;
    virtual void diag(double* out11) = 0;
    virtual void debug_phase(int phase, int64_t step_arg) = 0;
    virtual void sample() = 0;
    virtual void reset_means() = 0;
    virtual int64_t get_means(double* u, double* v, double* t, double* nut, double* uu) = 0;
    virtual void nu_accumulate(bool on) = 0;
    virtual void nu_accumulated(double* hot, double* cold, int64_t* n) = 0;
    virtual void sync() = 0;

    cav_params p{};
    Units U{};
    int64_t time_step = 0, spin_up = 0;
    double nu_start_mult = 1.0;
    std::vector<double> t_hot;
    int pitch = 0;
    cudaStream_t stream = nullptr;  // set before alloc() to share a stream (batches)
    bool own_stream = true;
    int64_t launches = 0;
    std::string err;
};

template <class St>
struct Impl final : Solver {
    using A = typename Fmt<St>::A;
    static constexpr bool SH = Fmt<St>::SHIFT;

    Geom G{};
    St* pop[2] = {nullptr, nullptr};
    A *rho = nullptr, *ux = nullptr, *uy = nullptr, *tt = nullptr, *fy = nullptr, *nut = nullptr;
    A* t_hot_d = nullptr;
    double *acc_hot = nullptr, *acc_cold = nullptr;
    double *partials = nullptr, *diag_out = nullptr;
    double* sums = nullptr;
    double* aos = nullptr;
    long long* step_dev = nullptr;   // step counter read by graph-replayed kernels
    long long step_dev_val = -1;     // host mirror of *step_dev
    int64_t n_samples = 0, n_acc = 0;
    bool acc_on = false;
    int cur = 0;
    bool pc_form = false;    // false: REF form in pop[cur]; true: PC form in pop[cur]
    bool ref_cached = false; // PC form with a materialized REF copy in pop[cur ^ 1]
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    dim3 blk{BX, BY}, grd{};

    ~Impl() override {
        for (auto& row : graph)
            for (auto& gx : row)
                if (gx) cudaGraphExecDestroy(gx);
        void* bufs[] = {pop[0], pop[1], rho, ux, uy, tt, fy, nut, t_hot_d, acc_hot, acc_cold,
                        partials, diag_out, sums, aos, step_dev};
        for (void* b : bufs)
            if (b) cudaFree(b);
        if (stream && own_stream) cudaStreamDestroy(stream);
    }

    size_t field_elems() const { return size_t(G.ny) * G.pitch; }

    void alloc() override {
        G.nx = p.nx;
        G.ny = p.ny;
        G.pitch = pitch;
        G.plane = (long long)p.ny * pitch;
        if ((long long)NPLANES * G.plane >= (1ll << 31))
            throw ArgError{CAV_ERR_ARG, "grid too large: 18 * ny * pitch must stay below 2^31 elements"};
        grd = dim3((p.nx + BX - 1) / BX, (p.ny + BY - 1) / BY);
        if (!stream) {
            CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            own_stream = true;
        } else {
            own_stream = false;
        }
        const size_t pop_bytes = sizeof(St) * NPLANES * field_elems();
        for (int b = 0; b < 2; ++b) {
            CK(cudaMalloc(&pop[b], pop_bytes));
            CK(cudaMemsetAsync(pop[b], 0, pop_bytes, stream));
        }
        A** fl[] = {&rho, &ux, &uy, &tt, &fy, &nut};
        for (A** f : fl) {
            CK(cudaMalloc(f, sizeof(A) * field_elems()));
            CK(cudaMemsetAsync(*f, 0, sizeof(A) * field_elems(), stream));
        }
        CK(cudaMalloc(&t_hot_d, sizeof(A) * p.ny));
        std::vector<A> th(p.ny);
        for (int i = 0; i < p.ny; ++i) th[i] = A(t_hot[i]);
        CK(cudaMemcpyAsync(t_hot_d, th.data(), sizeof(A) * p.ny, cudaMemcpyHostToDevice, stream));
        CK(cudaMalloc(&acc_hot, sizeof(double) * p.ny));
        CK(cudaMalloc(&acc_cold, sizeof(double) * p.ny));
        CK(cudaMemsetAsync(acc_hot, 0, sizeof(double) * p.ny, stream));
        CK(cudaMemsetAsync(acc_cold, 0, sizeof(double) * p.ny, stream));
        CK(cudaMalloc(&partials, sizeof(double) * DIAG_NPART * DIAG_BLOCKS_MAX));
        CK(cudaMalloc(&diag_out, sizeof(double) * 16));
        CK(cudaMalloc(&step_dev, sizeof(long long)));
        CK(cudaStreamSynchronize(stream));
    }

    // Per-step scalars of collide(step), src/uniform/solver.rs:421-454 and
    // ramp_nu_alpha :390-410, evaluated in FP64 as the reference does.
    StepScalars<A> scalars(int64_t s) const {
        double beta = s < spin_up ? U.beta_eff * (double(s) / double(spin_up)) : U.beta_eff;
        double nu_eff = U.nu, alpha_eff = U.alpha;
        if (s < spin_up) {
            double x = double(s) / double(spin_up);
            double nu_start = U.nu * nu_start_mult;
            nu_eff = nu_start * std::pow(U.nu / nu_start, x);
            double alpha_start = U.alpha * nu_start_mult;
            alpha_eff = alpha_start * std::pow(U.alpha / alpha_start, x);
        }
        StepScalars<A> c;
        c.tau_s = A(0.5 + 3.0 * std::fmax(nu_eff, 0.002 / 3.0));
        c.beta = A(beta);
        c.nu = A(nu_eff);
        c.alpha = A(alpha_eff);
        c.cs = A(p.cs);
        c.pr_t = A(p.pr_t);
        c.inv_tau_s = A(1.0 / (0.5 + 3.0 * std::fmax(nu_eff, 0.002 / 3.0)));
        c.inv_pr_t = A(1.0 / p.pr_t);
        c.t_cold = A(p.t_cold);
        c.geq_order = p.geq_order;
        c.t_hot = t_hot_d;
        c.sr_seed = uint32_t(p.seed) ^ uint32_t(p.seed >> 32) ^ 0x5bd1e995u;
        c.step = s;
        c.step_dev = nullptr;
        return c;
    }

    void check_launch() {
        ++launches;
        CK(cudaGetLastError());
    }

    // ---- host-built initial states ----------------------------------------
    void upload_ref(const std::vector<double>& f, const std::vector<double>& g, const std::vector<double>& r,
                    const std::vector<double>& u, const std::vector<double>& v, const std::vector<double>& t) {
        const int nx = p.nx, ny = p.ny;
        std::vector<St> hp(NPLANES * field_elems(), Fmt<St>::store(A(0), 0, RN_BITS));
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix) {
                const size_t k = size_t(iy) * nx + ix, d = size_t(iy) * pitch + ix;
                for (int i = 0; i < Q; ++i) {
                    double fv = f[k * Q + i];
                    if (SH) fv -= WD(i);
                    hp[size_t(i) * field_elems() + d] = Fmt<St>::store(A(fv), i, RN_BITS);
                    hp[size_t(Q + i) * field_elems() + d] = Fmt<St>::store(A(g[k * Q + i]), Q + i, RN_BITS);
                }
            }
        cur = 0;
        pc_form = false;
        ref_cached = false;
        CK(cudaMemcpyAsync(pop[0], hp.data(), sizeof(St) * hp.size(), cudaMemcpyHostToDevice, stream));
        upload_field(rho, r.data());
        upload_field(ux, u.data());
        upload_field(uy, v.data());
        upload_field(tt, t.data());
        CK(cudaStreamSynchronize(stream));
    }

    void upload_field(A* dst, const double* src) {
        std::vector<A> h(field_elems(), A(0));
        for (int iy = 0; iy < p.ny; ++iy)
            for (int ix = 0; ix < p.nx; ++ix) h[size_t(iy) * pitch + ix] = A(src[size_t(iy) * p.nx + ix]);
        CK(cudaMemcpyAsync(dst, h.data(), sizeof(A) * h.size(), cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));
    }

    void download_field(const A* src, double* dst) {
        std::vector<A> h(field_elems());
        CK(cudaMemcpyAsync(h.data(), src, sizeof(A) * h.size(), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (int iy = 0; iy < p.ny; ++iy)
            for (int ix = 0; ix < p.nx; ++ix) dst[size_t(iy) * p.nx + ix] = double(h[size_t(iy) * pitch + ix]);
    }

    // CavitySolver::new initial state, src/uniform/solver.rs:159-176.
    void init_default(const std::vector<double>& t0) override {
        const size_t n = size_t(p.nx) * p.ny;
        std::vector<double> f(n * Q), g(n * Q), r(n, 1.0), u(n, 0.0), v(n, 0.0);
        for (size_t k = 0; k < n; ++k)
            for (int i = 0; i < Q; ++i) {
                f[k * Q + i] = feq_full<double>(i, 1.0, 0.0, 0.0);
                g[k * Q + i] = geq_full<double>(i, t0[k], 0.0, 0.0, p.geq_order);
            }
        upload_ref(f, g, r, u, v, t0);
        time_step = 0;
    }

    // init_from_fields, src/uniform/solver.rs:232-262.
    void init_from_fields(const double* r, const double* u, const double* v, const double* t) override {
        const int nx = p.nx, ny = p.ny;
        const size_t n = size_t(nx) * ny;
        std::vector<double> f(n * Q), g(n * Q), rr(r, r + n), uu(u, u + n), vv(v, v + n), tt0(t, t + n);
        for (size_t k = 0; k < n; ++k)
            for (int i = 0; i < Q; ++i) {
                f[k * Q + i] = feq_full<double>(i, r[k], u[k], v[k]);
                g[k * Q + i] = geq_full<double>(i, t[k], u[k], v[k], p.geq_order);
            }
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix)
                if (ix == 0 || ix == nx - 1 || iy == 0 || iy == ny - 1) {
                    uu[size_t(iy) * nx + ix] = 0.0;
                    vv[size_t(iy) * nx + ix] = 0.0;
                }
        upload_ref(f, g, rr, uu, vv, tt0);
        time_step = 0;
    }

    // ---- form transitions ------------------------------------------------------
    St* ref_pop() { return pc_form ? pop[cur ^ 1] : pop[cur]; }

    void ensure_ref() {
        if (!pc_form || ref_cached) return;
        k_materialize<St><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, rho, ux, uy, tt, G,
                                                     scalars(time_step));
        check_launch();
        ref_cached = true;
    }

    void to_ref_form() {
        ensure_ref();
        if (pc_form) {
            cur ^= 1;
            pc_form = false;
            ref_cached = false;
        }
    }

    // ---- the step loop -----------------------------------------------------------
    void launch_fused(int64_t s, bool write_nut, bool acc, const long long* sdev = nullptr, int64_t off = 0) {
        StepScalars<A> c = scalars(s);
        if (sdev) {
            c.step_dev = sdev;
            c.step = off;
        }
        if (write_nut) {
            if (acc)
                k_fused<St, true, true, false><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, nut, acc_hot,
                                                                         acc_cold, G, c);
            else
                k_fused<St, true, false, false><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, nut, acc_hot,
                                                                          acc_cold, G, c);
        } else {
            if (acc)
                k_fused<St, false, true, false><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, nut, acc_hot,
                                                                          acc_cold, G, c);
            else
                k_fused<St, false, false, false><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, nut, acc_hot,
                                                                           acc_cold, G, c);
        }
        check_launch();
        cur ^= 1;
    }

    // GRAPH_STEPS steady-state fused steps (all scalars equal) as one graph.
    cudaGraphExec_t get_graph(bool acc) {
        cudaGraphExec_t& gx = graph[cur][acc ? 1 : 0];
        if (gx) return gx;
        const int cur0 = cur;
        const int64_t launches0 = launches;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < GRAPH_STEPS; ++j) launch_fused(spin_up, false, acc, step_dev, j);
        k_add_step<<<1, 1, 0, stream>>>(step_dev, GRAPH_STEPS);
        cudaGraph_t gr;
        CK(cudaStreamEndCapture(stream, &gr));
        cur = cur0;
        launches = launches0;
        CK(cudaGraphInstantiate(&gx, gr, 0));
        cudaGraphDestroy(gr);
        return gx;
    }

    void step(int64_t n) override {
        if (n <= 0) return;
        bool first = true;
        const int64_t n_total = n;
        while (n > 0) {
            const bool last = (n == 1);
            if (!pc_form) {
                k_collide_ref<St><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], rho, ux, uy, tt, fy, nut, G,
                                                           scalars(time_step));
                check_launch();
                cur ^= 1;
                pc_form = true;
            } else if (!first && time_step >= spin_up && n > GRAPH_STEPS) {
                cudaGraphExec_t gx = get_graph(acc_on);
                if (step_dev_val != time_step) {
                    k_set_step<<<1, 1, 0, stream>>>(step_dev, time_step);
                    check_launch();
                    step_dev_val = time_step;
                }
                CK(cudaGraphLaunch(gx, stream));
                step_dev_val += GRAPH_STEPS;
                launches += GRAPH_STEPS + 1;
                time_step += GRAPH_STEPS;
                n -= GRAPH_STEPS;
                ref_cached = false;
                continue;
            } else {
                launch_fused(time_step, last, acc_on && !first);
            }
            first = false;
            ref_cached = false;
            time_step += 1;
            n -= 1;
        }
        if (acc_on) {
            k_acc_nu_pc<St><<<(p.ny + 127) / 128, 128, 0, stream>>>(pop[cur], acc_hot, acc_cold, G,
                                                                   scalars(time_step));
            check_launch();
            n_acc += n_total;
        }
    }

    // ---- observables --------------------------------------------------------------
    void get_fields(double* r, double* u, double* v, double* t, double* nu_t, double* fyo) override {
        ensure_ref();
        if (r) download_field(rho, r);
        if (u) download_field(ux, u);
        if (v) download_field(uy, v);
        if (t) download_field(tt, t);
        if (nu_t) download_field(nut, nu_t);
        if (fyo) download_field(fy, fyo);
    }

    void set_fields(const double* r, const double* u, const double* v, const double* t, const double* fyi) override {
        to_ref_form();
        if (r) upload_field(rho, r);
        if (u) upload_field(ux, u);
        if (v) upload_field(uy, v);
        if (t) upload_field(tt, t);
        if (fyi) upload_field(fy, fyi);
    }

    void ensure_aos() {
        if (!aos) CK(cudaMalloc(&aos, sizeof(double) * 2 * Q * size_t(p.nx) * p.ny));
    }

    void get_pops(double* f, double* g) override {
        ensure_ref();
        ensure_aos();
        const size_t n = size_t(p.nx) * p.ny * Q;
        k_pops_to_aos<St><<<grd, blk, 0, stream>>>(ref_pop(), aos, aos + n, G);
        check_launch();
        if (f) CK(cudaMemcpyAsync(f, aos, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
        if (g) CK(cudaMemcpyAsync(g, aos + n, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    void set_pops(const double* f, const double* g) override {
        to_ref_form();
        ensure_aos();
        const size_t n = size_t(p.nx) * p.ny * Q;
        if (f) CK(cudaMemcpyAsync(aos, f, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        if (g) CK(cudaMemcpyAsync(aos + n, g, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        k_aos_to_pops<St><<<grd, blk, 0, stream>>>(pop[cur], aos, aos + n, f ? 1 : 0, g ? 1 : 0, G);
        check_launch();
        CK(cudaStreamSynchronize(stream));
    }

    void diag(double* out) override {
        ensure_ref();
        const long long n = (long long)p.nx * p.ny;
        int nb = int(std::min<long long>((n + DIAG_THREADS - 1) / DIAG_THREADS, DIAG_BLOCKS_MAX));
        k_diag_partials<St><<<nb, DIAG_THREADS, 0, stream>>>(ref_pop(), rho, ux, uy, tt, nut, partials, G);
        check_launch();
        k_diag_final<A><<<1, DIAG_THREADS, 0, stream>>>(partials, nb, ux, uy, tt, nut, U.nu, U.lz, diag_out, G);
        check_launch();
        CK(cudaMemcpyAsync(out, diag_out, sizeof(double) * 11, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    void debug_phase(int phase, int64_t step_arg) override {
        to_ref_form();
        switch (phase) {
            case CAV_PHASE_COLLIDE:
                k_dbg_collide<St><<<grd, blk, 0, stream>>>(pop[cur], rho, ux, uy, tt, fy, nut, G, scalars(step_arg));
                break;
            case CAV_PHASE_STREAM:
                k_dbg_stream<St><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], G);
                cur ^= 1;
                break;
            case CAV_PHASE_BOUNCE_BACK:
                k_dbg_bounce_back<St><<<grd, blk, 0, stream>>>(pop[cur], G);
                break;
            case CAV_PHASE_THERMAL_BC:
                k_dbg_thermal_v<St><<<(p.ny + 127) / 128, 128, 0, stream>>>(pop[cur], G, scalars(time_step));
                check_launch();
                k_dbg_thermal_h<St><<<(p.nx + 127) / 128, 128, 0, stream>>>(pop[cur], G);
                break;
            case CAV_PHASE_MACRO:
                k_dbg_macro<St><<<grd, blk, 0, stream>>>(pop[cur], fy, rho, ux, uy, tt, G);
                break;
            case CAV_PHASE_NOSLIP:
                k_dbg_noslip<A><<<grd, blk, 0, stream>>>(ux, uy, G);
                break;
            case CAV_PHASE_FUSED_IDENTITY: {
                // With an identity collision the REF populations are also the
                // post-collision ones: stream them step_arg times with the
                // production kernel, then materialize once more.
                if (step_arg < 0) throw ArgError{CAV_ERR_ARG, "negative pass count"};
                pc_form = true;
                ref_cached = false;
                for (int64_t j = 0; j < step_arg; ++j) {
                    k_fused<St, false, false, true><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, nut,
                                                                            acc_hot, acc_cold, G,
                                                                            scalars(time_step));
                    check_launch();
                    cur ^= 1;
                }
                to_ref_form();
                break;
            }
            default:
                throw ArgError{CAV_ERR_ARG, "unknown debug phase"};
        }
        check_launch();
        CK(cudaStreamSynchronize(stream));
    }

    void sample() override {
        ensure_ref();
        const size_t n = size_t(p.nx) * p.ny;
        if (!sums) {
            CK(cudaMalloc(&sums, sizeof(double) * 5 * n));
            CK(cudaMemsetAsync(sums, 0, sizeof(double) * 5 * n, stream));
        }
        k_avg_accumulate<A><<<grd, blk, 0, stream>>>(ux, uy, tt, nut, sums, G);
        check_launch();
        n_samples += 1;
    }

    void reset_means() override {
        if (sums) CK(cudaMemsetAsync(sums, 0, sizeof(double) * 5 * size_t(p.nx) * p.ny, stream));
        n_samples = 0;
    }

    int64_t get_means(double* u, double* v, double* t, double* nu_t, double* uu) override {
        const size_t n = size_t(p.nx) * p.ny;
        double* outs[5] = {u, v, t, nu_t, uu};
        if (!sums || n_samples == 0) {
            for (double* o : outs)
                if (o) std::memset(o, 0, sizeof(double) * n);
            return n_samples;
        }
        std::vector<double> h(5 * n);
        CK(cudaMemcpyAsync(h.data(), sums, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        const double inv = 1.0 / double(n_samples);
        for (int j = 0; j < 5; ++j)
            if (outs[j])
                for (size_t k = 0; k < n; ++k) outs[j][k] = h[j * n + k] * inv;
        return n_samples;
    }

    void nu_accumulate(bool on) override {
        CK(cudaMemsetAsync(acc_hot, 0, sizeof(double) * p.ny, stream));
        CK(cudaMemsetAsync(acc_cold, 0, sizeof(double) * p.ny, stream));
        n_acc = 0;
        acc_on = on;
    }

    void nu_accumulated(double* hot, double* cold, int64_t* n) override {
        std::vector<double> h(p.ny), c(p.ny);
        CK(cudaMemcpyAsync(h.data(), acc_hot, sizeof(double) * p.ny, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(c.data(), acc_cold, sizeof(double) * p.ny, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        double sh = 0.0, sc = 0.0;
        for (int i = 0; i < p.ny; ++i) {
            sh += h[i];
            sc += c[i];
        }
        const double denom = double(p.ny) * double(n_acc > 0 ? n_acc : 1);
        if (hot) *hot = sh / denom * U.lz;
        if (cold) *cold = sc / denom * U.lz;
        if (n) *n = n_acc;
    }

    void sync() override { CK(cudaStreamSynchronize(stream)); }
};

Solver* make_solver(int precision);

}  // namespace cav
