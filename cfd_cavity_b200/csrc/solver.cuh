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
#include <array>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cavity.h"
#include "adjoint.cuh"
#include "errors.cuh"
#include "diag.cuh"
#include "kernels.cuh"
#include "sgs.cuh"
#include "xpair.cuh"

namespace cav {

constexpr int GRAPH_STEPS = 64;  // even: a replay leaves the buffer parity unchanged
constexpr int BX = 32, BY = 2;
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
    // init_from_fields from DEVICE arrays (dense, k = iy*nx + ix).
    virtual void init_from_device_fields(const double* r, const double* u, const double* v, const double* t) = 0;
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
    // Forward n_steps with checkpoints every ck_every steps, then the adjoint
    // sweep; see Impl::adjoint_run.  out[0] = J, out[1] = dJ/dCs,
    // out[2] = forward ms, out[3] = reverse ms, out[4] = checkpoints.
    virtual void adjoint_run(int64_t n_steps, int64_t ws, int ck_every, double* grad_theta, double* out) = 0;
    // set_dynamic_sgs (src/uniform/solver.rs:215-220) and the model's
    // coefficient statistics (cs_dyn_mean, cs_dyn_max, kappa_dyn_mean,
    // kappa_dyn_max) of the last step.
    // Kernel of the fused step: 0 one node per thread (k_fused), 1 two
    // x-adjacent nodes per thread (k_fused_x, 16-bit formats).  Both give
    // the same bits.
    virtual void set_step_kernel(int k) = 0;
    virtual int step_kernel() const = 0;
    virtual void set_dynamic_sgs(bool on, double smag_alpha, double nu_sm_min, double eta_test) = 0;
    virtual void dynamic_stats(double* out4) = 0;
    bool dyn = false;

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
    // Block height: 32 x 4 for FP32 storage, 32 x 2 otherwise.  Measured on a
    // B200 with graph-replayed programmatic-launch steps (the next step's
    // CTAs are placed while the current step's are still resident, so the
    // balance over SMs depends on the CTA count): FP32 128x512 2.24 us / step
    // with 32 x 4 against 3.06 with 32 x 2; f16sr 2.47 with 32 x 2 against
    // 2.51 with 32 x 4.
    static constexpr int BYF = std::is_same<St, float>::value ? 4 : BY;
    dim3 blk{BX, BYF}, grd{};
    // the node-pair kernel: 32 x BYX threads cover 64 columns x BYX rows
    static constexpr int BYX = 2;
    dim3 blkx{BX, BYX}, grdx{};
    // the 16-bit formats' default step kernel: pairs split over two warps
    // for cavities that cannot fill the GPU (a step is then one thread's
    // latency chain; on a B200 128 x 512 f16sr 2.32 us against 2.42, 64 x 256
    // 1.67 against 2.00), plain pairs above (512 x 2048: 16.3 against 23.8)
    static constexpr long long SPLIT_MAX_NODES = 70000;
    int kern = is_p16<St>::value ? 1 : 0;
    // dynamic subgrid model
    double dyn_alpha = 0.5, dyn_min = -0.1, dyn_eta = 2.0;
    double* sgs_w = nullptr;       // S_NPLANES FP64 work planes
    A *nut_pre = nullptr, *at_pre = nullptr;
    double* sgs_out = nullptr;     // 4 statistics
    bool sgs_valid = false;        // the work planes hold the last step's coefficients

    ~Impl() override {
        for (auto& row : graph)
            for (auto& gx : row)
                if (gx) cudaGraphExecDestroy(gx);
        void* bufs[] = {pop[0], pop[1], rho, ux, uy, tt, fy, nut, t_hot_d, acc_hot, acc_cold,
                        partials, diag_out, sums, aos, step_dev, sgs_w, nut_pre, at_pre, sgs_out};
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
        grd = dim3((p.nx + BX - 1) / BX, (p.ny + BYF - 1) / BYF);
        grdx = dim3(((p.nx + 1) / 2 + BX - 1) / BX, (p.ny + BYX - 1) / BYX);
        if (is_p16<St>::value && (long long)p.nx * p.ny <= SPLIT_MAX_NODES) kern = 2;
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

    // Launch with programmatic dependent launch (the kernel begins with
    // pdl_wait(), so it overlaps only the tail of its predecessor).
    template <typename... KArgs, typename... Args>
    void launch_pdl(void (*kern)(KArgs...), cudaStream_t st, Args... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grd;
        cfg.blockDim = blk;
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, kern, args...));
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
    void init_from_device_fields(const double* r, const double* u, const double* v, const double* t) override {
        k_init_eq<St><<<grd, blk, 0, stream>>>(r, u, v, t, pop[0], rho, ux, uy, tt, G, p.geq_order);
        check_launch();
        cur = 0;
        pc_form = false;
        ref_cached = false;
        time_step = 0;
        CK(cudaStreamSynchronize(stream));
    }

    // init_from_fields (src/uniform/solver.rs:232-262) from host arrays: the
    // fields go to the device and the equilibria are set there (k_init_eq,
    // the host's FP64 arithmetic bit for bit).
    void init_from_fields(const double* r, const double* u, const double* v, const double* t) override {
        ensure_aos();
        const size_t n = size_t(p.nx) * p.ny;
        const double* src[4] = {r, u, v, t};
        for (int j = 0; j < 4; ++j)
            CK(cudaMemcpyAsync(aos + j * n, src[j], sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        init_from_device_fields(aos, aos + n, aos + 2 * n, aos + 3 * n);
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
    // k_fused with programmatic dependent launch: successive fused steps
    // overlap the next launch with the tail of the previous one.
    template <bool WN, bool ACC>
    void launch_fused_pdl(const StepScalars<A>& c) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grd;
        cfg.blockDim = blk;
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if constexpr (is_p16<St>::value) {
            if (kern == 1) {
                cfg.gridDim = grdx;
                cfg.blockDim = blkx;
                CK(cudaLaunchKernelEx(&cfg, k_fused_x<St, WN, ACC, false>, (const St*)pop[cur], pop[cur ^ 1], fy,
                                      nut, acc_hot, acc_cold, G, c));
                return;
            }
            if (kern == 2) {
                cfg.gridDim = dim3(((p.nx + 1) / 2 + 31) / 32, (p.ny + 1) / 2);
                cfg.blockDim = dim3(128);
                CK(cudaLaunchKernelEx(&cfg, k_fused_xs<St, WN, ACC>, (const St*)pop[cur], pop[cur ^ 1], fy, nut,
                                      acc_hot, acc_cold, G, c));
                return;
            }
        }
        CK(cudaLaunchKernelEx(&cfg, k_fused<St, WN, ACC, false>, (const St*)pop[cur], pop[cur ^ 1], fy, nut,
                              acc_hot, acc_cold, G, c));
    }

    void set_step_kernel(int k) override {
        if (k < 0 || k > 2) throw ArgError{CAV_ERR_ARG, "step kernel must be 0, 1 or 2"};
        if (k >= 1 && !is_p16<St>::value)
            throw ArgError{CAV_ERR_ARG, "the node-pair step kernel is for the 16-bit storage formats"};
        CK(cudaStreamSynchronize(stream));
        kern = k;
        for (auto& row : graph)
            for (auto& gx : row)
                if (gx) {
                    CK(cudaGraphExecDestroy(gx));
                    gx = nullptr;
                }
    }
    int step_kernel() const override { return kern; }

    void launch_fused(int64_t s, bool write_nut, bool acc, const long long* sdev = nullptr, int64_t off = 0) {
        StepScalars<A> c = scalars(s);
        if (sdev) {
            c.step_dev = sdev;
            c.step = off;
        }
        if (write_nut) {
            if (acc)
                launch_fused_pdl<true, true>(c);
            else
                launch_fused_pdl<true, false>(c);
        } else {
            if (acc)
                launch_fused_pdl<false, true>(c);
            else
                launch_fused_pdl<false, false>(c);
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

    void set_dynamic_sgs(bool on, double smag_alpha, double nu_sm_min, double eta_test) override {
        if (!(smag_alpha >= 0.0 && smag_alpha <= 1.0) || !(eta_test >= 1.0) || !std::isfinite(nu_sm_min))
            throw ArgError{CAV_ERR_ARG, "dynamic SGS: smag_alpha in [0, 1], eta_test >= 1, finite nu_sm_min"};
        dyn = on;
        dyn_alpha = smag_alpha;
        dyn_min = nu_sm_min;
        dyn_eta = eta_test;
        if (on && !sgs_w) {
            CK(cudaMalloc(&sgs_w, sizeof(double) * S_NPLANES * field_elems()));
            CK(cudaMemsetAsync(sgs_w, 0, sizeof(double) * S_NPLANES * field_elems(), stream));
            CK(cudaMalloc(&nut_pre, sizeof(A) * field_elems()));
            CK(cudaMalloc(&at_pre, sizeof(A) * field_elems()));
            CK(cudaMalloc(&sgs_out, sizeof(double) * 4));
        }
        sgs_valid = false;
    }

    void dynamic_stats(double* out4) override {
        if (!sgs_valid) {
            for (int i = 0; i < 4; ++i) out4[i] = 0.0;
            return;
        }
        k_sgs_stats<<<1, 256, 0, stream>>>(sgs_w, G, sgs_out);
        check_launch();
        CK(cudaMemcpyAsync(out4, sgs_out, sizeof(double) * 4, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    // One step with the dynamic model, in the reference's order
    // (src/uniform/solver.rs:279-291): compute_dynamic_sgs on the REF state,
    // collide with the per-node nu_t / alpha_t, then stream + BC + macro +
    // no-slip back to a REF state.
    void dyn_step() {
        to_ref_form();
        double nu_eff = U.nu;
        if (time_step < spin_up) {
            const double x = double(time_step) / double(spin_up);
            const double nu_start = U.nu * nu_start_mult;
            nu_eff = nu_start * std::pow(U.nu / nu_start, x);
        }
        SgsParams sp;
        const double eta = std::max(dyn_eta, 1.0);
        sp.width = std::max((int)std::llround(eta), 1);
        sp.dtest = eta * 1.0;
        sp.alpha_exp = dyn_alpha;
        sp.tau_s = 0.5 + 3.0 * std::fmax(nu_eff, 0.002 / 3.0);
        sp.nu_mol = U.nu;
        sp.alpha_mol = U.alpha;
        sp.nu_sm_min = dyn_min;
        SgsGrids<St> S{};
        S.g[0] = SgsGrid<St>{pop[cur], rho, ux, uy, tt, sgs_w, nut_pre, at_pre};
        k_sgs_b<St><<<grd, blk, 0, stream>>>(S, G, sp);
        check_launch();
        k_sgs_c<St><<<grd, blk, 0, stream>>>(S, G, sp);
        check_launch();
        k_sgs_d<St><<<grd, blk, 0, stream>>>(S, G, sp);
        check_launch();
        sgs_valid = true;
        k_collide_ref<St><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], rho, ux, uy, tt, fy, nut, G,
                                                   scalars(time_step), nut_pre, at_pre);
        check_launch();
        cur ^= 1;
        pc_form = true;
        ref_cached = false;
        to_ref_form();
        time_step += 1;
        if (acc_on) {
            k_acc_nu_ref<A><<<(p.ny + 127) / 128, 128, 0, stream>>>(tt, acc_hot, acc_cold, G);
            check_launch();
            n_acc += 1;
        }
    }

    void step(int64_t n) override {
        if (n <= 0) return;
        if (dyn) {
            for (int64_t j = 0; j < n; ++j) dyn_step();
            return;
        }
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
    // The fields, converted to dense FP64 on the device and copied straight
    // into the caller's arrays (one synchronisation).
    void get_fields(double* r, double* u, double* v, double* t, double* nu_t, double* fyo) override {
        ensure_ref();
        ensure_aos();
        const size_t n = size_t(p.nx) * p.ny;
        const A* src[6] = {rho, ux, uy, tt, nut, fy};
        double* dst[6] = {r, u, v, t, nu_t, fyo};
        for (int j = 0; j < 6; ++j) {
            if (!dst[j]) continue;
            k_field_to_dense<A><<<grd, blk, 0, stream>>>(src[j], aos + j * n, G);
            check_launch();
            CK(cudaMemcpyAsync(dst[j], aos + j * n, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
        }
        CK(cudaStreamSynchronize(stream));
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
                    bool done = false;
                    if constexpr (is_p16<St>::value) {
                        if (kern >= 1) {
                            k_fused_x<St, false, false, true><<<grdx, blkx, 0, stream>>>(
                                pop[cur], pop[cur ^ 1], fy, nut, acc_hot, acc_cold, G, scalars(time_step));
                            done = true;
                        }
                    }
                    if (!done)
                        k_fused<St, false, false, true><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, nut,
                                                                                acc_hot, acc_cold, G,
                                                                                scalars(time_step));
                    check_launch();
                    cur ^= 1;
                }
                to_ref_form();
                break;
            }
            case CAV_PHASE_CHANNEL: {
                // step_arg steps of the fused kernel's plane-channel variant
                // (k_fused CHANNEL), the first from the REF state by
                // collide(step), then back to a REF state by the channel pull
                if (step_arg < 1) throw ArgError{CAV_ERR_ARG, "the channel needs at least one step"};
                int64_t n = step_arg;
                if (!pc_form) {
                    k_collide_ref<St><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], rho, ux, uy, tt, fy, nut, G,
                                                               scalars(time_step));
                    check_launch();
                    cur ^= 1;
                    pc_form = true;
                    time_step += 1;
                    n -= 1;
                }
                ref_cached = false;
                for (int64_t j = 0; j < n; ++j) {
                    k_fused<St, false, false, false, true><<<grd, blk, 0, stream>>>(
                        pop[cur], pop[cur ^ 1], fy, nut, acc_hot, acc_cold, G, scalars(time_step));
                    check_launch();
                    cur ^= 1;
                    time_step += 1;
                }
                k_materialize<St, true><<<grd, blk, 0, stream>>>(pop[cur], pop[cur ^ 1], fy, rho, ux, uy, tt, G,
                                                                 scalars(time_step));
                check_launch();
                cur ^= 1;
                pc_form = false;
                ref_cached = false;
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


    // ---- adjoint ---------------------------------------------------------------
    // J = mean over s in [ws, N] of nusselt_hot(state after s steps).
    // Forward: the production step (graphs included), storing the PC state
    // every ck_every steps (X_1, X_{1+C}, ...).  Reverse: for each segment,
    // last first, recompute its states from the checkpoint with k_fwd_slot,
    // then run k_adj_step backwards through them.  Needs FP32 or FP64 storage
    // and a fresh state (step 0, as after create or init_from_fields).
    void adjoint_run(int64_t N, int64_t ws, int C, double* gth, double* out) override {
        if constexpr (!(std::is_same<St, float>::value || std::is_same<St, double>::value)) {
            throw ArgError{CAV_ERR_ARG, "the adjoint needs FP32 or FP64 storage"};
        } else {
            if (dyn) throw ArgError{CAV_ERR_STATE, "the adjoint needs the fixed-Cs model (dynamic SGS is on)"};
            if (pc_form || time_step != 0)
                throw ArgError{CAV_ERR_STATE, "adjoint_run starts from step 0 (after create or init_from_fields)"};
            if (N < 2 || ws < 1 || ws > N || C < 2) throw ArgError{CAV_ERR_ARG, "bad adjoint spec"};
            const size_t fld = field_elems(), popn = size_t(NPLANES) * fld;
            const int64_t n_ck = (N - 1 + C - 1) / C;
            St *ck_pop = nullptr, *seg_pop = nullptr;
            A *ck_fy = nullptr, *seg_fy = nullptr, *P[2] = {nullptr, nullptr};
            double *acc_cs_d = nullptr, *acc_th_d = nullptr;
            cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
            struct Free {
                std::vector<void*> v;
                ~Free() {
                    for (void* q : v)
                        if (q) cudaFree(q);
                }
            } fr;
            auto dalloc = [&](void** p2, size_t bytes) {
                CK(cudaMalloc(p2, bytes));
                fr.v.push_back(*p2);
            };
            dalloc((void**)&ck_pop, sizeof(St) * popn * n_ck);
            dalloc((void**)&ck_fy, sizeof(A) * fld * n_ck);
            St* seg_pop2 = nullptr;
            A* seg_fy2 = nullptr;
            dalloc((void**)&seg_pop, sizeof(St) * popn * C);
            dalloc((void**)&seg_fy, sizeof(A) * fld * C);
            dalloc((void**)&seg_pop2, sizeof(St) * popn * C);
            dalloc((void**)&seg_fy2, sizeof(A) * fld * C);
            long long* sdev2 = nullptr;
            dalloc((void**)&sdev2, 2 * sizeof(long long));
            for (auto& pp : P) dalloc((void**)&pp, sizeof(A) * APLANES * fld);
            dalloc((void**)&acc_cs_d, sizeof(double) * size_t(p.nx) * p.ny);
            dalloc((void**)&acc_th_d, sizeof(double) * p.ny);
            CK(cudaMemsetAsync(acc_cs_d, 0, sizeof(double) * size_t(p.nx) * p.ny, stream));
            CK(cudaMemsetAsync(acc_th_d, 0, sizeof(double) * p.ny, stream));
            for (auto& e : ev) CK(cudaEventCreate(&e));
            struct Ev {
                cudaEvent_t* e;
                ~Ev() {
                    for (int i = 0; i < 3; ++i)
                        if (e[i]) cudaEventDestroy(e[i]);
                }
            } evg{ev};
            auto save_ck = [&](int64_t k) {
                CK(cudaMemcpyAsync(ck_pop + popn * k, pop[cur], sizeof(St) * popn, cudaMemcpyDeviceToDevice, stream));
                CK(cudaMemcpyAsync(ck_fy + fld * k, fy, sizeof(A) * fld, cudaMemcpyDeviceToDevice, stream));
            };
            // ---- reverse-sweep setup (before any timing) ----
            // Per-step scalars as a device table (rows 0..spin_up) so that the
            // segment sweeps can be captured once as CUDA graphs and replayed
            // with the device step counter.
            const int S = int(spin_up);
            StepScalars<A>* table = nullptr;
            {
                std::vector<StepScalars<A>> tab(S + 1);
                for (int r2 = 0; r2 <= S; ++r2) tab[r2] = scalars(r2);
                dalloc((void**)&table, sizeof(StepScalars<A>) * tab.size());
                CK(cudaMemcpyAsync(table, tab.data(), sizeof(StepScalars<A>) * tab.size(), cudaMemcpyHostToDevice,
                                   stream));
                CK(cudaStreamSynchronize(stream));
            }
            AdjObj<A> obj;
            obj.ws = ws;
            obj.coef = A(U.lz / (double(p.ny) * double(N - ws + 1)));
            // Segments are processed last first.  The recomputation of
            // segment k-1 (stream rs, slot set (k-1) & 1) overlaps the
            // adjoint sweep of segment k (the solver's stream, set k & 1):
            // both are latency-bound on one cavity, so the GPU runs them side
            // by side.  Events order the reuse of a slot set.  Each stream has
            // its own device step counter; full segments (length C, even) are
            // CUDA graphs, one pair per slot set.
            St* setp[2] = {seg_pop, seg_pop2};
            A* setf[2] = {seg_fy, seg_fy2};
            long long* sd_rec = sdev2;
            long long* sd_adj = sdev2 + 1;
            cudaStream_t rs = nullptr, hs = nullptr;
            CK(cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking));
            // the adjoint sweep is the critical path: it runs on a stream of
            // the highest priority, the recomputation fills the rest of the GPU
            {
                int least = 0, greatest = 0;
                CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
                CK(cudaStreamCreateWithPriority(&hs, cudaStreamNonBlocking, greatest));
            }
            struct StreamGuard {
                cudaStream_t* s;
                ~StreamGuard() {
                    if (*s) {
                        cudaStreamSynchronize(*s);
                        cudaStreamDestroy(*s);
                    }
                }
            } hs_guard{&hs};
            std::vector<cudaEvent_t> ev_rec(n_ck, nullptr), ev_adj(n_ck, nullptr);
            cudaGraphExec_t g_rec[2] = {nullptr, nullptr}, g_adj[2] = {nullptr, nullptr};
            struct Cleanup {
                cudaStream_t* s;
                std::vector<cudaEvent_t>* a;
                std::vector<cudaEvent_t>* b;
                cudaGraphExec_t* g1;
                cudaGraphExec_t* g2;
                ~Cleanup() {
                    if (*s) {
                        cudaStreamSynchronize(*s);
                        cudaStreamDestroy(*s);
                    }
                    for (auto* v2 : {a, b})
                        for (cudaEvent_t e : *v2)
                            if (e) cudaEventDestroy(e);
                    for (int i = 0; i < 2; ++i) {
                        if (g1[i]) cudaGraphExecDestroy(g1[i]);
                        if (g2[i]) cudaGraphExecDestroy(g2[i]);
                    }
                }
            } cleanup{&rs, &ev_rec, &ev_adj, g_rec, g_adj};
            for (int64_t k = 0; k < n_ck; ++k) {
                CK(cudaEventCreateWithFlags(&ev_rec[k], cudaEventDisableTiming));
                CK(cudaEventCreateWithFlags(&ev_adj[k], cudaEventDisableTiming));
            }
            const bool use_graphs = (C % 2) == 0;
            auto capture = [&](cudaStream_t st, cudaGraphExec_t* out, auto&& body) {
                const int64_t l0 = launches;
                CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                body();
                cudaGraph_t gr;
                CK(cudaStreamEndCapture(st, &gr));
                launches = l0;
                CK(cudaGraphInstantiate(out, gr, 0));
                cudaGraphDestroy(gr);
            };
            auto seg_len = [&](int64_t k) { return std::min<int64_t>(1 + k * C + C, N) - (1 + k * C); };
            // recomputation of segment k on rs
            auto recompute = [&](int64_t k) {
                const int set = int(k & 1);
                const int64_t a = 1 + k * C, L = seg_len(k);
                St* sp = setp[set];
                A* sf = setf[set];
                if (k + 2 < n_ck) CK(cudaStreamWaitEvent(rs, ev_adj[k + 2], 0));  // set free again
                CK(cudaMemcpyAsync(sp, ck_pop + popn * k, sizeof(St) * popn, cudaMemcpyDeviceToDevice, rs));
                CK(cudaMemcpyAsync(sf, ck_fy + fld * k, sizeof(A) * fld, cudaMemcpyDeviceToDevice, rs));
                if (use_graphs && L == C) {
                    if (!g_rec[set])
                        capture(rs, &g_rec[set], [&] {
                            for (int64_t j = 0; j + 1 < C; ++j)
                                launch_pdl(k_fwd_slot<St>, rs, (const St*)sp + popn * j, sp + popn * (j + 1), sf + fld * j,
                                                                    sf + fld * (j + 1), G, table, S, sd_rec, j);
                        });
                    k_set_step<<<1, 1, 0, rs>>>(sd_rec, a);
                    check_launch();
                    CK(cudaGraphLaunch(g_rec[set], rs));
                    launches += C - 1;
                } else {
                    for (int64_t j = 0; j + 1 < L; ++j) {
                        launch_pdl(k_fwd_slot<St>, rs, (const St*)sp + popn * j, sp + popn * (j + 1), sf + fld * j,
                                                            sf + fld * (j + 1), G, table, S, nullptr, a + j);
                        check_launch();
                    }
                }
                CK(cudaEventRecord(ev_rec[k], rs));
            };
            int cp = 0;
            // adjoint sweep of segment k on the solver's stream
            auto sweep = [&](int64_t k) {
                const int set = int(k & 1);
                const int64_t a = 1 + k * C, L = seg_len(k);
                St* sp = setp[set];
                A* sf = setf[set];
                CK(cudaStreamWaitEvent(hs, ev_rec[k], 0));
                if (use_graphs && L == C) {
                    if (cp != 0) throw ArgError{CAV_ERR_STATE, "adjoint ping-pong out of phase"};
                    if (!g_adj[set])
                        capture(stream, &g_adj[set], [&] {
                            int q = 0;
                            for (int64_t j = C - 1; j >= 0; --j) {
                                launch_pdl(k_adj_step<St>, stream, (const St*)sp + popn * j, sf + fld * j, P[q], P[q ^ 1],
                                                                        acc_cs_d, acc_th_d, G, table, S, sd_adj, j,
                                                                        obj, j > 0 ? (const St*)sp + popn * (j - 1) : nullptr,
                                                                        j > 0 ? (const A*)sf + fld * (j - 1) : nullptr);
                                q ^= 1;
                            }
                        });
                    k_set_step<<<1, 1, 0, hs>>>(sd_adj, a);
                    check_launch();
                    CK(cudaGraphLaunch(g_adj[set], hs));
                    launches += C;
                } else {
                    for (int64_t j = L - 1; j >= 0; --j) {
                        launch_pdl(k_adj_step<St>, hs, (const St*)sp + popn * j, sf + fld * j, P[cp], P[cp ^ 1],
                                                                acc_cs_d, acc_th_d, G, table, S, nullptr, a + j, obj,
                                                                j > 0 ? (const St*)sp + popn * (j - 1) : nullptr,
                                                                j > 0 ? (const A*)sf + fld * (j - 1) : nullptr);
                        check_launch();
                        cp ^= 1;
                    }
                }
                CK(cudaEventRecord(ev_adj[k], hs));
            };
            // Build the segment graphs now, outside the timed passes (they only
            // depend on the buffers, not on the state).
            if (use_graphs && N - 1 >= C) {
                const int64_t l0 = launches;
                for (int set = 0; set < 2; ++set) {
                    St* sp = setp[set];
                    A* sf = setf[set];
                    capture(rs, &g_rec[set], [&] {
                        for (int64_t j = 0; j + 1 < C; ++j)
                            launch_pdl(k_fwd_slot<St>, rs, (const St*)sp + popn * j, sp + popn * (j + 1), sf + fld * j,
                                                                sf + fld * (j + 1), G, table, S, sd_rec, j);
                    });
                    capture(stream, &g_adj[set], [&] {
                        int q = 0;
                        for (int64_t j = C - 1; j >= 0; --j) {
                            launch_pdl(k_adj_step<St>, stream, (const St*)sp + popn * j, sf + fld * j, P[q], P[q ^ 1],
                                                                    acc_cs_d, acc_th_d, G, table, S, sd_adj, j, obj,
                                                                    j > 0 ? (const St*)sp + popn * (j - 1) : nullptr,
                                                                    j > 0 ? (const A*)sf + fld * (j - 1) : nullptr);
                            q ^= 1;
                        }
                    });
                    CK(cudaGraphUpload(g_rec[set], rs));
                    CK(cudaGraphUpload(g_adj[set], stream));
                }
                launches = l0;
                CK(cudaStreamSynchronize(rs));
                CK(cudaStreamSynchronize(stream));
            }
            // ---- forward ----
            CK(cudaEventRecord(ev[0], stream));
            nu_accumulate(false);
            if (ws == 1) nu_accumulate(true);
            step(1);  // X_1
            save_ck(0);
            int64_t next_ck = 1;
            while (time_step < N) {
                if (!acc_on && time_step == ws - 1) nu_accumulate(true);
                int64_t stop = N;
                if (next_ck < n_ck) stop = std::min<int64_t>(stop, 1 + next_ck * C);
                if (!acc_on && ws - 1 > time_step) stop = std::min<int64_t>(stop, ws - 1);
                step(stop - time_step);
                if (next_ck < n_ck && time_step == 1 + next_ck * C) save_ck(next_ck++);
            }
            double J = 0.0, jc = 0.0;
            int64_t nacc = 0;
            nu_accumulated(&J, &jc, &nacc);
            nu_accumulate(false);
            CK(cudaEventRecord(ev[1], stream));
            // ---- reverse ----
            // The P ping-pong must sit in P[0] when the first full-segment
            // graph runs: start in P[1] when the (processed first) partial
            // last segment has an odd length.
            {
                const int64_t L_last = seg_len(n_ck - 1);
                cp = (use_graphs && L_last != C && (L_last & 1)) ? 1 : 0;
            }
            CK(cudaStreamWaitEvent(hs, ev[1], 0));
            k_adj_final<St><<<grd, blk, 0, hs>>>(pop[cur], P[cp], G, scalars(N), obj, N);
            check_launch();
            CK(cudaStreamWaitEvent(rs, ev[1], 0));  // checkpoints complete
            recompute(n_ck - 1);
            for (int64_t k = n_ck - 1; k >= 0; --k) {
                if (k >= 1) recompute(k - 1);
                sweep(k);
            }
            CK(cudaEventRecord(ev[2], hs));
            CK(cudaStreamWaitEvent(stream, ev[2], 0));
            CK(cudaStreamSynchronize(hs));
            CK(cudaStreamDestroy(hs));
            hs = nullptr;
            std::vector<double> acs(size_t(p.nx) * p.ny), ath(p.ny);
            CK(cudaMemcpyAsync(acs.data(), acc_cs_d, sizeof(double) * acs.size(), cudaMemcpyDeviceToHost, stream));
            CK(cudaMemcpyAsync(ath.data(), acc_th_d, sizeof(double) * ath.size(), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            double gcs = 0.0;
            for (double v2 : acs) gcs += v2;
            // wall rows 0 and ny-1 take theta of rows 1 and ny-2 (solver.rs:974-987)
            for (int i = 0; i < p.ny; ++i) gth[i] = 0.0;
            for (int i = 0; i < p.ny; ++i) {
                const int gy = i == 0 ? 1 : (i == p.ny - 1 ? p.ny - 2 : i);
                gth[gy] += ath[i];
            }
            float ms_f = 0.f, ms_r = 0.f;
            CK(cudaEventElapsedTime(&ms_f, ev[0], ev[1]));
            CK(cudaEventElapsedTime(&ms_r, ev[1], ev[2]));
            out[0] = J;
            out[1] = gcs;
            out[2] = ms_f;
            out[3] = ms_r;
            out[4] = double(n_ck);
        }
    }

    void sync() override { CK(cudaStreamSynchronize(stream)); }
};

Solver* make_solver(int precision);

}  // namespace cav
