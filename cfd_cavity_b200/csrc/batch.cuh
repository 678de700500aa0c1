// batch.cuh -- many cavities of uneven size and Rayleigh number advanced by
// one launch per lattice step.
//
// Each cavity is an ordinary Impl<St> (own buffers, REF/PC state machine,
// diagnostics); the batch only replaces their per-cavity fused launches by
// one persistent-grid kernel over a work list of (cavity, 32-column x
// `rows`-row) tiles: grid = ctas_per_sm x #SMs CTAs of 128 threads that
// stride over the list.  Tiles are ordered cavity-major, row-block-minor, so
// the tiles in flight at one time are neighbours and the halo rows they
// share are served by L2.  Per-cavity step scalars (ramps, seeds, wall
// temperature pointers) come from a device table precomputed on the host with
// the single-cavity code (Impl::scalars), row min(step, spin_up), and every
// node runs the same fused_node() as k_fused: a cavity advanced in a batch
// is bit-identical to the same cavity advanced alone.  Steps run as CUDA
// graphs of GRAPH_STEPS launches reading a device step counter.
#pragma once

#include "solver.cuh"
#include "tile.cuh"
#include "tilex.cuh"
#include "xpair.cuh"

namespace cav {

template <class St>
struct BatchCav {
    St* pop[2];
    typename Fmt<St>::A* fy;
    typename Fmt<St>::A* nut;
    Geom G;
    int parity;   // buffer holding the state at batch step s: pop[(parity + s) & 1]
    int spin_up;  // scalar-table row of the steady state
};

struct BatchItem {
    int cav, tx0, ty0, rows;
};

constexpr int BATCH_THREADS = 128;

template <class St, bool WRITE_NUT>
__global__ void __launch_bounds__(BATCH_THREADS)
    k_batch(const BatchCav<St>* __restrict__ cavs, const BatchItem* __restrict__ items, int n_items,
            const StepScalars<typename Fmt<St>::A>* __restrict__ table, int n_cav, long long step,
            const long long* __restrict__ step_dev) {
    using A = typename Fmt<St>::A;
    const long long s = step_dev ? *step_dev + step : step;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchItem item = items[it];
        const BatchCav<St> cv = cavs[item.cav];
        const Geom G = cv.G;
        const int row = s < cv.spin_up ? int(s) : cv.spin_up;
        StepScalars<A> c = table[(long long)row * n_cav + item.cav];
        c.step = s;
        c.step_dev = nullptr;
        const int cur = (cv.parity + int(s & 1)) & 1;
        const St* src = cv.pop[cur];
        St* dst = cv.pop[cur ^ 1];
        const int ix = item.tx0 + lane;
        if (ix < G.nx) {
            for (int r = w; r < item.rows; r += BATCH_THREADS / 32)
                fused_node<St, WRITE_NUT, false, false>(src, dst, cv.fy, cv.nut, nullptr, nullptr, G, ix,
                                                        item.ty0 + r, c);
        }
    }
}

// The same node body with one CTA per (cavity, 32-column x rows) item, one
// node per thread (no persistent loop): the per-cavity pointers and scalars
// are not kept live across items, so the kernel needs the registers of
// k_fused, not of k_batch; capped at 56 (with 128-thread CTAs, 9 resident
// per SM; a word or three spilled to L1; on a B200 +3 % binary16, +15 %
// bfloat16 with stochastic rounding against 64 registers and 8 CTAs).
template <class St, bool WRITE_NUT>
__global__ void __maxnreg__(56)
    k_batch_np(const BatchCav<St>* __restrict__ cavs, const BatchItem* __restrict__ items,
               const StepScalars<typename Fmt<St>::A>* __restrict__ table, int n_cav, long long step,
               const long long* __restrict__ step_dev) {
    using A = typename Fmt<St>::A;
    pdl_wait();
    pdl_trigger();
    const long long s = step_dev ? *step_dev + step : step;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const BatchItem item = items[blockIdx.x];
    const BatchCav<St>& cv = cavs[item.cav];
    const int row = s < cv.spin_up ? int(s) : cv.spin_up;
    StepScalars<A> c = table[(long long)row * n_cav + item.cav];
    c.step = s;
    c.step_dev = nullptr;
    const int cur = (cv.parity + int(s & 1)) & 1;
    const int ix = item.tx0 + lane;
    if (ix < cv.G.nx && w < item.rows)
        fused_node<St, WRITE_NUT, false, false>(cv.pop[cur], cv.pop[cur ^ 1], cv.fy, cv.nut, nullptr, nullptr, cv.G,
                                                ix, item.ty0 + w, c);
}

// k_batch_np with two rows per thread (fused_pair: the arithmetic of both
// nodes on packed FP32x2 lanes): rows / 2 warps per item.  FP32-arithmetic
// formats only.  Register budget 96 (10 resident 64-thread CTAs per SM, a
// few words spilled to L1): more warps to hide the loads' latency beat the
// spill traffic on a B200.
template <class St, bool WRITE_NUT>
__global__ void __maxnreg__(96)
    k_batch_np2(const BatchCav<St>* __restrict__ cavs, const BatchItem* __restrict__ items,
                const StepScalars<float>* __restrict__ table, int n_cav, long long step,
                const long long* __restrict__ step_dev) {
    pdl_wait();
    pdl_trigger();
    const long long s = step_dev ? *step_dev + step : step;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const BatchItem item = items[blockIdx.x];
    const BatchCav<St>& cv = cavs[item.cav];
    const int row = s < cv.spin_up ? int(s) : cv.spin_up;
    StepScalars<float> c = table[(long long)row * n_cav + item.cav];
    c.step = s;
    c.step_dev = nullptr;
    const int cur = (cv.parity + int(s & 1)) & 1;
    const int ix = item.tx0 + lane;
    if (ix < cv.G.nx && 2 * w < item.rows)
        fused_pair<St, WRITE_NUT, false>(cv.pop[cur], cv.pop[cur ^ 1], cv.fy, cv.nut, nullptr, nullptr, cv.G, ix,
                                         item.ty0 + 2 * w, 2 * w + 1 < item.rows, c);
}

// The node-pair body of k_fused_x (xpair.cuh: two x-adjacent nodes per
// thread, every plane one 32-bit word) with one CTA per (cavity, 64-column x
// rows) item: warp w takes row ty0 + w.  16-bit formats only.
template <class St, bool WRITE_NUT>
__global__ void __maxnreg__(XPAIR_MAXNREG)
    k_batch_x(const BatchCav<St>* __restrict__ cavs, const BatchItem* __restrict__ items,
              const StepScalars<float>* __restrict__ table, int n_cav, long long step,
              const long long* __restrict__ step_dev) {
    pdl_wait();
    pdl_trigger();
    const long long s = step_dev ? *step_dev + step : step;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const BatchItem item = items[blockIdx.x];
    const BatchCav<St>& cv = cavs[item.cav];
    const int row = s < cv.spin_up ? int(s) : cv.spin_up;
    StepScalars<float> c = table[(long long)row * n_cav + item.cav];
    c.step = s;
    c.step_dev = nullptr;
    const int cur = (cv.parity + int(s & 1)) & 1;
    const int ix = item.tx0 + 2 * lane;
    if (ix < cv.G.nx && w < item.rows)
        fused_xpair<St, WRITE_NUT, false>(cv.pop[cur], cv.pop[cur ^ 1], cv.fy, cv.fy, cv.nut, nullptr, nullptr, cv.G,
                                          ix, item.ty0 + w, c);
}

// Which kernel runs a batched step, and the parameters it uses:
//   0  k_batch      persistent grid of ctas_per_sm x #SMs CTAs over
//                   32-column x rows_per_item tiles, one thread per node;
//   1, 2  k_tile    TMA-staged shared-memory tiles of shape 1 or 2,
//                   ctas_per_sm persistent CTAs per SM;
//   3  k_batch_np   one CTA per 32-column x rows_per_item item (rows_per_item
//                   in {1, 2, 4, 8}), one node per thread;
//   4  k_batch_np2  the same items, two rows per thread on packed FP32x2
//                   lanes (rows_per_item in {2, 4, 8}; FP32-arithmetic formats);
//   5  k_batch_x    one CTA per 64-column x rows_per_item item (rows_per_item
//                   in {1, 2, 4, 8}), two x-adjacent nodes per thread, every
//                   plane one 32-bit word (16-bit formats);
//   6  k_tile_x     the node-pair body on TMA-staged shared-memory tiles of
//                   64 columns x rows_per_item rows (4 or 8), ctas_per_sm
//                   persistent CTAs per SM (16-bit formats).
// A kernel a format has no version of runs as kernel 3 (FP64: 4, 5 and 6;
// FP32: 5 and 6).  Parameters a kernel does not use are ignored.
struct BatchTuning {
    int rows_per_item = 4;
    int ctas_per_sm = 8;
    int kernel = 3;
};

struct BatchBase {
    virtual ~BatchBase() = default;
    virtual void setup() = 0;
    virtual void step(int64_t n) = 0;
    virtual void set_tuning(const BatchTuning& t) = 0;
    virtual double time_steps(int steps) = 0;  // ms for `steps` batched steps (advances the state)
    virtual void sync() = 0;
    virtual void set_stall_copies(bool on) = 0;
    std::vector<Solver*> cavs;  // owned
    BatchTuning tun;
    cudaStream_t stream = nullptr;
    int64_t time_step = 0;
    int64_t launches = 0;
    long long total_nodes = 0;
    std::string err;
};

template <class St>
struct Batch final : BatchBase {
    using A = typename Fmt<St>::A;
    std::vector<Impl<St>*> cv;
    BatchCav<St>* d_cavs = nullptr;
    BatchItem* d_items = nullptr;
    StepScalars<A>* d_table = nullptr;
    long long* step_dev = nullptr;
    long long step_dev_val = -1;
    int n_items = 0, grid = 0, n_sm = 0, table_rows = 0;
    cudaGraphExec_t graph = nullptr;
    bool cavs_dirty = true;
    // the tile kernel (tile.cuh)
    TileCav<St>* d_tcavs = nullptr;
    CUtensorMap* d_maps[3] = {nullptr, nullptr, nullptr};   // per tile shape
    // the node-pair tile kernel: tensor maps and tile lists per tile height (4, 8)
    CUtensorMap* d_xmaps[2] = {nullptr, nullptr};
    CUtensorMap* d_fmaps[2] = {nullptr, nullptr};  // the Guo force field of every cavity
    TileItem* d_xitems[2] = {nullptr, nullptr};
    int n_xitems[2] = {0, 0}, xgrid = 0;
    TileItem* d_titems[3] = {nullptr, nullptr, nullptr};
    unsigned* d_err = nullptr;
    unsigned* h_err = nullptr;  // pinned copy of *d_err
    int n_titems[3] = {0, 0, 0}, tgrid = 0;
    bool stall_copies = false;  // test of the bounded waits: arm the barriers, issue no copy

    ~Batch() override {
        if (graph) cudaGraphExecDestroy(graph);
        if (h_err) cudaFreeHost(h_err);
        void* bufs[] = {d_cavs,      d_items,     d_table, step_dev, d_tcavs,   d_maps[1],
                        d_maps[2],   d_titems[1], d_titems[2], d_err,  d_xmaps[0],
                        d_xmaps[1],  d_xitems[0], d_xitems[1], d_fmaps[0], d_fmaps[1]};
        for (void* b : bufs)
            if (b) cudaFree(b);
        for (Solver* s : cavs) delete s;
        if (stream) cudaStreamDestroy(stream);
    }

    // Builds the device tables once all cavities exist (sharing `stream`).
    void setup() override {
        for (Solver* s : cavs) cv.push_back(static_cast<Impl<St>*>(s));
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
        const int n = int(cv.size());
        int max_spin = 0;
        for (auto* c : cv) {
            max_spin = std::max<int>(max_spin, int(c->spin_up));
            total_nodes += (long long)c->p.nx * c->p.ny;
        }
        table_rows = max_spin + 1;
        std::vector<StepScalars<A>> tab(size_t(table_rows) * n);
        for (int r = 0; r < table_rows; ++r)
            for (int i = 0; i < n; ++i) tab[size_t(r) * n + i] = cv[i]->scalars(std::min<int64_t>(r, cv[i]->spin_up));
        CK(cudaMalloc(&d_table, sizeof(StepScalars<A>) * tab.size()));
        CK(cudaMemcpyAsync(d_table, tab.data(), sizeof(StepScalars<A>) * tab.size(), cudaMemcpyHostToDevice,
                           stream));
        CK(cudaMalloc(&d_cavs, sizeof(BatchCav<St>) * n));
        CK(cudaMalloc(&step_dev, sizeof(long long)));
        CK(cudaMalloc(&d_tcavs, sizeof(TileCav<St>) * n));
        CK(cudaMalloc(&d_err, sizeof(unsigned)));
        CK(cudaMemsetAsync(d_err, 0, sizeof(unsigned), stream));
        CK(cudaMallocHost(&h_err, sizeof(unsigned)));
        *h_err = 0;
        setup_tiles<1>();
        setup_tiles<2>();
        if constexpr (is_p16<St>::value) {
            setup_xtiles<4>(0);
            setup_xtiles<8>(1);
        }
        set_tuning(tun);
        CK(cudaStreamSynchronize(stream));
    }

    // Tensor maps of both population buffers of every cavity and the tile
    // list, for tile shape V.
    template <int V>
    void setup_tiles() {
        const int n = int(cv.size());
        std::vector<CUtensorMap> maps(2 * size_t(n));
        for (int i = 0; i < n; ++i)
            for (int b = 0; b < 2; ++b) maps[2 * size_t(i) + b] = make_tile_map<St, V>(cv[i]->pop[b], cv[i]->G);
        CK(cudaMalloc(&d_maps[V], sizeof(CUtensorMap) * maps.size()));
        CK(cudaMemcpyAsync(d_maps[V], maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice,
                           stream));
        std::vector<std::pair<int, int>> sizes;
        for (auto* c : cv) sizes.push_back({c->p.nx, c->p.ny});
        std::vector<TileItem> ti;
        tile_items(sizes, TileShape<St, V>::TY, ti);
        n_titems[V] = int(ti.size());
        CK(cudaMalloc(&d_titems[V], sizeof(TileItem) * ti.size()));
        CK(cudaMemcpyAsync(d_titems[V], ti.data(), sizeof(TileItem) * ti.size(), cudaMemcpyHostToDevice, stream));
        CK(cudaFuncSetAttribute(k_tile<St, V, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TileShape<St, V>::SMEM));
        CK(cudaFuncSetAttribute(k_tile<St, V, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TileShape<St, V>::SMEM));
        CK(cudaStreamSynchronize(stream));
    }

    // Tensor maps (64 + 16 columns x TY + 4 rows x 18 planes) and the tile
    // list of the node-pair tile kernel for tile height TY.
    template <int TY>
    void setup_xtiles(int slot) {
        using TS = TileXShape<TY>;
        const int n = int(cv.size());
        std::vector<CUtensorMap> maps(2 * size_t(n));
        for (int i = 0; i < n; ++i)
            for (int b = 0; b < 2; ++b) maps[2 * size_t(i) + b] = make_box_map<St>(cv[i]->pop[b], cv[i]->G, TX_BX, TS::BY);
        CK(cudaMalloc(&d_xmaps[slot], sizeof(CUtensorMap) * maps.size()));
        CK(cudaMemcpyAsync(d_xmaps[slot], maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice,
                           stream));
        std::vector<CUtensorMap> fmaps(n);
        if constexpr (is_p16<St>::value)
            for (int i = 0; i < n; ++i) fmaps[i] = make_field_map(cv[i]->fy, cv[i]->G, TX_W, TY);
        CK(cudaMalloc(&d_fmaps[slot], sizeof(CUtensorMap) * fmaps.size()));
        CK(cudaMemcpyAsync(d_fmaps[slot], fmaps.data(), sizeof(CUtensorMap) * fmaps.size(), cudaMemcpyHostToDevice,
                           stream));
        std::vector<std::pair<int, int>> sizes;
        for (auto* c : cv) sizes.push_back({c->p.nx, c->p.ny});
        std::vector<TileItem> ti;
        tilex_items(sizes, TY, ti);
        n_xitems[slot] = int(ti.size());
        CK(cudaMalloc(&d_xitems[slot], sizeof(TileItem) * ti.size()));
        CK(cudaMemcpyAsync(d_xitems[slot], ti.data(), sizeof(TileItem) * ti.size(), cudaMemcpyHostToDevice, stream));
        if constexpr (is_p16<St>::value) {
            CK(cudaFuncSetAttribute(k_tile_x<St, TY, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TS::SMEM));
            CK(cudaFuncSetAttribute(k_tile_x<St, TY, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TS::SMEM));
        }
        CK(cudaStreamSynchronize(stream));
    }

    template <int TY>
    int xtile_grid(int slot, int ctas_per_sm) {
        int occ = 0;
        if constexpr (is_p16<St>::value)
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile_x<St, TY, false>, TileXShape<TY>::THREADS,
                                                             TileXShape<TY>::SMEM));
        return std::max(1, std::min(n_xitems[slot], std::max(1, std::min(ctas_per_sm, occ)) * n_sm));
    }

    template <int V>
    int tile_grid(int ctas_per_sm) {
        int occ = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile<St, V, false, false>, TileShape<St, V>::THREADS,
                                                         TileShape<St, V>::SMEM));
        return std::max(1, std::min(n_titems[V], std::max(1, std::min(ctas_per_sm, occ)) * n_sm));
    }

    // The kernel this format runs for a requested one (see BatchTuning).
    static int effective_kernel(int k) {
        if ((k == 5 || k == 6) && !is_p16<St>::value) k = 3;
        if (k == 4 && !Fmt<St>::SHIFT) k = 3;
        return k;
    }

    void set_tuning(const BatchTuning& t) override {
        if (t.rows_per_item < 1 || t.rows_per_item > 1024 || t.ctas_per_sm < 1 || t.ctas_per_sm > 32 ||
            t.kernel < 0 || t.kernel > 6)
            throw ArgError{CAV_ERR_ARG, "tuning out of range"};
        const int k = effective_kernel(t.kernel);
        const int r = t.rows_per_item;
        if ((k == 3 || k == 5) && !(r == 1 || r == 2 || r == 4 || r == 8))
            throw ArgError{CAV_ERR_ARG, "rows_per_item of kernels 3 and 5 must be 1, 2, 4 or 8"};
        if (k == 4 && !(r == 2 || r == 4 || r == 8))
            throw ArgError{CAV_ERR_ARG, "rows_per_item of kernel 4 must be 2, 4 or 8"};
        if (k == 6 && !(r == 4 || r == 8)) throw ArgError{CAV_ERR_ARG, "rows_per_item of kernel 6 must be 4 or 8"};
        tun = t;
        // work items: 64 columns for the node-pair kernel, 32 otherwise
        const int width = k == 5 ? 64 : 32;
        std::vector<BatchItem> items;
        for (int i = 0; i < int(cv.size()); ++i) {
            const int nx = cv[i]->p.nx, ny = cv[i]->p.ny;
            for (int y0 = 0; y0 < ny; y0 += r)
                for (int x0 = 0; x0 < nx; x0 += width) items.push_back({i, x0, y0, std::min(r, ny - y0)});
        }
        if (d_items) CK(cudaFree(d_items));
        n_items = int(items.size());
        CK(cudaMalloc(&d_items, sizeof(BatchItem) * items.size()));
        CK(cudaMemcpyAsync(d_items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice,
                           stream));
        grid = std::max(1, std::min(n_items, t.ctas_per_sm * n_sm));
        if (t.kernel == 1) tgrid = tile_grid<1>(t.ctas_per_sm);
        if (t.kernel == 2) tgrid = tile_grid<2>(t.ctas_per_sm);
        if (k == 6) xgrid = r == 4 ? xtile_grid<4>(0, t.ctas_per_sm) : xtile_grid<8>(1, t.ctas_per_sm);
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        CK(cudaStreamSynchronize(stream));
    }

    // Brings every cavity to PC form at the shared step and refreshes the
    // cavity table (buffer parity relative to the batch clock).
    void enter() {
        for (auto* c : cv) {
            if (!c->pc_form) {
                k_collide_ref<St><<<c->grd, c->blk, 0, stream>>>(c->pop[c->cur], c->pop[c->cur ^ 1], c->rho, c->ux,
                                                                   c->uy, c->tt, c->fy, c->nut, c->G,
                                                                   c->scalars(c->time_step));
                c->check_launch();
                c->cur ^= 1;
                c->pc_form = true;
                c->ref_cached = false;
                c->time_step += 1;
                cavs_dirty = true;
            }
        }
        time_step = cv[0]->time_step;
        for (auto* c : cv)
            if (c->time_step != time_step) throw ArgError{CAV_ERR_STATE, "cavities of a batch out of step"};
        if (cavs_dirty) {
            std::vector<BatchCav<St>> h(cv.size());
            for (size_t i = 0; i < cv.size(); ++i) {
                auto* c = cv[i];
                h[i].pop[0] = c->pop[0];
                h[i].pop[1] = c->pop[1];
                h[i].fy = c->fy;
                h[i].nut = c->nut;
                h[i].G = c->G;
                h[i].parity = (c->cur + int(time_step & 1)) & 1;
                h[i].spin_up = int(c->spin_up);
            }
            CK(cudaMemcpyAsync(d_cavs, h.data(), sizeof(BatchCav<St>) * h.size(), cudaMemcpyHostToDevice, stream));
            std::vector<TileCav<St>> t(cv.size());
            for (size_t i = 0; i < cv.size(); ++i) {
                t[i].pop[0] = h[i].pop[0];
                t[i].pop[1] = h[i].pop[1];
                t[i].fy = h[i].fy;
                t[i].nut = h[i].nut;
                t[i].acc_hot = nullptr;
                t[i].acc_cold = nullptr;
                t[i].G = h[i].G;
                t[i].parity = h[i].parity;
                t[i].spin_up = h[i].spin_up;
            }
            CK(cudaMemcpyAsync(d_tcavs, t.data(), sizeof(TileCav<St>) * t.size(), cudaMemcpyHostToDevice, stream));
            CK(cudaStreamSynchronize(stream));
            cavs_dirty = false;
        }
    }

    template <int V, bool WN>
    void launch_tiles(const long long* sdev, long long step) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(tgrid);
        cfg.blockDim = dim3(TileShape<St, V>::THREADS);
        cfg.dynamicSmemBytes = TileShape<St, V>::SMEM;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, k_tile<St, V, WN, false>, (const TileCav<St>*)d_tcavs,
                              (const CUtensorMap*)d_maps[V], (const TileItem*)d_titems[V], n_titems[V],
                              (const StepScalars<A>*)d_table, int(cv.size()), step, sdev, d_err,
                              int(stall_copies)));
    }

    // The one-CTA-per-item kernels (3, 4, 5) over d_items.
    template <bool WN>
    void launch_np(int k, const long long* sdev, long long step) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(n_items);
        cfg.blockDim = dim3(32 * tun.rows_per_item);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if constexpr (is_p16<St>::value) {
            if (k == 5) {
                CK(cudaLaunchKernelEx(&cfg, k_batch_x<St, WN>, (const BatchCav<St>*)d_cavs, (const BatchItem*)d_items,
                                      (const StepScalars<float>*)d_table, int(cv.size()), step, sdev));
                return;
            }
        }
        if constexpr (Fmt<St>::SHIFT) {
            if (k == 4) {
                cfg.blockDim = dim3(16 * tun.rows_per_item);
                CK(cudaLaunchKernelEx(&cfg, k_batch_np2<St, WN>, (const BatchCav<St>*)d_cavs,
                                      (const BatchItem*)d_items, (const StepScalars<float>*)d_table, int(cv.size()),
                                      step, sdev));
                return;
            }
        }
        CK(cudaLaunchKernelEx(&cfg, k_batch_np<St, WN>, (const BatchCav<St>*)d_cavs, (const BatchItem*)d_items,
                              (const StepScalars<A>*)d_table, int(cv.size()), step, sdev));
    }

    template <int TY, bool WN>
    void launch_xtiles(int slot, const long long* sdev, long long step) {
        if constexpr (is_p16<St>::value) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(xgrid);
            cfg.blockDim = dim3(TileXShape<TY>::THREADS);
            cfg.dynamicSmemBytes = TileXShape<TY>::SMEM;
            cfg.stream = stream;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            CK(cudaLaunchKernelEx(&cfg, k_tile_x<St, TY, WN>, (const TileCav<St>*)d_tcavs,
                                  (const CUtensorMap*)d_xmaps[slot], (const CUtensorMap*)d_fmaps[slot],
                                  (const TileItem*)d_xitems[slot], n_xitems[slot], (const StepScalars<float>*)d_table,
                                  int(cv.size()), step, sdev, d_err));
        }
    }

    void launch(bool write_nut, const long long* sdev, long long step) {
        const int k = effective_kernel(tun.kernel);
        if (k == 6) {
            if (tun.rows_per_item == 4)
                write_nut ? launch_xtiles<4, true>(0, sdev, step) : launch_xtiles<4, false>(0, sdev, step);
            else
                write_nut ? launch_xtiles<8, true>(1, sdev, step) : launch_xtiles<8, false>(1, sdev, step);
            ++launches;
            CK(cudaGetLastError());
            return;
        }
        if (k >= 3) {
            write_nut ? launch_np<true>(k, sdev, step) : launch_np<false>(k, sdev, step);
            ++launches;
            CK(cudaGetLastError());
            return;
        }
        if (tun.kernel == 1 || tun.kernel == 2) {
            if (tun.kernel == 1)
                write_nut ? launch_tiles<1, true>(sdev, step) : launch_tiles<1, false>(sdev, step);
            else
                write_nut ? launch_tiles<2, true>(sdev, step) : launch_tiles<2, false>(sdev, step);
            ++launches;
            CK(cudaGetLastError());
            return;
        }
        if (write_nut)
            k_batch<St, true><<<grid, BATCH_THREADS, 0, stream>>>(d_cavs, d_items, n_items, d_table, int(cv.size()),
                                                                   step, sdev);
        else
            k_batch<St, false><<<grid, BATCH_THREADS, 0, stream>>>(d_cavs, d_items, n_items, d_table,
                                                                    int(cv.size()), step, sdev);
        ++launches;
        CK(cudaGetLastError());
    }

    cudaGraphExec_t get_graph() {
        if (graph) return graph;
        const int64_t l0 = launches;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < GRAPH_STEPS; ++j) launch(false, step_dev, j);
        k_add_step<<<1, 1, 0, stream>>>(step_dev, GRAPH_STEPS);
        cudaGraph_t gr;
        CK(cudaStreamEndCapture(stream, &gr));
        launches = l0;
        CK(cudaGraphInstantiate(&graph, gr, 0));
        cudaGraphDestroy(gr);
        return graph;
    }

    void advance_cavities(int64_t k) {
        for (auto* c : cv) {
            if (k & 1) c->cur ^= 1;
            c->time_step += k;
            c->ref_cached = false;
        }
        time_step += k;
    }

    void step(int64_t n) override {
        if (n <= 0) return;
        bool entered_with_collide = false;
        for (auto* c : cv) entered_with_collide |= !c->pc_form;
        enter();  // may run one collision (the first step from a REF state)
        if (entered_with_collide) n -= 1;
        while (n > 0) {
            if (n > GRAPH_STEPS) {
                cudaGraphExec_t gx = get_graph();
                if (step_dev_val != time_step) {
                    k_set_step<<<1, 1, 0, stream>>>(step_dev, time_step);
                    CK(cudaGetLastError());
                    ++launches;
                    step_dev_val = time_step;
                }
                CK(cudaGraphLaunch(gx, stream));
                launches += GRAPH_STEPS + 1;
                step_dev_val += GRAPH_STEPS;
                advance_cavities(GRAPH_STEPS);
                n -= GRAPH_STEPS;
            } else {
                launch(n == 1, nullptr, time_step);
                advance_cavities(1);
                n -= 1;
            }
        }
    }

    double time_steps(int steps) override {
        enter();
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        step(GRAPH_STEPS + 1);  // warm-up, builds the graph
        CK(cudaEventRecord(a, stream));
        step(steps);
        CK(cudaEventRecord(b, stream));
        CK(cudaEventSynchronize(b));
        check_err();
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return ms;
    }

    // A tile CTA that gave up waiting for its copies (k_tile) sets *d_err;
    // reported once, then cleared (the steps of that launch are lost).
    void check_err() {
        CK(cudaMemcpyAsync(h_err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        if (*h_err) {
            *h_err = 0;
            CK(cudaMemsetAsync(d_err, 0, sizeof(unsigned), stream));
            CK(cudaStreamSynchronize(stream));
            throw ArgError{CAV_ERR_TIMEOUT, "a tile copy did not complete within its bounded wait"};
        }
    }

    void set_stall_copies(bool on) override {
        CK(cudaStreamSynchronize(stream));
        stall_copies = on;
        if (graph) {
            CK(cudaGraphExecDestroy(graph));
            graph = nullptr;
        }
    }

    void sync() override { check_err(); }
};

}  // namespace cav
