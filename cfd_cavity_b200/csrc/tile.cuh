// tile.cuh -- the fused step on shared-memory tiles staged by TMA.
//
// A CTA owns a tile of TILE_X x TY nodes of one cavity (WARPS warps, one
// warp per row, each thread TY / WARPS rows).  The 18 population planes of the tile plus a halo (8 columns on
// each side, so that the box starts on a 16-byte boundary, and 2 rows, the
// reach of the g boundary rows) arrive in shared memory with one
// cp.async.bulk.tensor load per tile, completed on an mbarrier.  CTAs are
// persistent: they stride over a work list of tiles and prefetch the next
// tile into the second stage while the current one is computed, so the bytes
// in flight per SM no longer depend on how many registers the collision
// needs.  The pull reads shared memory with the boundary rules of pull_f /
// pull_g and everything after it is fused_core: a tile kernel step is
// bit-identical to k_fused.
//
// Every wait on an mbarrier is bounded (about one second of %globaltimer);
// a CTA that gives up sets *err, finishes its loop without blocking and
// waits (bounded again) for the copies it issued before returning.  With
// `no_copy` (a test of that path) the barriers are armed but no copy is
// issued, so every wait runs out and nothing is left in flight.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "errors.cuh"
#include "kernels.cuh"

namespace cav {

constexpr int TILE_X = 32;                       // tile columns: one warp per row
constexpr int TILE_HX = 8;                       // staged x halo (16 bytes at 2-byte elements)
constexpr int TILE_HY = 2;                       // staged y halo
constexpr int TILE_BX = TILE_X + 2 * TILE_HX;    // box width
constexpr unsigned long long TILE_WAIT_NS = 1000000000ull;

// Tile shapes: variant 1 (three CTAs per SM for 16-bit storage), variant 2
// (taller tiles, less halo per node).  TY rows, WARPS warps.
template <class St, int V>
struct TileShape {
    static constexpr int E = int(sizeof(St));
    static constexpr int TY = V == 1 ? (E == 2 ? 16 : (E == 4 ? 8 : 4)) : (E == 2 ? 24 : (E == 4 ? 12 : 8));
    static constexpr int WARPS = E == 8 ? 4 : (V == 1 || E == 2 ? 8 : 4);
    static constexpr int BY = TY + 2 * TILE_HY;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int STAGE_ELEMS = NPLANES * BY * TILE_BX;
    static constexpr int STAGE_BYTES = STAGE_ELEMS * E;
    static constexpr int SMEM = 2 * STAGE_BYTES + 128;  // + alignment slack of the stage base
    static_assert(TY % WARPS == 0, "rows per thread");
};

// One cavity as the tile kernel sees it; maps[2 * cav + b] describes pop[b]
// as a 3-D tensor (pitch x ny x 18 planes).
template <class St>
struct TileCav {
    St* pop[2];
    typename Fmt<St>::A* fy;
    typename Fmt<St>::A* nut;
    double* acc_hot;
    double* acc_cold;
    Geom G;
    int parity;   // pop[(parity + s) & 1] holds the state at step s
    int spin_up;  // scalar-table row of the steady state
};
struct TileItem {
    int cav, x0, y0, y1;  // rows y0 .. y1 - 1
};

// ---- mbarrier / TMA (inline PTX) ---------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the phase `parity` of *bar; false after TILE_WAIT_NS.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > TILE_WAIT_NS) return false;
    return true;
}
// One box of a 3-D tensor map into shared memory, completing on *bar.
// x * element size must be a multiple of 16 bytes (the caller's x0 - 8).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// ---- the pull from a staged tile ---------------------------------------------
// S: the stage; (col, row): the node's position in the stage (halo included).
template <class St, int BY>
__device__ __forceinline__ typename Fmt<St>::A tile_at(const St* __restrict__ S, int q, int row, int col) {
    return Fmt<St>::load(S[(q * BY + row) * TILE_BX + col], q);
}

// pull_f / pull_g (kernels.cuh) with the sources taken from the stage, in
// lane units (Fmt::lload).
template <class St, int BY>
__device__ __forceinline__ void pull_tile(const St* __restrict__ S, const Geom& G, int ix, int iy, int row, int col,
                                          const StepScalars<typename Fmt<St>::A>& c, typename Fmt<St>::A (&f)[Q],
                                          typename Fmt<St>::A (&g)[Q]) {
    using A = typename Fmt<St>::A;
    const bool xm = ix > 0, xp = ix < G.nx - 1, ym = iy > 0, yp = iy < G.ny - 1;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = CX(i), cy = CY(i);
        const bool ok = (cx > 0 ? xm : (cx < 0 ? xp : true)) && (cy > 0 ? ym : (cy < 0 ? yp : true));
        const int off = ok ? (i * BY + row - cy) * TILE_BX + col - cx : (OPP(i) * BY + row) * TILE_BX + col;
        f[i] = Fmt<St>::lload(S[off], i);
    }
    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
    const int grow = row + (gy - iy);
    const bool wall_col = (ix == 0) || (ix == G.nx - 1);
    const A tw = (ix == 0 ? c.t_hot[gy] : c.t_cold) * p2(Fmt<St>::EG);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int off = wall_col ? ((Q + i) * BY + row) * TILE_BX + col
                                 : ((Q + i) * BY + grow - CY(i)) * TILE_BX + col - CX(i);
        const A v = Fmt<St>::lload(S[off], Q + i);
        g[i] = wall_col ? geq_rest<A>(i, tw, c.geq_order) : v;
    }
}

// gather_t (kernels.cuh) from the stage: T of the streamed state at column x
// of the node's row (x inside the tile or its halo).
template <class St, int BY>
__device__ __forceinline__ typename Fmt<St>::A tile_t(const St* __restrict__ S, const Geom& G, int x, int iy, int row,
                                                     int col_x, const StepScalars<typename Fmt<St>::A>& c) {
    using A = typename Fmt<St>::A;
    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
    const int grow = row + (gy - iy);
    A g[Q];
    if (x == 0) {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = geq_rest<A>(i, c.t_hot[gy], c.geq_order);
    } else if (x == G.nx - 1) {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = geq_rest<A>(i, c.t_cold, c.geq_order);
    } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = tile_at<St, BY>(S, Q + i, grow - CY(i), col_x - CX(i));
    }
    A t = g[0];
#pragma unroll
    for (int j = 1; j < Q; ++j) t = t + g[j];
    return t;
}

// ---- the kernel --------------------------------------------------------------
// One lattice step of every tile in `items`; step scalars of cavity c at
// step s are table[min(s, spin_up) * n_cav + c] (step = s, as k_batch).
template <class St, int V, bool WRITE_NUT, bool ACC_NU>
__global__ void __launch_bounds__(TileShape<St, V>::THREADS)
    k_tile(const TileCav<St>* __restrict__ cavs, const CUtensorMap* __restrict__ maps,
           const TileItem* __restrict__ items, int n_items, const StepScalars<typename Fmt<St>::A>* __restrict__ table,
           int n_cav, long long step, const long long* __restrict__ step_dev, unsigned* __restrict__ err,
           int no_copy) {
    using A = typename Fmt<St>::A;
    using TS = TileShape<St, V>;
    extern __shared__ __align__(128) unsigned char tile_smem[];
    __shared__ __align__(8) uint64_t bar[2];
    // TMA destinations on a 128-byte boundary
    unsigned char* base = tile_smem + ((128u - (smem_u32(tile_smem) & 127u)) & 127u);
    St* stage0 = reinterpret_cast<St*>(base);
    St* stage1 = reinterpret_cast<St*>(base + TS::STAGE_BYTES);
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;  // column, first row
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    const long long s = step_dev ? *step_dev + step : step;
    auto issue = [&](int item, int st) {
        const TileItem I = items[item];
        const int b = (cavs[I.cav].parity + int(s & 1)) & 1;
        uint64_t* br = &bar[st];
        mbar_expect_tx(br, TS::STAGE_BYTES);
        if (!no_copy)
            tma_load_3d(st ? stage1 : stage0, maps + 2 * I.cav + b, br, I.x0 - TILE_HX, I.y0 - TILE_HY, 0);
    };
    if (threadIdx.x == 0 && int(blockIdx.x) < n_items) issue(blockIdx.x, 0);
    int k = 0;
    bool next_issued = false, failed = false;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x, ++k) {
        const int st = k & 1;
        next_issued = it + int(gridDim.x) < n_items;
        if (threadIdx.x == 0 && next_issued) issue(it + gridDim.x, st ^ 1);
        const bool ok = mbar_wait_bounded(&bar[st], uint32_t((k >> 1) & 1));
        const TileItem I = items[it];
        const TileCav<St> cv = cavs[I.cav];
        const Geom G = cv.G;
        const int ix = I.x0 + lx;
        if (ok && ix < G.nx) {
            const int row = s < cv.spin_up ? int(s) : cv.spin_up;
            StepScalars<A> c = table[(long long)row * n_cav + I.cav];
            c.step = s;
            c.step_dev = nullptr;
            const int cur = (cv.parity + int(s & 1)) & 1;
            const St* S = st ? stage1 : stage0;
            const int tcol = lx + TILE_HX;
#pragma unroll 1
            for (int r = ly; r < TS::TY; r += TS::WARPS) {
                const int iy = I.y0 + r;
                if (iy >= G.ny) break;
                const int trow = r + TILE_HY;
                A f[Q], g[Q];
                pull_tile<St, TS::BY>(S, G, ix, iy, trow, tcol, c, f, g);
                fused_core<St, WRITE_NUT, ACC_NU, false>(
                    f, g, cv.pop[cur ^ 1], cv.fy, cv.fy, cv.nut, cv.acc_hot, cv.acc_cold, G, ix, iy, c,
                    [&](int x) { return tile_t<St, TS::BY>(S, G, x, iy, trow, x - I.x0 + TILE_HX, c); });
            }
        }
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
    }
    if (failed && threadIdx.x == 0) {
        // let the copies this CTA issued land before it exits (bounded)
        atomicOr(err, 1u);
        mbar_wait_bounded(&bar[k & 1], uint32_t((k >> 1) & 1));
        if (next_issued) mbar_wait_bounded(&bar[(k + 1) & 1], uint32_t(((k + 1) >> 1) & 1));
    }
}

// ---- host: tensor maps ---------------------------------------------------------
inline PFN_cuTensorMapEncodeTiled_v12000 tile_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) throw ArgError{CAV_ERR_CUDA, "cuTensorMapEncodeTiled unavailable"};
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// pop (18 planes of ny x pitch St) as a 3-D tensor with a box of box_x x
// box_y x 18 elements.
template <class St>
CUtensorMap make_box_map(const St* pop, const Geom& G, int box_x, int box_y) {
    static_assert(sizeof(St) == 2 || sizeof(St) == 4 || sizeof(St) == 8, "element size");
    if ((G.pitch * sizeof(St)) % 16 != 0 || (reinterpret_cast<uintptr_t>(pop) & 15) != 0)
        throw ArgError{CAV_ERR_ARG, "tile map: rows must start on 16-byte boundaries"};
    CUtensorMap m;
    const CUtensorMapDataType dt = sizeof(St) == 2   ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                   : sizeof(St) == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32
                                                     : CU_TENSOR_MAP_DATA_TYPE_UINT64;
    const cuuint64_t dims[3] = {cuuint64_t(G.pitch), cuuint64_t(G.ny), cuuint64_t(NPLANES)};
    const cuuint64_t strides[2] = {cuuint64_t(G.pitch) * sizeof(St), cuuint64_t(G.plane) * sizeof(St)};
    if ((box_x * sizeof(St)) % 16 != 0 || box_x > 256 || box_y > 256)
        throw ArgError{CAV_ERR_ARG, "tile map: box rows must be multiples of 16 bytes, at most 256 elements"};
    const cuuint32_t box[3] = {cuuint32_t(box_x), cuuint32_t(box_y), cuuint32_t(NPLANES)};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = tile_map_encoder()(&m, dt, 3, const_cast<St*>(pop), dims, strides, box, estr,
                                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw ArgError{CAV_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")"};
    return m;
}

// A pitched FP32 field (ny rows of pitch floats) as a 2-D tensor with a box
// of box_x x box_y elements.
inline CUtensorMap make_field_map(const float* field, const Geom& G, int box_x, int box_y) {
    if ((G.pitch * sizeof(float)) % 16 != 0 || (reinterpret_cast<uintptr_t>(field) & 15) != 0 ||
        (box_x * sizeof(float)) % 16 != 0 || box_x > 256 || box_y > 256)
        throw ArgError{CAV_ERR_ARG, "field map: rows and box rows must be multiples of 16 bytes"};
    CUtensorMap m;
    const cuuint64_t dims[2] = {cuuint64_t(G.pitch), cuuint64_t(G.ny)};
    const cuuint64_t strides[1] = {cuuint64_t(G.pitch) * sizeof(float)};
    const cuuint32_t box[2] = {cuuint32_t(box_x), cuuint32_t(box_y)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = tile_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(field), dims,
                                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw ArgError{CAV_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")"};
    return m;
}

// ... with the box of tile shape V.
template <class St, int V>
CUtensorMap make_tile_map(const St* pop, const Geom& G) {
    return make_box_map<St>(pop, G, TILE_BX, TileShape<St, V>::BY);
}

// Tiles of every cavity, cavity-major then row-block then column block.
inline void tile_items(const std::vector<std::pair<int, int>>& sizes, int ty, std::vector<TileItem>& out) {
    out.clear();
    for (int i = 0; i < int(sizes.size()); ++i)
        for (int y0 = 0; y0 < sizes[i].second; y0 += ty)
            for (int x0 = 0; x0 < sizes[i].first; x0 += TILE_X)
                out.push_back({i, x0, y0, std::min(y0 + ty, sizes[i].second)});
}

}  // namespace cav
