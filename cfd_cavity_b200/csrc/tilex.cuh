// tilex.cuh -- the node-pair step on shared-memory tiles staged by TMA
// (16-bit storage).
//
// A CTA owns tiles of 64 columns x TY rows of one cavity: four warps, each
// a row at a time, each thread the node pair (2 lane, 2 lane + 1) of the
// tile's row.  The 18 population planes of a tile plus a halo (8 columns on
// each side, so that the box starts on a 16-byte boundary, and 2 rows, the
// reach of the g boundary rows) arrive in shared memory with one
// cp.async.bulk.tensor load completing on an mbarrier.  CTAs are persistent:
// they stride over the work list and prefetch the next tile into the second
// stage while the current one is computed, so the population loads of the
// pull come from shared memory (no DRAM latency in the node's chain) and the
// tensor engine keeps the bytes of the next tile in flight.  The pull reads
// the staged words with the selectors of pull_f_x / pull_g_x and everything
// after it is xpair_core: bit-identical to k_fused_x and k_batch_x.
//
// Every wait on an mbarrier is bounded (tile.cuh: about one second); a CTA
// that gives up sets *err, leaves its loop and waits (bounded again) for the
// copies it issued before returning.
#pragma once

#include "tile.cuh"
#include "xpair.cuh"

namespace cav {

constexpr int TX_W = 64;                   // tile columns (32 node pairs)
constexpr int TX_BX = TX_W + 2 * TILE_HX;  // box width, halo included (80)
constexpr int TX_WORDS = TX_BX / 2;        // 32-bit words per staged row (40)

template <int TY_>
struct TileXShape {
    static constexpr int TY = TY_;
    static constexpr int WARPS = 4;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int BY = TY + 2 * TILE_HY;
    static constexpr int STAGE_BYTES = NPLANES * BY * TX_BX * 2;
    static constexpr int SMEM = 2 * STAGE_BYTES + 128;  // + alignment slack of the stage base
    static_assert(TY % WARPS == 0 && STAGE_BYTES % 128 == 0, "tile shape");
};

// pull_f_x from a staged tile: trow = the row's position in the stage (halo
// included), wc = the pair's word column (4 + lane).
template <int BY>
__device__ __forceinline__ void pull_f_tx(const uint32_t* __restrict__ S, const Geom& G, int ix, int iy, int trow,
                                          int wc, uint32_t (&w)[Q]) {
    const bool ym = iy > 0, yp = iy < G.ny - 1;
    const bool x0 = ix == 0, xe = ix + 1 >= G.nx, xl = ix + 2 >= G.nx;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = CX(i), cy = CY(i);
        const bool y_ok = cy > 0 ? ym : (cy < 0 ? yp : true);
        const int own = (OPP(i) * BY + trow) * TX_WORDS + wc;
        const int srow = (i * BY + trow - cy) * TX_WORDS + wc;
        if (cx == 0) {
            w[i] = S[y_ok ? srow : own];
        } else if (cx > 0) {
            const uint32_t w1 = S[y_ok ? srow : own];
            const uint32_t w0 = S[(y_ok && !x0) ? srow - 1 : own];
            w[i] = __byte_perm(w0, w1, !y_ok ? 0x7654u : (x0 ? 0x5410u : 0x5432u));
        } else {
            const uint32_t w0 = S[(y_ok && !xe) ? srow : own];
            const uint32_t w1 = S[(y_ok && !xl) ? srow + 1 : own];
            w[i] = __byte_perm(w0, w1, (!y_ok || xe) ? 0x3210u : (xl ? 0x7632u : 0x5432u));
        }
    }
}

// pull_g_x from a staged tile.
template <int BY>
__device__ __forceinline__ void pull_g_tx(const uint32_t* __restrict__ S, const Geom& G, int ix, int iy, int trow,
                                          int wc, uint32_t (&w)[Q]) {
    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
    const int grow = trow + (gy - iy);
    const bool x0 = ix == 0, xl = ix + 2 >= G.nx;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = CX(i), cy = CY(i);
        const int srow = ((Q + i) * BY + grow - cy) * TX_WORDS + wc;
        if (cx == 0) {
            w[i] = S[srow];
        } else if (cx > 0) {
            w[i] = __byte_perm(S[x0 ? srow : srow - 1], S[srow], 0x5432u);
        } else {
            w[i] = __byte_perm(S[srow], S[xl ? srow : srow + 1], 0x5432u);
        }
    }
}

// One lattice step of every tile in `items` (x0 multiples of 64, y0 of TY);
// step scalars of cavity c at step s are table[min(s, spin_up) * n_cav + c].
template <class St, int TY, bool WRITE_NUT>
__global__ void __launch_bounds__(TileXShape<TY>::THREADS, 4)
    k_tile_x(const TileCav<St>* __restrict__ cavs, const CUtensorMap* __restrict__ maps,
             const TileItem* __restrict__ items, int n_items, const StepScalars<float>* __restrict__ table, int n_cav,
             long long step, const long long* __restrict__ step_dev, unsigned* __restrict__ err) {
    using TS = TileXShape<TY>;
    extern __shared__ __align__(128) unsigned char tilex_smem[];
    __shared__ __align__(8) uint64_t bar[2];
    // TMA destinations on a 128-byte boundary
    unsigned char* base = tilex_smem + ((128u - (smem_u32(tilex_smem) & 127u)) & 127u);
    const uint32_t* stage0 = reinterpret_cast<const uint32_t*>(base);
    const uint32_t* stage1 = reinterpret_cast<const uint32_t*>(base + TS::STAGE_BYTES);
    const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
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
        tma_load_3d(const_cast<uint32_t*>(st ? stage1 : stage0), maps + 2 * I.cav + b, br, I.x0 - TILE_HX,
                    I.y0 - TILE_HY, 0);
    };
    if (threadIdx.x == 0 && int(blockIdx.x) < n_items) issue(blockIdx.x, 0);
    int k = 0;
    bool next_issued = false, failed = false;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x, ++k) {
        const int st = k & 1;
        next_issued = it + int(gridDim.x) < n_items;
        if (threadIdx.x == 0 && next_issued) issue(it + gridDim.x, st ^ 1);
        // what does not depend on the staged tile, before the wait: the
        // tile's cavity and step scalars, and this warp's rows of the
        // previous Guo force (the only per-node global loads of the step)
        const TileItem I = items[it];
        const TileCav<St> cv = cavs[I.cav];
        const Geom G = cv.G;
        const int ix = I.x0 + 2 * lane;
        const int srow = s < cv.spin_up ? int(s) : cv.spin_up;
        StepScalars<float> c = table[(long long)srow * n_cav + I.cav];
        c.step = s;
        c.step_dev = nullptr;
        // (a select, not cv.pop[index]: an indexed copy would live in local memory)
        St* const dst = ((cv.parity + int(s & 1)) & 1) ? cv.pop[0] : cv.pop[1];
        constexpr int RPW = TY / TS::WARPS;  // rows per warp
        float2 fyp[RPW];
        float thp[RPW];
#pragma unroll
        for (int j = 0; j < RPW; ++j) {
            const int iy = I.y0 + wy + j * TS::WARPS;
            const bool in = ix < G.nx && iy < G.ny;
            fyp[j] = in ? *reinterpret_cast<const float2*>(cv.fy + iy * G.pitch + ix) : make_float2(0.0f, 0.0f);
            const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
            thp[j] = in ? c.t_hot[gy] : 0.0f;
        }
        const bool ok = mbar_wait_bounded(&bar[st], uint32_t((k >> 1) & 1));
        if (ok && ix < G.nx) {
            const uint32_t* S = st ? stage1 : stage0;
#pragma unroll
            for (int j = 0; j < RPW; ++j) {
                const int r = wy + j * TS::WARPS;
                const int iy = I.y0 + r;
                if (iy < G.ny) {
                    const int trow = r + TILE_HY, wc = TILE_HX / 2 + lane;
                    xpair_core<St, WRITE_NUT, false, false>(
                        [=](uint32_t(&w)[Q]) { pull_f_tx<TS::BY>(S, G, ix, iy, trow, wc, w); },
                        [=](uint32_t(&w)[Q]) { pull_g_tx<TS::BY>(S, G, ix, iy, trow, wc, w); },
                        [](int) { return 0.0f; }, dst, fyp[j], thp[j], cv.fy, cv.nut, nullptr, nullptr, G, ix, iy,
                        c);
                }
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

// Tiles of 64 columns x ty rows of every cavity, cavity-major then row block
// then column block.
inline void tilex_items(const std::vector<std::pair<int, int>>& sizes, int ty, std::vector<TileItem>& out) {
    out.clear();
    for (int i = 0; i < int(sizes.size()); ++i)
        for (int y0 = 0; y0 < sizes[i].second; y0 += ty)
            for (int x0 = 0; x0 < sizes[i].first; x0 += TX_W) out.push_back({i, x0, y0});
}

}  // namespace cav
