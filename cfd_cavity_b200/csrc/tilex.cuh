// tilex.cuh -- the node-pair step on shared-memory tiles staged by TMA
// (16-bit storage).
//
// A CTA owns tiles of 64 columns x (at most) TY rows of one cavity: four
// warps, each a row at a time, each thread the node pair (2 lane,
// 2 lane + 1) of the tile's row.  The 18 population planes of a tile plus a
// halo (8 columns on each side, so that the box starts on a 16-byte
// boundary, and 1 row) arrive in shared memory with one cp.async.bulk.tensor
// load completing on an mbarrier.  The g boundary rows 0 / ny-1 read rows up
// to 2 away (the post-stream g of rows 1 / ny-2); one halo row suffices
// because every tile is at least two rows tall (tilex_items), so those rows
// lie inside the tile or its halo.  CTAs are persistent:
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
constexpr int TX_HY = 1;                   // staged y halo

template <int TY_>
struct TileXShape {
    static constexpr int TY = TY_;
    static constexpr int WARPS = 4;  // each warp TY / WARPS rows
    // resident CTAs per SM the register budget is sized for (4-row tiles: 96
    // registers, 5 CTAs)
    static constexpr int MIN_CTAS = TY_ == 4 ? 5 : 4;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int BY = TY + 2 * TX_HY;
    static constexpr int POP_BYTES = NPLANES * BY * TX_BX * 2;  // the populations of the tile and its halo
    static constexpr int FY_BYTES = TY * TX_W * 4;              // the previous Guo force of the tile
    static constexpr int STAGE_BYTES = POP_BYTES + FY_BYTES;
    static constexpr int SMEM = 2 * STAGE_BYTES + 128;  // + alignment slack of the stage base
    static_assert(TY % WARPS == 0 && POP_BYTES % 128 == 0 && FY_BYTES % 128 == 0, "tile shape");
};

// The cavity of the tiles in flight, kept in shared memory (refreshed when
// a CTA's tile range crosses into another cavity).
template <class St>
struct TileXMeta {
    TileCav<St> cv;
    StepScalars<float> c;
};

// One box of a 2-D tensor map into shared memory, completing on *bar
// (x * element size a multiple of 16 bytes).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// pull_f_x from a staged tile: trow = the row's position in the stage (halo
// included), wc = the pair's word column (4 + lane).  INTERIOR: the row is
// neither 0 nor ny - 1 (no bounce-back in y; the caller branches on the
// row, the same for the whole warp).
template <int BY, bool INTERIOR = false>
__device__ __forceinline__ void pull_f_tx(const uint32_t* __restrict__ S, const Geom& G, int ix, int iy, int trow,
                                          int wc, uint32_t (&w)[Q]) {
    const bool ym = INTERIOR || iy > 0, yp = INTERIOR || iy < G.ny - 1;
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

// One lattice step of every tile in `items` (x0 multiples of 64, y0 of TY;
// cavity-major); step scalars of cavity c at step s are
// table[min(s, spin_up) * n_cav + c].  CTA b takes the contiguous range of
// tiles [b per, (b + 1) per), so consecutive tiles share the cavity (its
// metadata is loaded once per range crossing) and their halo rows (L2).  Per
// tile, the populations with their halo (maps[2 cav + buffer]) and the
// previous Guo force of the tile (fmaps[cav]) arrive by TMA; the next tile's
// copies are issued before the current one is computed.
template <class St, int TY, bool WRITE_NUT>
__global__ void __launch_bounds__(TileXShape<TY>::THREADS, TileXShape<TY>::MIN_CTAS)
    k_tile_x(const TileCav<St>* __restrict__ cavs, const CUtensorMap* __restrict__ maps,
             const CUtensorMap* __restrict__ fmaps, const TileItem* __restrict__ items, int n_items,
             const StepScalars<float>* __restrict__ table, int n_cav, long long step,
             const long long* __restrict__ step_dev, unsigned* __restrict__ err) {
    using TS = TileXShape<TY>;
    extern __shared__ __align__(128) unsigned char tilex_smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ TileXMeta<St> meta;
    // TMA destinations on a 128-byte boundary
    unsigned char* base = tilex_smem + ((128u - (smem_u32(tilex_smem) & 127u)) & 127u);
    unsigned char* const stage0 = base;
    unsigned char* const stage1 = base + TS::STAGE_BYTES;
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
    const int per = (n_items + int(gridDim.x) - 1) / int(gridDim.x);
    const int it0 = min(n_items, int(blockIdx.x) * per), it1 = min(n_items, it0 + per);
    // the issuing thread's cavity and its buffer parity
    int icav = -1, ipar = 0;
    auto issue = [&](const TileItem& I, int st) {
        if (I.cav != icav) {
            icav = I.cav;
            ipar = cavs[I.cav].parity;
        }
        const int b = (ipar + int(s & 1)) & 1;
        mbar_expect_tx(&bar[st], TS::STAGE_BYTES);
        unsigned char* const d = st ? stage1 : stage0;
        tma_load_3d(d, maps + 2 * I.cav + b, &bar[st], I.x0 - TILE_HX, I.y0 - TX_HY, 0);
        tma_load_2d(d + TS::POP_BYTES, fmaps + I.cav, &bar[st], I.x0, I.y0);
    };
    TileItem Icur{0, 0, 0, 0}, Inext{0, 0, 0, 0};
    if (it0 < it1) {
        Icur = items[it0];
        if (threadIdx.x == 0) issue(Icur, 0);
    }
    if (it0 + 1 < it1) Inext = items[it0 + 1];
    int mcav = -1;  // the cavity whose metadata is in `meta`
    int k = 0;
    bool next_issued = false, failed = false;
    for (int it = it0; it < it1; ++it, ++k) {
        const int st = k & 1;
        next_issued = it + 1 < it1;
        if (threadIdx.x == 0 && next_issued) issue(Inext, st ^ 1);
        const TileItem I = Icur;
        Icur = Inext;
        if (it + 2 < it1) Inext = items[it + 2];
        if (I.cav != mcav) {  // the same for every thread of the CTA
            if (threadIdx.x == 0) {
                meta.cv = cavs[I.cav];
                const int row = s < meta.cv.spin_up ? int(s) : meta.cv.spin_up;
                meta.c = table[(long long)row * n_cav + I.cav];
                meta.c.step = s;
                meta.c.step_dev = nullptr;
            }
            __syncthreads();
            mcav = I.cav;
        }
        const Geom G = meta.cv.G;
        const int ix = I.x0 + 2 * lane;
        const bool ok = mbar_wait_bounded(&bar[st], uint32_t((k >> 1) & 1));
        if (ok && ix < G.nx) {
            const unsigned char* const sb = st ? stage1 : stage0;
            const uint32_t* S = reinterpret_cast<const uint32_t*>(sb);
            const float* FY = reinterpret_cast<const float*>(sb + TS::POP_BYTES);
            // (a select, not pop[index]: an indexed copy would live in local memory)
            St* const dst = ((meta.cv.parity + int(s & 1)) & 1) ? meta.cv.pop[0] : meta.cv.pop[1];
#pragma unroll
            for (int j = 0; j < TY / TS::WARPS; ++j) {
                const int r = wy + j * TS::WARPS;
                const int iy = I.y0 + r;
                if (iy < I.y1) {
                    const int trow = r + TX_HY, wc = TILE_HX / 2 + lane;
                    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
                    const float th = ix == 0 ? meta.c.t_hot[gy] : 0.0f;
                    xpair_core<St, WRITE_NUT, false, false>(
                        [=](uint32_t(&w)[Q]) {
                            if (iy > 0 && iy < G.ny - 1)
                                pull_f_tx<TS::BY, true>(S, G, ix, iy, trow, wc, w);
                            else
                                pull_f_tx<TS::BY, false>(S, G, ix, iy, trow, wc, w);
                        },
                        [=](uint32_t(&w)[Q]) { pull_g_tx<TS::BY>(S, G, ix, iy, trow, wc, w); },
                        [](int) { return 0.0f; }, dst, *reinterpret_cast<const float2*>(FY + r * TX_W + 2 * lane),
                        th, meta.cv.fy, meta.cv.nut, nullptr, nullptr, G, ix, iy, meta.c);
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
// then column block; where the last row block would be a single row, the
// block before it gives it one row (every tile at least two rows tall).
inline void tilex_items(const std::vector<std::pair<int, int>>& sizes, int ty, std::vector<TileItem>& out) {
    out.clear();
    for (int i = 0; i < int(sizes.size()); ++i) {
        const int ny = sizes[i].second;
        std::vector<std::pair<int, int>> rows;
        for (int y0 = 0; y0 < ny; y0 += ty) rows.push_back({y0, std::min(y0 + ty, ny)});
        if (rows.size() > 1 && rows.back().second - rows.back().first == 1) {
            rows[rows.size() - 2].second -= 1;
            rows.back().first -= 1;
        }
        for (const auto& r : rows)
            for (int x0 = 0; x0 < sizes[i].first; x0 += TX_W) out.push_back({i, x0, r.first, r.second});
    }
}

}  // namespace cav
