// xpair.cuh -- the fused step on two x-adjacent nodes per thread (16-bit
// population storage).
//
// A thread owns the nodes (ix, iy) and (ix + 1, iy), ix even.  In the SoA
// planes (pitch a multiple of 32 elements) those two 16-bit values are one
// aligned 32-bit word, node ix in the low half, so every plane is pulled and
// stored as words:
//  - directions with c_x = 0: one word load (the source pair is aligned);
//  - c_x = +1 / -1: the two source values straddle two words; both words are
//    loaded and one byte permute (prmt) assembles the pair, with the
//    bounce-back / wall cases chosen by the permute selector;
//  - the collision's results for a plane of the two nodes are rounded
//    together by one cvt.{rn,rs}.{f16x2,bf16x2}.f32 and written by one
//    32-bit store.
// The macroscopic update and the collision run on Blackwell's packed FP32x2
// add / mul / fma (the lane arithmetic of lattice.cuh): every operation is
// explicitly rounded, so each node gets exactly the bits the one-node
// kernels give it.  Stochastic rounding draws its bits per node pair (see
// sr_pair_rng in kernels.cuh), the convention every uniform-solver kernel
// follows, so a cavity stepped by either kernel is bit for bit the same.
#pragma once

#include "kernels.cuh"

namespace cav {

// Register budget of the node-pair kernels.
#ifndef XPAIR_MAXNREG
#define XPAIR_MAXNREG 96
#endif

template <class St>
struct PairEnc;

template <int KIND, bool SRND>
struct PairEnc<P16<KIND, SRND>> {
    using F = Fmt<P16<KIND, SRND>>;
    static constexpr bool SR = SRND;
    // lane units (the formats' own power-of-two scales), as Fmt::lload
    __device__ static float2 dec(uint32_t w, int q) {
        if constexpr (KIND == K_BF16) {
            return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
        } else {
            if (KIND == K_MIX && q >= Q)
                return make_float2(fx_load((unsigned short)(w & 0xffffu), q), fx_load((unsigned short)(w >> 16), q));
            return make_float2(h16_raw((unsigned short)(w & 0xffffu)), h16_raw((unsigned short)(w >> 16)));
        }
    }
    // v.x -> low half (node ix), v.y -> high half (node ix + 1); r: the
    // pair's draw for this plane (stochastic formats).
    __device__ static uint32_t enc(float2 v, int q, uint32_t r) {
        uint32_t d;
        if constexpr (KIND == K_BF16) {
            if constexpr (SRND)
                asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(v.y), "f"(v.x), "r"(sr_bits_bf16(r)));
            else
                asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(v.y), "f"(v.x));
        } else {
            if (KIND == K_MIX && q >= Q) {
                const uint32_t lo = fx_store(v.x, q, SRND, sr_bits_fx(r, 0));
                const uint32_t hi = fx_store(v.y, q, SRND, sr_bits_fx(r, 1));
                return (lo & 0xffffu) | (hi << 16);
            }
            if constexpr (SRND)
                asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(v.y), "f"(v.x), "r"(sr_bits_f16(r)));
            else
                asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(v.y), "f"(v.x));
        }
        return d;
    }
};

// Pull of the f planes of the pair (stream, src/uniform/solver.rs:838-913):
// f_i(x) = f*_i(x - c_i) in the domain, else f*_opp(i)(x) (bounce-back).
// Words of raw storage bits, node ix in the low half.
template <class St>
__device__ __forceinline__ void pull_f_x(const St* __restrict__ src, const Geom& G, int ix, int iy,
                                         uint32_t (&w)[Q]) {
    const uint32_t* __restrict__ s = reinterpret_cast<const uint32_t*>(src);
    const int P2 = int(G.plane >> 1), W2 = G.pitch >> 1;
    const int k2 = iy * W2 + (ix >> 1);
    const bool ym = iy > 0, yp = iy < G.ny - 1;
    const bool x0 = ix == 0;            // node ix: its c_x = +1 sources are outside
    const bool xe = ix + 1 >= G.nx;     // node ix (the last column, odd nx): its c_x = -1 sources are outside
    const bool xl = ix + 2 >= G.nx;     // node ix + 1: its c_x = -1 sources are outside
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = CX(i), cy = CY(i);
        const bool y_ok = cy > 0 ? ym : (cy < 0 ? yp : true);
        const int own = OPP(i) * P2 + k2;       // the pair's word of the opposite plane
        const int srow = i * P2 + k2 - cy * W2; // word (ix, iy - c_y) of plane i
        if (cx == 0) {
            w[i] = s[y_ok ? srow : own];
        } else if (cx > 0) {
            // low half: (ix - 1) = high half of the word to the left; high
            // half: (ix) = low half of the word above/below
            const uint32_t w1 = s[y_ok ? srow : own];
            const uint32_t w0 = s[(y_ok && !x0) ? srow - 1 : own];
            w[i] = __byte_perm(w0, w1, !y_ok ? 0x7654u : (x0 ? 0x5410u : 0x5432u));
        } else {
            // low half: (ix + 1) = high half of the pair's word; high half:
            // (ix + 2) = low half of the word to the right; where a source
            // is outside, the opposite plane's value at the node itself
            // (the pair's own word: low half for ix, high half for ix + 1)
            const uint32_t w0 = s[(y_ok && !xe) ? srow : own];
            const uint32_t w1 = s[(y_ok && !xl) ? srow + 1 : own];
            w[i] = __byte_perm(w0, w1, (!y_ok || xe) ? 0x3210u : (xl ? 0x7632u : 0x5432u));
        }
    }
}

// Pull of the g planes with the thermal boundary conditions
// (src/uniform/solver.rs:951-988): rows 0 / ny-1 take the post-stream g of
// rows 1 / ny-2; wall columns are overwritten by the caller (equilibrium of
// the wall temperature), so their words may hold anything.
template <class St>
__device__ __forceinline__ void pull_g_x(const St* __restrict__ src, const Geom& G, int ix, int iy,
                                         uint32_t (&w)[Q]) {
    const uint32_t* __restrict__ s = reinterpret_cast<const uint32_t*>(src);
    const int P2 = int(G.plane >> 1), W2 = G.pitch >> 1;
    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
    const int k2 = gy * W2 + (ix >> 1);
    const bool x0 = ix == 0, xl = ix + 2 >= G.nx;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = CX(i), cy = CY(i);
        const int srow = (Q + i) * P2 + k2 - cy * W2;
        if (cx == 0) {
            w[i] = s[srow];
        } else if (cx > 0) {
            w[i] = __byte_perm(s[x0 ? srow : srow - 1], s[srow], 0x5432u);
        } else {
            w[i] = __byte_perm(s[srow], s[xl ? srow : srow + 1], 0x5432u);
        }
    }
}

// Everything of one node-pair step after the pull: the macroscopic update
// with the Guo half force, no-slip, the collision of the next step and the
// stores (what fused_core does for one node).  pull_f(wf) / pull_g(wg) fill
// the pulled f / g words (from global memory or a staged tile); t_at(x) is T
// of the streamed state at column x of the row (Nusselt accumulation only);
// fy_prev the previous collision's Guo force of the pair.  Node ix + 1 may
// lie in the row padding (odd nx): its values are computed and stored into
// the padding, which no kernel reads as a node.
// NO_COLLIDE: identity collision (the pulled values are stored back; checks
// the pull / bounce-back / boundary index maps bit for bit).
// t_hot_row: the hot-wall theta of the row's g source row (c.t_hot[gy]).
template <class St, bool WRITE_NUT, bool ACC_NU, bool NO_COLLIDE, class PF, class PG, class TAt>
__device__ __forceinline__ void xpair_core(PF&& pull_f, PG&& pull_g, TAt&& t_at, St* __restrict__ dst,
                                           float2 fy_prev, float t_hot_row, float* fy_out, float* __restrict__ nut,
                                           double* __restrict__ acc_hot, double* __restrict__ acc_cold,
                                           const Geom& G, int ix, int iy, const StepScalars<float>& c) {
    using E = PairEnc<St>;
    constexpr int EF = Fmt<St>::EF, EG = Fmt<St>::EG;
    const int k0 = iy * G.pitch + ix;
    // f first: rho, u and the f collision's coefficients need no g
    float2 f[Q];
    uint32_t wg[Q], wf[Q];
    pull_f(wf);
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = E::dec(wf[i], i);
    const bool wy = iy == 0 || iy == G.ny - 1;
    const Mask2 wall{wy || ix == 0 || ix == G.nx - 1, wy || ix + 1 == G.nx - 1};
    Macro<float2, true> m = macro_f_lane<float2, EF>(f, fy_prev, wall);
    // the relaxation coefficients now; the non-equilibrium parts are formed
    // again at the f update (same expressions, same bits), so they are not
    // held in registers across the g half of the step
    const CollCoef<float2> kc = collide_f_coef_lane<float2, EF>(f, m, c, nullptr);
    float2 g[Q];
    {
        pull_g(wg);
        const bool h0 = ix == 0, c0 = ix == G.nx - 1, c1 = ix + 1 == G.nx - 1;
        const float tw0 = (h0 ? t_hot_row : c.t_cold) * p2(EG), tw1 = c.t_cold * p2(EG);
        const float2 tw = make_float2(tw0, tw1);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const float2 v = E::dec(wg[i], Q + i);
            // wall columns: geq(T_wall, 0, 0) = w_i T_wall (geq_rest), both
            // halves in one packed multiply
            const float2 wv = lmul(lbc<float2>(float(WD(i))), tw);
            g[i].x = (h0 || c0) ? wv.x : v.x;
            g[i].y = c1 ? wv.y : v.y;
        }
    }
    m.t = sum_g<float2>(g);
    if (!NO_COLLIDE && ACC_NU) {
        const float t0 = m.t.x * p2(-EG), t1 = m.t.y * p2(-EG);
        if (ix + 1 == 1) acc_hot[iy] += fabs(double(t1) - double(t_at(2)));
        if (ix == G.nx - 2) acc_cold[iy] += fabs(double(t0) - double(t_at(G.nx - 3)));
        if (ix + 1 == G.nx - 2) acc_cold[iy] += fabs(double(t1) - double(t_at(G.nx - 3)));
    }
    // g collided and stored first (its registers free), then the f update;
    // stores: one word per plane, the draws in plane order 0..17
    uint32_t* __restrict__ d = reinterpret_cast<uint32_t*>(dst);
    const int P2 = int(G.plane >> 1), k2 = k0 >> 1;
    if (!NO_COLLIDE) {
        float2 qv[5];
        const float2 m15u2 = m15u2_lane<float2>(m.ux, m.uy);
#pragma unroll
        for (int p = 1; p <= 4; ++p) qv[p] = q_lane<float2>(p, m.ux, m.uy, m15u2);
        collide_g_lane<float2>(g, m.t, m.ux, m.uy, kc.nut, qv, c, nullptr);
    }
    // the pair's generator: planes 0..8 (f) draw from rng_f, 9..17 (g) from
    // the same stream nine draws on
    NodeRng rng_f(0u, 0, 0);
    if constexpr (E::SR) {
        rng_f = sr_pair_rng(c, G, ix, iy);
        NodeRng rng = rng_f;
        rng.skip<Q>();
#pragma unroll
        for (int q = 0; q < Q; ++q) d[(Q + q) * P2 + k2] = E::enc(g[q], Q + q, rng.next());
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) d[(Q + q) * P2 + k2] = E::enc(g[q], Q + q, 0u);
    }
    if (!NO_COLLIDE) {
        const CollF<float2> o = collide_f_parts_lane<float2, EF>(f, m, kc);
        const float2 fyv = collide_f_post_lane<float2, EF, EG>(f, o, m, c, m.t);
        *reinterpret_cast<float2*>(fy_out + k0) = fyv;
        if (WRITE_NUT) *reinterpret_cast<float2*>(nut + k0) = kc.nut;
    }
    if constexpr (E::SR) {
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q * P2 + k2] = E::enc(f[q], q, rng_f.next());
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) d[q * P2 + k2] = E::enc(f[q], q, 0u);
    }
}

// One reference step of the nodes (ix, iy), (ix + 1, iy) pulled from global
// memory (xpair_core after pull_f_x / pull_g_x).
template <class St, bool WRITE_NUT, bool ACC_NU, bool NO_COLLIDE = false>
__device__ __forceinline__ void fused_xpair(const St* __restrict__ src, St* __restrict__ dst,
                                            const float* fy_in, float* fy_out, float* __restrict__ nut,
                                            double* __restrict__ acc_hot, double* __restrict__ acc_cold,
                                            const Geom& G, int ix, int iy, const StepScalars<float>& c) {
    const int k0 = iy * G.pitch + ix;
    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
    xpair_core<St, WRITE_NUT, ACC_NU, NO_COLLIDE>(
        [&](uint32_t(&w)[Q]) { pull_f_x<St>(src, G, ix, iy, w); },
        [&](uint32_t(&w)[Q]) { pull_g_x<St>(src, G, ix, iy, w); },
        [&](int x) { return gather_t<St>(src, G, x, iy, c); }, dst, *reinterpret_cast<const float2*>(fy_in + k0),
        c.t_hot[gy], fy_out, nut, acc_hot, acc_cold, G, ix, iy, c);
}

// The node-pair step with the work of each pair split over two warps: an f
// warp (pull of f, macroscopic update, the collision's coefficients, the f
// update and stores) and a g warp (pull of g with the boundary conditions,
// T, the g collision and stores) exchange T and (u, v, nu_t) through shared
// memory at one named barrier per row.  Twice the warps of k_fused_x, each
// with about half its dependent chain: for grids too small to fill the GPU,
// where a step is one thread's latency.  The same expressions in the same
// order per node: bit-identical to k_fused_x.  CTA: 32 pairs x 2 rows x 2
// roles (warps 0-1: f of rows 0-1; warps 2-3: g).
__device__ __forceinline__ void named_bar_sync(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// The f half of a split node-pair step: pull of f, macroscopic update,
// relaxation coefficients, publish (u, v, nu_t), named barrier `bar_id`
// (64 threads: this warp and its g warp), read T, the f update and its
// stores (draws 0..8 of the pair).  act: the pair is in the grid (an
// inactive warp lane still takes the barrier).
template <class St, bool WRITE_NUT, class PF>
__device__ __forceinline__ void xpair_f_half(PF&& pull_f, float2* xu, float2* xv, float2* xnut, const float2* xt,
                                             int bar_id, bool act, St* __restrict__ dst, float2 fy_prev,
                                             float* fy_out, float* __restrict__ nut, const Geom& G, int ix, int iy,
                                             const StepScalars<float>& c) {
    using E = PairEnc<St>;
    constexpr int EF = Fmt<St>::EF, EG = Fmt<St>::EG;
    const int k0 = iy * G.pitch + ix, k2 = k0 >> 1;
    const int P2 = int(G.plane >> 1);
    uint32_t* __restrict__ d = reinterpret_cast<uint32_t*>(dst);
    float2 f[Q];
    Macro<float2, true> m{};
    CollCoef<float2> kc{};
    if (act) {
        uint32_t wf[Q];
        pull_f(wf);
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = E::dec(wf[i], i);
        const bool wy = iy == 0 || iy == G.ny - 1;
        const Mask2 wall{wy || ix == 0 || ix == G.nx - 1, wy || ix + 1 == G.nx - 1};
        m = macro_f_lane<float2, EF>(f, fy_prev, wall);
        kc = collide_f_coef_lane<float2, EF>(f, m, c, nullptr);
        *xu = m.ux;
        *xv = m.uy;
        *xnut = kc.nut;
    }
    named_bar_sync(bar_id, 64);
    if (act) {
        m.t = *xt;
        const CollF<float2> o = collide_f_parts_lane<float2, EF>(f, m, kc);
        const float2 fyv = collide_f_post_lane<float2, EF, EG>(f, o, m, c, m.t);
        *reinterpret_cast<float2*>(fy_out + k0) = fyv;
        if (WRITE_NUT) *reinterpret_cast<float2*>(nut + k0) = kc.nut;
        if constexpr (E::SR) {
            NodeRng rng = sr_pair_rng(c, G, ix, iy);
#pragma unroll
            for (int q = 0; q < Q; ++q) d[q * P2 + k2] = E::enc(f[q], q, rng.next());
        } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) d[q * P2 + k2] = E::enc(f[q], q, 0u);
        }
    }
}

// The g half: pull of g with the boundary conditions (t_hot_row: the hot
// wall's theta at the row's g source row), T, publish T, the Nusselt
// accumulation (t_at as in xpair_core), the named barrier, read
// (u, v, nu_t), the g collision and its stores (draws 9..17 of the pair).
template <class St, bool ACC_NU, class PG, class TAt>
__device__ __forceinline__ void xpair_g_half(PG&& pull_g, TAt&& t_at, float2* xt, const float2* xu,
                                             const float2* xv, const float2* xnut, int bar_id, bool act,
                                             St* __restrict__ dst, float t_hot_row, double* __restrict__ acc_hot,
                                             double* __restrict__ acc_cold, const Geom& G, int ix, int iy,
                                             const StepScalars<float>& c) {
    using E = PairEnc<St>;
    constexpr int EG = Fmt<St>::EG;
    const int k2 = (iy * G.pitch + ix) >> 1;
    const int P2 = int(G.plane >> 1);
    uint32_t* __restrict__ d = reinterpret_cast<uint32_t*>(dst);
    float2 g[Q], t{};
    if (act) {
        uint32_t wg[Q];
        pull_g(wg);
        const bool h0 = ix == 0, c0 = ix == G.nx - 1, c1 = ix + 1 == G.nx - 1;
        const float2 tw = make_float2((h0 ? t_hot_row : c.t_cold) * p2(EG), c.t_cold * p2(EG));
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const float2 v = E::dec(wg[i], Q + i);
            const float2 wv = lmul(lbc<float2>(float(WD(i))), tw);
            g[i].x = (h0 || c0) ? wv.x : v.x;
            g[i].y = c1 ? wv.y : v.y;
        }
        t = sum_g<float2>(g);
        *xt = t;
        if (ACC_NU) {
            const float t0 = t.x * p2(-EG), t1 = t.y * p2(-EG);
            if (ix + 1 == 1) acc_hot[iy] += fabs(double(t1) - double(t_at(2)));
            if (ix == G.nx - 2) acc_cold[iy] += fabs(double(t0) - double(t_at(G.nx - 3)));
            if (ix + 1 == G.nx - 2) acc_cold[iy] += fabs(double(t1) - double(t_at(G.nx - 3)));
        }
    }
    named_bar_sync(bar_id, 64);
    if (act) {
        const float2 u = *xu, v = *xv, nt = *xnut;
        float2 qv[5];
        const float2 m15u2 = m15u2_lane<float2>(u, v);
#pragma unroll
        for (int p = 1; p <= 4; ++p) qv[p] = q_lane<float2>(p, u, v, m15u2);
        collide_g_lane<float2>(g, t, u, v, nt, qv, c, nullptr);
        if constexpr (E::SR) {
            NodeRng rng = sr_pair_rng(c, G, ix, iy);
            rng.skip<Q>();
#pragma unroll
            for (int q = 0; q < Q; ++q) d[(Q + q) * P2 + k2] = E::enc(g[q], Q + q, rng.next());
        } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) d[(Q + q) * P2 + k2] = E::enc(g[q], Q + q, 0u);
        }
    }
}

template <class St, bool WRITE_NUT, bool ACC_NU>
__global__ void __launch_bounds__(128) k_fused_xs(const St* __restrict__ src, St* __restrict__ dst,
                                                  float* __restrict__ fy, float* __restrict__ nut,
                                                  double* __restrict__ acc_hot, double* __restrict__ acc_cold, Geom G,
                                                  StepScalars<float> c) {
    __shared__ float2 sh_t[2][32], sh_u[2][32], sh_v[2][32], sh_nut[2][32];
    pdl_wait();
    pdl_trigger();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int r = w & 1, role = w >> 1;
    const int ix = 2 * (blockIdx.x * 32 + lane);
    const int iy = blockIdx.y * 2 + r;
    const bool act = ix < G.nx && iy < G.ny;
    if (role == 0) {
        const float2 fy_prev = act ? *reinterpret_cast<const float2*>(fy + iy * G.pitch + ix) : make_float2(0.f, 0.f);
        xpair_f_half<St, WRITE_NUT>([&](uint32_t(&wf)[Q]) { pull_f_x<St>(src, G, ix, iy, wf); }, &sh_u[r][lane],
                                    &sh_v[r][lane], &sh_nut[r][lane], &sh_t[r][lane], 1 + r, act, dst, fy_prev, fy,
                                    nut, G, ix, iy, c);
    } else {
        const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
        const float th = (act && ix == 0) ? c.t_hot[gy] : 0.0f;
        xpair_g_half<St, ACC_NU>([&](uint32_t(&wg)[Q]) { pull_g_x<St>(src, G, ix, iy, wg); },
                                 [&](int x) { return gather_t<St>(src, G, x, iy, c); }, &sh_t[r][lane], &sh_u[r][lane],
                                 &sh_v[r][lane], &sh_nut[r][lane], 1 + r, act, dst, th, acc_hot, acc_cold, G, ix,
                                 iy, c);
    }
}
// The single-cavity step on node pairs: 32 x BY threads cover 64 columns x
// BY rows.
template <class St, bool WRITE_NUT, bool ACC_NU, bool NO_COLLIDE>
__global__ void __launch_bounds__(256) k_fused_x(const St* __restrict__ src, St* __restrict__ dst,
                                                 float* __restrict__ fy, float* __restrict__ nut,
                                                 double* __restrict__ acc_hot, double* __restrict__ acc_cold, Geom G,
                                                 StepScalars<float> c) {
    pdl_wait();
    pdl_trigger();
    const int ix = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    fused_xpair<St, WRITE_NUT, ACC_NU, NO_COLLIDE>(src, dst, fy, fy, nut, acc_hot, acc_cold, G, ix, iy, c);
}

}  // namespace cav
