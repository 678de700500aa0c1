// kernels.cuh -- device kernels of the uniform cavity step.
//
// Two representations of one state (see cavity.cu):
//   REF  the reference's own: post-stream f, g plus rho, u, T fields
//        (what CavitySolver holds between step() calls, src/uniform/solver.rs:35-104);
//   PC   post-collision f*, g* of the last collide (the form the fused
//        kernel streams from).
// k_fused advances PC -> PC by one reference step in one pass: pull-stream
// with bounce-back for f, thermal boundary conditions for g, macroscopic
// update with the Guo half-force correction, no-slip, then the collision of
// the next step.  This is the reference order collide -> stream -> BC ->
// macroscopic -> no-slip (solver.rs:279-293) rotated by one phase.
#pragma once

#include "lattice.cuh"

namespace cav {

template <class St>
__device__ __forceinline__ typename Fmt<St>::A ldp(const St* __restrict__ buf, const Geom& G, int q, int iy,
                                                  int ix) {
    return Fmt<St>::load(buf[(long long)q * G.plane + (long long)iy * G.pitch + ix], q);
}
template <class St>
__device__ __forceinline__ void stp(St* __restrict__ buf, const Geom& G, int q, int iy, int ix,
                                    typename Fmt<St>::A v, uint32_t r = RN_BITS) {
    buf[(long long)q * G.plane + (long long)iy * G.pitch + ix] = Fmt<St>::store(v, q, r);
}

// Stochastic rounding draws.  The two x-adjacent nodes (2j, iy) and
// (2j + 1, iy) share one generator, seeded by the seed, the step and the pair
// index iy * ceil(nx / 2) + j (NodeRng), and one 32-bit draw r per plane,
// planes 0..17 in order: node 2j takes its dither from r's high bits, node
// 2j + 1 from its low bits (binary16: r[31:19] / r[15:3]; bfloat16:
// r[31:16] / r[15:0]; 16-bit fixed point: r[31:16] / r[15:0]).  The x-pair
// kernels round a plane of both nodes with one cvt.rs (the draw rotated so
// that the hardware takes those bits); the one-node kernels compute the
// pair's draws and use their half, so every kernel gives a node the same bits.
__device__ __forceinline__ uint32_t sr_bits_f16(uint32_t r) { return __funnelshift_r(r, r, 19); }
__device__ __forceinline__ uint32_t sr_bits_bf16(uint32_t r) { return __funnelshift_r(r, r, 16); }
__host__ __device__ __forceinline__ uint32_t sr_bits_fx(uint32_t r, int half) {
    return half ? r << 16 : r & 0xffff0000u;
}
// The software rounding's draw for node half h (h16_enc / bf16_store take
// their dither from the top bits of the word they are given).
__host__ __device__ __forceinline__ uint32_t sr_bits_sw(uint32_t r, int half) { return half ? r << 16 : r; }
template <class A>
__device__ __forceinline__ NodeRng sr_pair_rng(const StepScalars<A>& c, const Geom& G, int ix, int iy) {
    const long long step = c.step_dev ? *c.step_dev + c.step : c.step;
    return NodeRng(c.sr_seed, step, (long long)iy * ((G.nx + 1) >> 1) + (ix >> 1));
}

// Rounds x (in the plane's stored units) to the 16 bits of node half h of
// plane q, from the pair's draw r for that plane.
template <class St, bool LANE>
__device__ __forceinline__ St store_sr_pairdraw(typename Fmt<St>::A x, int q, uint32_t r, int h) {
    if constexpr (Fmt<St>::HW_SR_F) {
        const bool hw = q < Q || Fmt<St>::HW_SR_G;
        if (hw) {
            const float s = LANE ? 1.0f : (q < Q ? p2(Fmt<St>::EF) : p2(Fmt<St>::EG));
            const float v = x * s;
            uint32_t d;
            if constexpr (Fmt<St>::KIND_BF16)
                asm("cvt.rs.bf16x2.f32 %0, %1, %1, %2;" : "=r"(d) : "f"(v), "r"(sr_bits_bf16(r)));
            else
                asm("cvt.rs.f16x2.f32 %0, %1, %1, %2;" : "=r"(d) : "f"(v), "r"(sr_bits_f16(r)));
            St o;
            o.bits = (unsigned short)(h ? d >> 16 : d & 0xffffu);
            return o;
        }
        return LANE ? Fmt<St>::lstore_sr(x, q, sr_bits_fx(r, h)) : Fmt<St>::store_sr(x, q, sr_bits_fx(r, h));
    } else {
        const uint32_t b = (Fmt<St>::FIXED_G && q >= Q) ? sr_bits_fx(r, h) : sr_bits_sw(r, h);
        return LANE ? Fmt<St>::lstore_sr(x, q, b) : Fmt<St>::store_sr(x, q, b);
    }
}

// Stores the 18 populations of one node (32-bit offsets, like pull_node);
// the stochastically rounded formats draw their random bits from the node
// pair's (seed, step, pair) stream (sr_pair_rng).
// LANE: f and g in lane units (Fmt::lstore).
template <class St, bool LANE = false>
__device__ __forceinline__ void store_node(St* __restrict__ dst, const Geom& G, int iy, int ix,
                                           const typename Fmt<St>::A (&f)[Q], const typename Fmt<St>::A (&g)[Q],
                                           const StepScalars<typename Fmt<St>::A>& c) {
    const int P = int(G.plane);
    const int k = iy * G.pitch + ix;
    if constexpr (Fmt<St>::SR) {
        NodeRng rng = sr_pair_rng(c, G, ix, iy);
        const int h = ix & 1;
#pragma unroll
        for (int q = 0; q < NPLANES; ++q) {
            const uint32_t r = rng.next();
            dst[q * P + k] = store_sr_pairdraw<St, LANE>(q < Q ? f[q] : g[q - Q], q, r, h);
        }
    } else {
#pragma unroll
        for (int q = 0; q < NPLANES; ++q) {
            const auto x = q < Q ? f[q] : g[q - Q];
            dst[q * P + k] = LANE ? Fmt<St>::lstore(x, q, RN_BITS) : Fmt<St>::store(x, q, RN_BITS);
        }
    }
}

// Stores the 9 planes Q0..Q0+8 (Q0 = 0: f, Q0 = 9: g) of one node from lane
// units, drawing the same random bits per plane as store_node.
template <class St, int Q0>
__device__ __forceinline__ void store_planes(St* __restrict__ dst, const Geom& G, int iy, int ix,
                                             const typename Fmt<St>::A (&v)[Q],
                                             const StepScalars<typename Fmt<St>::A>& c) {
    const int P = int(G.plane);
    const int k = iy * G.pitch + ix;
    if constexpr (Fmt<St>::SR) {
        NodeRng rng = sr_pair_rng(c, G, ix, iy);
#pragma unroll
        for (int j = 0; j < Q0; ++j) rng.next();  // the draws of planes 0..Q0-1
        const int h = ix & 1;
#pragma unroll
        for (int q = Q0; q < Q0 + Q; ++q) dst[q * P + k] = store_sr_pairdraw<St, true>(v[q - Q0], q, rng.next(), h);
    } else {
#pragma unroll
        for (int q = Q0; q < Q0 + Q; ++q) dst[q * P + k] = Fmt<St>::lstore(v[q - Q0], q, RN_BITS);
    }
}

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialisation attribute may start while its predecessor finishes;
// it must not touch global memory before pdl_wait() (which returns once the
// predecessor grid has completed and its writes are visible; a no-op without
// the attribute).  pdl_trigger() lets the successor launch early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

static __global__ void k_set_step(long long* p, long long v) { *p = v; }
static __global__ void k_add_step(long long* p, long long d) { *p += d; }

// Pull-stream of one node from a PC buffer (stream, solver.rs:838-913) fused
// with the thermal boundary conditions (solver.rs:951-988):
//  f_i(x) = f*_i(x - c_i) in the domain, else f*_opp(i)(x) (bounce-back);
//  g on x = 0 / x = nx-1 is geq(T_wall, 0, 0); rows y = 0 / ny-1 take the
//  post-stream g of rows 1 / ny-2 (corners: the vertical wall value of that
//  row, as the vertical loop runs first).  Every other g source is inside
//  the domain, so the reference's "keep g at out-of-domain sources" value
//  is always overwritten and never needed here.
// LANE: values in lane units (Fmt::lload).
// CHANNEL: the plane-channel variant (periodic in y, bounce-back walls at
// x = 0 and nx - 1), see k_fused.
template <class St, bool LANE = false, bool CHANNEL = false>
__device__ __forceinline__ void pull_f(const St* __restrict__ src, const Geom& G, int ix, int iy,
                                       typename Fmt<St>::A (&f)[Q]) {
    // 32-bit element offsets: 18 * plane < 2^31 is checked at allocation.
    const int P = int(G.plane), W = G.pitch;
    const int k = iy * W + ix;
    const bool xm = ix > 0, xp = ix < G.nx - 1, ym = iy > 0, yp = iy < G.ny - 1;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = CX(i), cy = CY(i);
        if constexpr (CHANNEL) {
            const int sy = cy > 0 ? (ym ? iy - 1 : G.ny - 1) : (cy < 0 ? (yp ? iy + 1 : 0) : iy);
            const bool ok = cx > 0 ? xm : (cx < 0 ? xp : true);
            const int idx = ok ? i * P + sy * W + ix - cx : OPP(i) * P + k;
            f[i] = LANE ? Fmt<St>::lload(src[idx], i) : Fmt<St>::load(src[idx], i);
        } else {
            const bool ok = (cx > 0 ? xm : (cx < 0 ? xp : true)) && (cy > 0 ? ym : (cy < 0 ? yp : true));
            const int idx = ok ? i * P + k - cx - cy * W : OPP(i) * P + k;  // else bounce-back
            f[i] = LANE ? Fmt<St>::lload(src[idx], i) : Fmt<St>::load(src[idx], i);
        }
    }
}

// g of the plane channel: periodic in y; an out-of-domain x source keeps the
// node's own value (stream(), src/uniform/solver.rs:879-881); no thermal
// boundary conditions.
template <class St, bool LANE = false>
__device__ __forceinline__ void pull_g_channel(const St* __restrict__ src, const Geom& G, int ix, int iy,
                                               typename Fmt<St>::A (&g)[Q]) {
    const int P = int(G.plane), W = G.pitch;
    const int k = iy * W + ix;
    const bool xm = ix > 0, xp = ix < G.nx - 1, ym = iy > 0, yp = iy < G.ny - 1;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int cx = CX(i), cy = CY(i);
        const int sy = cy > 0 ? (ym ? iy - 1 : G.ny - 1) : (cy < 0 ? (yp ? iy + 1 : 0) : iy);
        const bool ok = cx > 0 ? xm : (cx < 0 ? xp : true);
        const int idx = (Q + i) * P + (ok ? sy * W + ix - cx : k);
        g[i] = LANE ? Fmt<St>::lload(src[idx], Q + i) : Fmt<St>::load(src[idx], Q + i);
    }
}

template <class St, bool LANE = false>
__device__ __forceinline__ void pull_g(const St* __restrict__ src, const Geom& G, int ix, int iy,
                                       const StepScalars<typename Fmt<St>::A>& c, typename Fmt<St>::A (&g)[Q]) {
    using A = typename Fmt<St>::A;
    const int P = int(G.plane), W = G.pitch;
    const int k = iy * W + ix;
    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
    const bool wall_col = (ix == 0) || (ix == G.nx - 1);
    // (w_i T scaled by a power of two is w_i T rounded, scaled)
    const A tw = (ix == 0 ? c.t_hot[gy] : c.t_cold) * A(LANE ? p2(Fmt<St>::EG) : 1.0f);
    const int kg = wall_col ? k : gy * W + ix;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        // wall columns read their own node (a valid address) and discard it
        const int idx = (Q + i) * P + (wall_col ? kg : kg - CX(i) - CY(i) * W);
        const A v = LANE ? Fmt<St>::lload(src[idx], Q + i) : Fmt<St>::load(src[idx], Q + i);
        g[i] = wall_col ? geq_rest<A>(i, tw, c.geq_order) : v;
    }
}

template <class St, bool LANE = false>
__device__ __forceinline__ void pull_node(const St* __restrict__ src, const Geom& G, int ix, int iy,
                                          const StepScalars<typename Fmt<St>::A>& c,
                                          typename Fmt<St>::A (&f)[Q], typename Fmt<St>::A (&g)[Q]) {
    pull_f<St, LANE>(src, G, ix, iy, f);
    pull_g<St, LANE>(src, G, ix, iy, c, g);
}

// Temperature of node (ix, iy) of the streamed state, gathered from a PC
// buffer (used for the per-step Nusselt accumulation).
template <class St>
__device__ __forceinline__ typename Fmt<St>::A gather_t(const St* __restrict__ src, const Geom& G, int ix, int iy,
                                                       const StepScalars<typename Fmt<St>::A>& c) {
    using A = typename Fmt<St>::A;
    const int gy = iy == 0 ? 1 : (iy == G.ny - 1 ? G.ny - 2 : iy);
    A g[Q];
    if (ix == 0) {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = geq_rest<A>(i, c.t_hot[gy], c.geq_order);
    } else if (ix == G.nx - 1) {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = geq_rest<A>(i, c.t_cold, c.geq_order);
    } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = ldp(src, G, Q + i, gy - CY(i), ix - CX(i));
    }
    return sum_g<A>(g);
}

__device__ __forceinline__ bool is_wall(const Geom& G, int ix, int iy) {
    return ix == 0 || ix == G.nx - 1 || iy == 0 || iy == G.ny - 1;
}

// One full reference step, PC(src) -> PC(dst).
//  WRITE_NUT   store nu_t of this collision (only the last step of a call
//              needs it: the reference reads nu_t after step()).
//  ACC_NU      add |T(1)-T(2)| and |T(nx-2)-T(nx-3)| of the streamed state
//              to the per-row FP64 accumulators (nusselt_hot/cold, post.rs:68-111).
//  NO_COLLIDE  identity collision: checks the streaming / bounce-back /
//              boundary index maps bit for bit.
// fy_in / fy_out: the Guo force of the previous / this collision (the same
// array in the production step, where every node reads then rewrites its own
// entry; separate arrays when states are kept, as in the adjoint's
// recomputation).
// Everything of the step after the pull (f, g streamed into the node):
// macroscopic, no-slip, the Nusselt accumulation (t_at(x) gives T of the
// streamed state at column x of the same row), the collision, the stores.
// Shared by the global-memory pull (fused_node_io) and the shared-memory
// tiles (tile.cuh), so both give the same bits.  f and g arrive in lane units
// (pull with LANE); t_at returns T unscaled.
template <class St, bool WRITE_NUT, bool ACC_NU, bool NO_COLLIDE, class TAt, bool CHANNEL = false>
__device__ __forceinline__ void fused_core(typename Fmt<St>::A (&f)[Q], typename Fmt<St>::A (&g)[Q],
                                           St* __restrict__ dst, const typename Fmt<St>::A* fy_in,
                                           typename Fmt<St>::A* fy_out, typename Fmt<St>::A* __restrict__ nut,
                                           double* __restrict__ acc_hot, double* __restrict__ acc_cold,
                                           const Geom& G, int ix, int iy, const StepScalars<typename Fmt<St>::A>& c,
                                           TAt&& t_at) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    constexpr int EF = Fmt<St>::EF, EG = Fmt<St>::EG;
    const int k = iy * G.pitch + ix;
    const bool wall = !CHANNEL && is_wall(G, ix, iy);
    Macro<A, SH> m;
    if constexpr (SH) {
        m = macro_f_lane<A, EF>(f, fy_in[k], wall);
        m.t = sum_g<A>(g);
    } else {
        m = macro_node<A, SH>(f, g, fy_in[k], wall);
    }
    if (ACC_NU) {
        const A t = m.t * A(p2(-EG));
        if (ix == 1) {
            A t2 = t_at(2);
            acc_hot[iy] += fabs(double(t) - double(t2));
        }
        if (ix == G.nx - 2) {
            A t0 = t_at(G.nx - 3);
            acc_cold[iy] += fabs(double(t) - double(t0));
        }
    }
    A fyv, nutv;
    if (CHANNEL) {
        // body force rho beta along +y (the temperature factor taken as 1)
        if constexpr (SH) {
            const CollF<A> o = collide_f_pre_lane<A, EF>(f, m, c, nullptr);
            nutv = o.nut;
            fyv = collide_f_post_lane<A, EF, EG>(f, o, m, c, A(p2(EG)));
            collide_g_lane<A>(g, m.t, m.ux, m.uy, o.nut, o.q, c, nullptr);
        } else {
            const CollF<A> o = collide_f_pre<A, SH>(f, m, c);
            nutv = o.nut;
            fyv = collide_f_post<A, SH>(f, o, m, c, A(1.0));
            collide_g<A, SH>(g, m.t, m.ux, m.uy, o.nut, c);
        }
        fy_out[k] = fyv;
        if (WRITE_NUT) nut[k] = nutv;
    } else if (!NO_COLLIDE) {
        if constexpr (SH)
            collide_node_lane<A, EF, EG>(f, g, m, c, fyv, nutv);
        else
            collide_node<A, SH>(f, g, m, c, fyv, nutv);
        fy_out[k] = fyv;
        if (WRITE_NUT) nut[k] = nutv;
    }
    store_node<St, true>(dst, G, iy, ix, f, g, c);
}

template <class St, bool WRITE_NUT, bool ACC_NU, bool NO_COLLIDE, bool CHANNEL = false>
__device__ __forceinline__ void fused_node_io(const St* __restrict__ src, St* __restrict__ dst,
                                              const typename Fmt<St>::A* fy_in, typename Fmt<St>::A* fy_out,
                                              typename Fmt<St>::A* __restrict__ nut, double* __restrict__ acc_hot,
                                              double* __restrict__ acc_cold, const Geom& G, int ix, int iy,
                                              const StepScalars<typename Fmt<St>::A>& c) {
    using A = typename Fmt<St>::A;
    A f[Q], g[Q];
    if constexpr (CHANNEL) {
        pull_f<St, true, true>(src, G, ix, iy, f);
        pull_g_channel<St, true>(src, G, ix, iy, g);
    } else {
        pull_node<St, true>(src, G, ix, iy, c, f, g);
    }
    auto t_at = [&](int x) { return gather_t<St>(src, G, x, iy, c); };
    fused_core<St, WRITE_NUT, ACC_NU && !CHANNEL, NO_COLLIDE, decltype(t_at)&, CHANNEL>(
        f, g, dst, fy_in, fy_out, nut, acc_hot, acc_cold, G, ix, iy, c, t_at);
}

template <class St, bool WRITE_NUT, bool ACC_NU, bool NO_COLLIDE, bool CHANNEL = false>
__device__ __forceinline__ void fused_node(const St* __restrict__ src, St* __restrict__ dst,
                                           typename Fmt<St>::A* fy, typename Fmt<St>::A* __restrict__ nut,
                                           double* __restrict__ acc_hot, double* __restrict__ acc_cold,
                                           const Geom& G, int ix, int iy, const StepScalars<typename Fmt<St>::A>& c) {
    fused_node_io<St, WRITE_NUT, ACC_NU, NO_COLLIDE, CHANNEL>(src, dst, fy, fy, nut, acc_hot, acc_cold, G, ix, iy,
                                                              c);
}

// Two nodes of one column, (ix, iy) and (ix, iy + 1), in one thread: the
// pulls, boundary conditions and stores per node, the macroscopic update and
// the collision of both on packed FP32x2 lanes (one add / mul / fma
// instruction for the two nodes).  The lane arithmetic rounds every operation
// once, so each node gets the bits fused_node gives it.  hi: whether
// (ix, iy + 1) is in the grid (else the upper lane recomputes (ix, iy) and
// is not stored).
template <class St, bool WRITE_NUT, bool ACC_NU>
__device__ __forceinline__ void fused_pair(const St* __restrict__ src, St* __restrict__ dst, float* fy,
                                           float* __restrict__ nut, double* __restrict__ acc_hot,
                                           double* __restrict__ acc_cold, const Geom& G, int ix, int iy, bool hi,
                                           const StepScalars<float>& c) {
    static_assert(Fmt<St>::SHIFT, "the two-node lanes carry the FP32 arithmetic");
    constexpr int EF = Fmt<St>::EF, EG = Fmt<St>::EG;
    const int iy1 = hi ? iy + 1 : iy;
    // f first: rho, u and the f collision's coefficients need no g, so the
    // g populations are pulled only once those are formed (fewer values
    // live at once: more resident warps)
    float fa[Q], ga[Q], fb[Q], gb[Q];
    pull_f<St, true>(src, G, ix, iy, fa);
    pull_f<St, true>(src, G, ix, iy1, fb);
    float2 f[Q], g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = make_float2(fa[i], fb[i]);
    const int k0 = iy * G.pitch + ix, k1 = iy1 * G.pitch + ix;
    Macro<float2, true> m = macro_f_lane<float2, EF>(f, make_float2(fy[k0], fy[k1]),
                                                     Mask2{is_wall(G, ix, iy), is_wall(G, ix, iy1)});
    const CollF<float2> o = collide_f_pre_lane<float2, EF>(f, m, c, nullptr);
    pull_g<St, true>(src, G, ix, iy, c, ga);
    pull_g<St, true>(src, G, ix, iy1, c, gb);
#pragma unroll
    for (int i = 0; i < Q; ++i) g[i] = make_float2(ga[i], gb[i]);
    m.t = sum_g<float2>(g);
    if (ACC_NU) {
        const float ta = m.t.x * p2(-EG), tb = m.t.y * p2(-EG);
        if (ix == 1) {
            acc_hot[iy] += fabs(double(ta) - double(gather_t<St>(src, G, 2, iy, c)));
            if (hi) acc_hot[iy1] += fabs(double(tb) - double(gather_t<St>(src, G, 2, iy1, c)));
        }
        if (ix == G.nx - 2) {
            acc_cold[iy] += fabs(double(ta) - double(gather_t<St>(src, G, G.nx - 3, iy, c)));
            if (hi) acc_cold[iy1] += fabs(double(tb) - double(gather_t<St>(src, G, G.nx - 3, iy1, c)));
        }
    }
    // then g (collided and stored), then the f update
    collide_g_lane<float2>(g, m.t, m.ux, m.uy, o.nut, o.q, c, nullptr);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        ga[i] = g[i].x;
        gb[i] = g[i].y;
    }
    store_planes<St, Q>(dst, G, iy, ix, ga, c);
    if (hi) store_planes<St, Q>(dst, G, iy1, ix, gb, c);
    const float2 fyv = collide_f_post_lane<float2, EF, EG>(f, o, m, c, m.t);
    fy[k0] = fyv.x;
    if (WRITE_NUT) nut[k0] = o.nut.x;
    if (hi) {
        fy[k1] = fyv.y;
        if (WRITE_NUT) nut[k1] = o.nut.y;
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        fa[i] = f[i].x;
        fb[i] = f[i].y;
    }
    store_planes<St, 0>(dst, G, iy, ix, fa, c);
    if (hi) store_planes<St, 0>(dst, G, iy1, ix, fb, c);
}

// One full reference step, PC(src) -> PC(dst), one thread per node.
//  WRITE_NUT   store nu_t of this collision (only the last step of a call
//              needs it: the reference reads nu_t after step()).
//  ACC_NU      add |T(1)-T(2)| and |T(nx-2)-T(nx-3)| of the streamed state
//              to the per-row FP64 accumulators (nusselt_hot/cold, post.rs:68-111).
//  NO_COLLIDE  identity collision: checks the streaming / bounce-back /
//              boundary index maps bit for bit.
//  CHANNEL     the same node body on a plane channel instead of the cavity:
//              periodic in y, bounce-back walls at x = 0 and nx - 1 with no
//              wall-velocity override and no thermal boundary conditions,
//              body force rho beta along +y (the reference's Poiseuille
//              test of the TRT + Guo collision, src/uniform/tests.rs:246-376,
//              turned by 90 degrees).
template <class St, bool WRITE_NUT, bool ACC_NU, bool NO_COLLIDE, bool CHANNEL = false>
__global__ void __launch_bounds__(256) k_fused(const St* __restrict__ src, St* __restrict__ dst,
                                               typename Fmt<St>::A* __restrict__ fy,
                                               typename Fmt<St>::A* __restrict__ nut, double* __restrict__ acc_hot,
                                               double* __restrict__ acc_cold, Geom G,
                                               StepScalars<typename Fmt<St>::A> c) {
    pdl_wait();
    pdl_trigger();
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    fused_node<St, WRITE_NUT, ACC_NU, NO_COLLIDE, CHANNEL>(src, dst, fy, nut, acc_hot, acc_cold, G, ix, iy, c);
}

// collide(step) on a REF state (populations + fields), writing PC to dst.
// This is the reference's first phase of step() when the state comes from
// new()/init_from_fields() or from the debug phases.
template <class St>
__global__ void __launch_bounds__(256) k_collide_ref(const St* __restrict__ src, St* __restrict__ dst,
                                                     const typename Fmt<St>::A* __restrict__ rho,
                                                     const typename Fmt<St>::A* __restrict__ ux,
                                                     const typename Fmt<St>::A* __restrict__ uy,
                                                     const typename Fmt<St>::A* __restrict__ tt,
                                                     typename Fmt<St>::A* __restrict__ fy,
                                                     typename Fmt<St>::A* __restrict__ nut, Geom G,
                                                     StepScalars<typename Fmt<St>::A> c,
                                                     const typename Fmt<St>::A* __restrict__ nut_pre = nullptr,
                                                     const typename Fmt<St>::A* __restrict__ at_pre = nullptr) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.pitch + ix;
    A f[Q], g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        f[i] = ldp(src, G, i, iy, ix);
        g[i] = ldp(src, G, Q + i, iy, ix);
    }
    Macro<A, SH> m;
    m.rho = rho[k];
    m.drho = m.rho - A(1.0);
    m.inv_rho = A(1.0) / m.rho;
    m.ux = ux[k];
    m.uy = uy[k];
    m.t = tt[k];
    A fyv, nutv;
    collide_node<A, SH>(f, g, m, c, fyv, nutv, nut_pre ? nut_pre + k : nullptr, at_pre ? at_pre + k : nullptr);
    fy[k] = fyv;
    nut[k] = nutv;
    store_node<St>(dst, G, iy, ix, f, g, c);
}

// PC(src) -> REF(dst): stream + thermal BC + macroscopic + no-slip, without
// the next collision.  Produces the reference's observable state.
template <class St, bool CHANNEL = false>
__global__ void __launch_bounds__(256) k_materialize(const St* __restrict__ src, St* __restrict__ dst,
                                                     const typename Fmt<St>::A* __restrict__ fy,
                                                     typename Fmt<St>::A* __restrict__ rho,
                                                     typename Fmt<St>::A* __restrict__ ux,
                                                     typename Fmt<St>::A* __restrict__ uy,
                                                     typename Fmt<St>::A* __restrict__ tt, Geom G,
                                                     StepScalars<typename Fmt<St>::A> c) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.pitch + ix;
    A f[Q], g[Q];
    if constexpr (CHANNEL) {
        pull_f<St, false, true>(src, G, ix, iy, f);
        pull_g_channel<St>(src, G, ix, iy, g);
    } else {
        pull_node<St>(src, G, ix, iy, c, f, g);
    }
    Macro<A, SH> m = macro_node<A, SH>(f, g, fy[k], !CHANNEL && is_wall(G, ix, iy));
    rho[k] = m.rho;
    ux[k] = m.ux;
    uy[k] = m.uy;
    tt[k] = m.t;
#pragma unroll
    for (int i = 0; i < Q; ++i) stp(dst, G, i, iy, ix, f[i]);
#pragma unroll
    for (int i = 0; i < Q; ++i) stp(dst, G, Q + i, iy, ix, g[i]);
}

// init_from_fields (src/uniform/solver.rs:232-262) on the device: fields
// from dense FP64 arrays (k = iy*nx + ix), populations their equilibria, then
// no-slip on the stored velocity (the populations keep the given u).
// feq_full / geq_full in FP64 with explicit round-to-nearest operations (no
// contraction in any translation unit): the host's init_from_fields
// arithmetic bit for bit, in the reference's expression order.
__device__ __forceinline__ double eq_rn(int i, double a, double ux, double uy, int order) {
    const double cs2 = CS2;
    const double eu = __dadd_rn(__dmul_rn(double(CX(i)), ux), __dmul_rn(double(CY(i)), uy));
    double br = __dadd_rn(1.0, __ddiv_rn(eu, cs2));
    if (order != 1) {
        const double u2 = __dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy));
        br = __dadd_rn(br, __ddiv_rn(__dmul_rn(eu, eu), __dmul_rn(__dmul_rn(2.0, cs2), cs2)));
        br = __dsub_rn(br, __ddiv_rn(u2, __dmul_rn(2.0, cs2)));
    }
    return __dmul_rn(__dmul_rn(WD(i), a), br);
}

template <class St>
__global__ void __launch_bounds__(256) k_init_eq(const double* __restrict__ r, const double* __restrict__ u,
                                                 const double* __restrict__ v, const double* __restrict__ t,
                                                 St* __restrict__ dst, typename Fmt<St>::A* __restrict__ rho,
                                                 typename Fmt<St>::A* __restrict__ ux,
                                                 typename Fmt<St>::A* __restrict__ uy,
                                                 typename Fmt<St>::A* __restrict__ tt, Geom G, int geq_order) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const int kd = iy * G.nx + ix;
    const long long k = (long long)iy * G.pitch + ix;
    const double rk = r[kd], uk = u[kd], vk = v[kd], tk = t[kd];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        double fv = eq_rn(i, rk, uk, vk, 2);
        if (SH) fv = __dsub_rn(fv, WD(i));
        stp(dst, G, i, iy, ix, A(fv));
        stp(dst, G, Q + i, iy, ix, A(eq_rn(i, tk, uk, vk, geq_order)));
    }
    const bool wall = is_wall(G, ix, iy);
    rho[k] = A(rk);
    ux[k] = wall ? A(0.0) : A(uk);
    uy[k] = wall ? A(0.0) : A(vk);
    tt[k] = A(tk);
}

// A pitched field of the arithmetic type to a dense FP64 array (k = iy*nx + ix).
template <class A>
__global__ void __launch_bounds__(256) k_field_to_dense(const A* __restrict__ src, double* __restrict__ dst, Geom G) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    dst[iy * G.nx + ix] = double(src[(long long)iy * G.pitch + ix]);
}

// Nusselt accumulation of the streamed state of a PC buffer (one thread per row).
template <class St>
__global__ void k_acc_nu_pc(const St* __restrict__ src, double* __restrict__ acc_hot, double* __restrict__ acc_cold,
                            Geom G, StepScalars<typename Fmt<St>::A> c) {
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    if (iy >= G.ny) return;
    double t1 = gather_t<St>(src, G, 1, iy, c), t2 = gather_t<St>(src, G, 2, iy, c);
    double tc2 = gather_t<St>(src, G, G.nx - 2, iy, c), tc3 = gather_t<St>(src, G, G.nx - 3, iy, c);
    acc_hot[iy] += fabs(t1 - t2);
    acc_cold[iy] += fabs(tc2 - tc3);
}

// Same on a REF state (temperature field).
template <class A>
__global__ void k_acc_nu_ref(const A* __restrict__ tt, double* __restrict__ acc_hot, double* __restrict__ acc_cold,
                             Geom G) {
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    if (iy >= G.ny) return;
    const long long r = (long long)iy * G.pitch;
    acc_hot[iy] += fabs(double(tt[r + 1]) - double(tt[r + 2]));
    acc_cold[iy] += fabs(double(tt[r + G.nx - 2]) - double(tt[r + G.nx - 3]));
}

// ---------------------------------------------------------------------------
// Debug phases on a REF state (the pub(crate) methods of the reference,
// called one at a time by src/uniform/tests.rs:154-169).
// ---------------------------------------------------------------------------
// collide(step), src/uniform/solver.rs:421-540, in place.
template <class St>
__global__ void k_dbg_collide(St* __restrict__ pop, const typename Fmt<St>::A* __restrict__ rho,
                              const typename Fmt<St>::A* __restrict__ ux, const typename Fmt<St>::A* __restrict__ uy,
                              const typename Fmt<St>::A* __restrict__ tt, typename Fmt<St>::A* __restrict__ fy,
                              typename Fmt<St>::A* __restrict__ nut, Geom G, StepScalars<typename Fmt<St>::A> c) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.pitch + ix;
    A f[Q], g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        f[i] = ldp(pop, G, i, iy, ix);
        g[i] = ldp(pop, G, Q + i, iy, ix);
    }
    Macro<A, SH> m;
    m.rho = rho[k];
    m.drho = m.rho - A(1.0);
    m.inv_rho = A(1.0) / m.rho;
    m.ux = ux[k];
    m.uy = uy[k];
    m.t = tt[k];
    A fyv, nutv;
    collide_node<A, SH>(f, g, m, c, fyv, nutv);
    fy[k] = fyv;
    nut[k] = nutv;
    store_node<St>(pop, G, iy, ix, f, g, c);
}

// stream(), src/uniform/solver.rs:838-913: pull, bounce-back for f, g kept
// at out-of-domain sources.
template <class St>
__global__ void k_dbg_stream(const St* __restrict__ src, St* __restrict__ dst, Geom G) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.pitch + ix;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int sx = ix - CX(i), sy = iy - CY(i);
        if (sx >= 0 && sx < G.nx && sy >= 0 && sy < G.ny) {
            const long long s = (long long)sy * G.pitch + sx;
            dst[i * G.plane + k] = src[i * G.plane + s];
            dst[(Q + i) * G.plane + k] = src[(Q + i) * G.plane + s];
        } else {
            dst[i * G.plane + k] = src[OPP(i) * G.plane + k];
            dst[(Q + i) * G.plane + k] = src[(Q + i) * G.plane + k];
        }
    }
}

// apply_bounce_back / swap_opposite, src/uniform/solver.rs:920-946: on every
// wall node swap f_i and f_opp(i) for i = 1..4 (corners are visited twice).
template <class St>
__global__ void k_dbg_bounce_back(St* __restrict__ pop, Geom G) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    int visits = (ix == 0 || ix == G.nx - 1 ? 1 : 0) + (iy == 0 || iy == G.ny - 1 ? 1 : 0);
    if (visits % 2 == 0) return;  // not a wall node, or a corner swapped twice
    const long long k = (long long)iy * G.pitch + ix;
#pragma unroll
    for (int i = 1; i < 5; ++i) {
        St a = pop[i * G.plane + k];
        pop[i * G.plane + k] = pop[OPP(i) * G.plane + k];
        pop[OPP(i) * G.plane + k] = a;
    }
}

// apply_thermal_boundary_conditions, src/uniform/solver.rs:951-988, vertical walls.
template <class St>
__global__ void k_dbg_thermal_v(St* __restrict__ pop, Geom G, StepScalars<typename Fmt<St>::A> c) {
    using A = typename Fmt<St>::A;
    const int iy = blockIdx.x * blockDim.x + threadIdx.x;
    if (iy >= G.ny) return;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        stp(pop, G, Q + i, iy, 0, geq_rest<A>(i, c.t_hot[iy], c.geq_order));
        stp(pop, G, Q + i, iy, G.nx - 1, geq_rest<A>(i, c.t_cold, c.geq_order));
    }
}
// ... then the horizontal walls copy rows 1 and ny-2.
template <class St>
__global__ void k_dbg_thermal_h(St* __restrict__ pop, Geom G) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    if (ix >= G.nx) return;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const long long p = (long long)(Q + i) * G.plane;
        pop[p + ix] = pop[p + G.pitch + ix];
        pop[p + (long long)(G.ny - 1) * G.pitch + ix] = pop[p + (long long)(G.ny - 2) * G.pitch + ix];
    }
}

// update_macroscopic, src/uniform/solver.rs:298-367 (no wall override).
template <class St>
__global__ void k_dbg_macro(const St* __restrict__ pop, const typename Fmt<St>::A* __restrict__ fy,
                            typename Fmt<St>::A* __restrict__ rho, typename Fmt<St>::A* __restrict__ ux,
                            typename Fmt<St>::A* __restrict__ uy, typename Fmt<St>::A* __restrict__ tt, Geom G) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.pitch + ix;
    A f[Q], g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        f[i] = ldp(pop, G, i, iy, ix);
        g[i] = ldp(pop, G, Q + i, iy, ix);
    }
    Macro<A, SH> m = macro_node<A, SH>(f, g, fy[k], false);
    rho[k] = m.rho;
    ux[k] = m.ux;
    uy[k] = m.uy;
    tt[k] = m.t;
}

// enforce_wall_velocity, src/uniform/solver.rs:992-1009.
template <class A>
__global__ void k_dbg_noslip(A* __restrict__ ux, A* __restrict__ uy, Geom G) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    if (!is_wall(G, ix, iy)) return;
    const long long k = (long long)iy * G.pitch + ix;
    ux[k] = A(0.0);
    uy[k] = A(0.0);
}

// ---------------------------------------------------------------------------
// Population format conversion (ABI arrays are FP64 AoS [k][9]).
// ---------------------------------------------------------------------------
template <class St>
__global__ void k_pops_to_aos(const St* __restrict__ pop, double* __restrict__ f, double* __restrict__ g, Geom G) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.nx + ix;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        double fv = double(ldp(pop, G, i, iy, ix));
        if (Fmt<St>::SHIFT) fv += WD(i);
        f[k * Q + i] = fv;
        g[k * Q + i] = double(ldp(pop, G, Q + i, iy, ix));
    }
}
template <class St>
__global__ void k_aos_to_pops(St* __restrict__ pop, const double* __restrict__ f, const double* __restrict__ g,
                              int do_f, int do_g, Geom G) {
    using A = typename Fmt<St>::A;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.nx + ix;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        if (do_f) {
            double fv = f[k * Q + i];
            if (Fmt<St>::SHIFT) fv -= WD(i);
            stp(pop, G, i, iy, ix, A(fv));
        }
        if (do_g) stp(pop, G, Q + i, iy, ix, A(g[k * Q + i]));
    }
}

}  // namespace cav
