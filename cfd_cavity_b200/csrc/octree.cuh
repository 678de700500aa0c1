// octree.cuh -- the block-refined (octree) cavity of src/octree/ on the GPU.
//
// Levels: L0 the full coarse grid; L1 two blocks (hot / cold wall) of
// (2 w + 3) x (2 (ny0 - 1) + 3) nodes, ghost ring included
// (OctreeGrid::build, src/octree/grid.rs:103-204); with levels = 3, L2 one
// strip per L1 block, nested on the L1 grid (src/octree/solver.rs:368-431).
// One coarse step (step_cavity, src/octree/solver.rs:647-947) is
//   L0 step; c2f(L0 -> L1); L1 sub-step; [c2f(L1 -> L2); L2 sub-step x 2;
//   f2c(L2 -> L1) + refresh]; L1 sub-step; f2c(L1 -> L0) + refresh
// where a (sub-)step is collide -> stream -> thermal BC -> macroscopic (Guo)
// -> no-slip.  The hot and cold blocks are independent between the two
// couplings, so every launch covers both (blockIdx.y = block).
//
// Each level holds
//   REF  post-stream populations + rho/u/T (what the reference holds
//        between its phases; read by the couplings and the diagnostics),
//   PC   post-collision populations of the level's next collision,
// both double-buffered.  k_oct_step does pull + BC + macroscopic + no-slip
// of one (sub-)step, writes REF, then runs the level's NEXT collision and
// writes PC (the reference order rotated by one phase, as in the uniform
// solver).  The ghost ring of an L1/L2 level is never collided: interior
// nodes pull it from REF.  f2c injects into the coarser level's REF,
// refreshes its moments and runs that node's next collision, so the
// coarser level's PC stays consistent.
//
// Storage: OctImpl<StC, StF> keeps L0 in StC and L1/L2 in StF; A is the
// arithmetic type of both.  FP64 (double, double) reproduces the FP64 oracle
// bit for bit (translation unit built without FMA contraction); the shifted
// formats keep f - w_i and, in the moment planes, rho - 1.
#pragma once

#include "solver.cuh"

namespace cav {
namespace oct {

constexpr int OT = 128;          // threads per CTA, node kernels
constexpr int OCT_GRAPH_STEPS = 16;  // even: a replay leaves every buffer parity unchanged
constexpr int OSTAT = 6;         // per-CTA statistics: min rho, max rho, max |u|, nonfinite, sum (d)rho, unused
constexpr int OSTAT_CTAS = 64;
constexpr double T_HOT_C = 0.5, T_COLD_C = -0.5;

// Collision constants of one level for one coarse step: RelaxTimes::from_nu_alpha
// (src/octree/lbm.rs:90-98) and the coefficients of collide_node_cavity
// (src/octree/cavity.rs:100-121), evaluated on the host in FP64.
template <class A>
struct LvlScal {
    A a_f, b_f, a_g, c_m, c_p;           // reference (FP64) form
    A om_p, om_m, om_g, k_p, k_m;        // pairwise (FP32) form
    A beta;
    A tp, tt;                            // tau+ and tau_t of the level (the dynamic model's base)
    // fixed-Cs Smagorinsky on the level (an extension: the reference octree
    // has none; cs = 0 is the reference)
    A cs, nu, alpha, tau_s, inv_tau_s, pr_t, inv_pr_t;
};
template <class A>
struct OctScal {
    LvlScal<A> l[3];
};

// Rescaling factors (rescaling_factors_multilevel, src/octree/interface.rs:112-131).
template <class A>
struct Xi {
    A even, odd, th;
    A inv_even, inv_odd, inv_th;
};

// Per-node nu_t / alpha_t of the dynamic model for the two blocks of a launch
// (nullptr: the level's relaxation times).
template <class A>
struct DynPtr {
    const A* nut[2];
    const A* at[2];
};

// One level (or one block of a level) as the kernels see it.
template <class St>
struct LvlIO {
    using A = typename Fmt<St>::A;
    const St* ref_in;
    St* ref_out;
    const St* pc_in;
    St* pc_out;
    A* mac;   // 4 planes: rho (rho - 1 when shifted), ux, uy, T
    A* fy;    // Guo force of the last collision (0 on ghosts)
    int nx, ny;
    int n;    // nx * ny (plane stride)
    int hot, cold;
    int node_off;  // offset of this level's nodes in the rounding streams
};
template <class St>
struct LvlPair {
    LvlIO<St> b[2];
};

template <class A>
struct GhostE {
    int kf;
    int kc[4];
    A w[4];
};
struct CoinE {
    int kc;  // node on the coarser grid
    int a, b;  // centre of the 3x3 stencil on the finer grid
};

template <class A>
__device__ __forceinline__ const OctScal<A>& row_of(const OctScal<A>* tab, int S, const long long* step_dev, int off,
                                                    long long* s_out) {
    const long long s = *step_dev + off;
    *s_out = s;
    return tab[s < S ? s : S];
}

// ---------------------------------------------------------------------------
// Collision of one node (collide_node_cavity, src/octree/cavity.rs:70-150,
// nu_t = 0): TRT + Guo forcing for f, BGK for g.
// ---------------------------------------------------------------------------
// The shifted formats' collision in two halves (pairwise (i, opp(i)) TRT on
// h_i = f_i - w_i, as in the uniform FP32 collision, with the level's fixed
// relaxation rates; BGK for g): the f half needs T for the Guo force, the g
// half u, v; u^2 is formed once (oct_u2) and handed to both.  Every operation
// is an explicitly rounded intrinsic (no contraction left to the compiler),
// so the two halves give the same bits whether one thread runs them or two.
__device__ __forceinline__ float oct_u2(float u, float v) { return __fmaf_rn(u, u, __fmul_rn(v, v)); }
// c_p . u for p = 1..4 (c_x, c_y in {-1, 0, 1}: the products are exact)
__device__ __forceinline__ float oct_eu(int p, float u, float v) {
    return __fadd_rn(__fmul_rn(float(CX(p)), u), __fmul_rn(float(CY(p)), v));
}
// 4.5 (c_p . u)^2 - 1.5 u^2
__device__ __forceinline__ float oct_q(float eu, float u2) {
    return __fmaf_rn(__fmul_rn(4.5f, eu), eu, __fmul_rn(-1.5f, u2));
}
__device__ __forceinline__ void oct_collide_f_sh(float (&f)[Q], float r, float drho, float u, float v, float u2,
                                                 float temp, const LvlScal<float>& c, float& fy_out) {
    const float fyv = __fmul_rn(__fmul_rn(r, c.beta), temp);
    fy_out = fyv;
    const float hp = __fmul_rn(-0.5f, c.om_p), hm = __fmul_rn(-0.5f, c.om_m);
    const float m3v = __fmul_rn(-3.0f, v);
    const float feq0 = __fmul_rn(float(WD(0)), __fmaf_rn(-__fmul_rn(1.5f, r), u2, drho));
    const float d0 = __fsub_rn(f[0], feq0);
    const float s0 = __fmul_rn(__fmul_rn(__fmul_rn(c.k_p, float(WD(0))), m3v), fyv);
    f[0] = __fmaf_rn(-c.om_p, d0, __fadd_rn(f[0], s0));
    const float r3 = __fmul_rn(r, 3.0f);
#pragma unroll
    for (int p = 1; p <= 4; ++p) {
        const float w = float(WD(p)), cy = float(CY(p));
        const float eu = oct_eu(p, u, v);
        const float feS = __fmul_rn(w, __fmaf_rn(r, oct_q(eu, u2), drho));
        const float feA = __fmul_rn(w, __fmul_rn(r3, eu));
        const float dS = __fmaf_rn(-2.0f, feS, __fadd_rn(f[p], f[p + 4]));
        const float dD = __fmaf_rn(-2.0f, feA, __fsub_rn(f[p], f[p + 4]));
        const float sE = __fmaf_rn(__fmul_rn(9.0f, cy), eu, m3v);
        const float E = __fmaf_rn(hp, dS, __fmul_rn(__fmul_rn(__fmul_rn(c.k_p, w), sE), fyv));
        const float O = __fmaf_rn(hm, dD, __fmul_rn(__fmul_rn(__fmul_rn(c.k_m, w), __fmul_rn(3.0f, cy)), fyv));
        f[p] = __fadd_rn(f[p], __fadd_rn(E, O));
        f[p + 4] = __fadd_rn(f[p + 4], __fsub_rn(E, O));
    }
}
__device__ __forceinline__ void oct_collide_g_sh(float (&g)[Q], float u, float v, float u2, float temp,
                                                 const LvlScal<float>& c) {
    const float om_g = c.om_g, one_m = __fsub_rn(1.0f, om_g);
    const float a0 = __fmul_rn(__fmul_rn(om_g, float(WD(0))), temp);
    g[0] = __fmaf_rn(one_m, g[0], __fmul_rn(a0, __fmaf_rn(-1.5f, u2, 1.0f)));
#pragma unroll
    for (int p = 1; p <= 4; ++p) {
        const float eu = oct_eu(p, u, v);
        const float ogw = __fmul_rn(__fmul_rn(om_g, float(WD(p))), temp);
        const float gS = __fmul_rn(ogw, __fadd_rn(1.0f, oct_q(eu, u2)));
        const float gA = __fmul_rn(ogw, __fmul_rn(3.0f, eu));
        g[p] = __fmaf_rn(one_m, g[p], __fadd_rn(gS, gA));
        g[p + 4] = __fmaf_rn(one_m, g[p + 4], __fsub_rn(gS, gA));
    }
}

template <class A, bool SHIFT>
__device__ __forceinline__ void oct_collide(A (&f)[Q], A (&g)[Q], const Macro<A, SHIFT>& m, const LvlScal<A>& c0,
                                            A& fy_out, const A* nut = nullptr, const A* at = nullptr) {
    LvlScal<A> c = c0;
    if (nut) {
        // dynamic model: relaxation times rebuilt per node from the level's
        // tau and the node's nu_t / alpha_t (src/octree/cavity.rs:100-110)
        const A tp = A(0.5) + A(3.0) * (c0.tp - A(0.5)) / A(3.0) + A(3.0) * *nut;
        const A tm = A(0.5) + A(LAMBDA_TRT) / (tp - A(0.5));
        const A tt = A(0.5) + A(3.0) * (c0.tt - A(0.5)) / A(3.0) + A(3.0) * *at;
        c.a_f = A(0.5) * (A(1.0) / tp + A(1.0) / tm);
        c.b_f = A(0.5) * (A(1.0) / tp - A(1.0) / tm);
        c.a_g = A(1.0) / tt;
        c.c_m = A(1.0) - A(0.5) / tm;
        c.c_p = A(1.0) - A(0.5) / tp;
        c.om_p = A(1.0) / tp;
        c.om_m = A(1.0) / tm;
        c.om_g = A(1.0) / tt;
        c.k_p = c.c_p;
        c.k_m = c.c_m;
        c.cs = A(0.0);
    }
    if (c.cs != A(0.0)) {
        // with the Smagorinsky extension: the uniform solver's collision
        // (collide_node, src/uniform/solver.rs:1054-1185) with the level's
        // molecular nu / alpha and lattice spacing 1
        StepScalars<A> u{};
        u.tau_s = c.tau_s;
        u.beta = c.beta;
        u.nu = c.nu;
        u.alpha = c.alpha;
        u.cs = c.cs;
        u.pr_t = c.pr_t;
        u.inv_tau_s = c.inv_tau_s;
        u.inv_pr_t = c.inv_pr_t;
        u.geq_order = 2;
        A nut;
        collide_node<A, SHIFT>(f, g, m, u, fy_out, nut);
        return;
    }
    if constexpr (!SHIFT) {
        const double r = m.rho, u = m.ux, v = m.uy, temp = m.t;
        const double fyv = r * c.beta * 1.0 * (temp - 0.0);
        fy_out = fyv;
        double d_f[Q], d_g[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            d_f[i] = f[i] - feq_full<double>(i, r, u, v);
            d_g[i] = g[i] - geq_full<double>(i, temp, u, v, 2);
        }
        double fo[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const double cx = CX(i), cy = CY(i);
            const double ei_u = cx * u + cy * v;
            const double s_i = WD(i) * ((cy - v) / CS2 + ei_u * cy / (CS2 * CS2)) * fyv;
            const double s_minus = WD(i) * (cy / CS2) * fyv;
            const double s_plus = s_i - s_minus;
            fo[i] = f[i] + (-c.a_f * d_f[i] - c.b_f * d_f[OPP(i)] + c.c_m * s_minus + c.c_p * s_plus);
        }
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = fo[i];
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = g[i] + (-c.a_g * d_g[i] - 0.0 * d_g[OPP(i)]);
    } else {
        const float u2 = oct_u2(m.ux, m.uy);
        oct_collide_f_sh(f, m.rho, m.drho, m.ux, m.uy, u2, m.t, c, fy_out);
        oct_collide_g_sh(g, m.ux, m.uy, u2, m.t, c);
    }
}

// f_i^eq in the storage convention (f - w_i when shifted) from the stored moments.
template <class A, bool SHIFT>
__device__ __forceinline__ A feq_st(int i, A rho0, A ux, A uy) {
    if constexpr (SHIFT) {
        const A drho = rho0, r = A(1.0) + rho0;
        const A eu = A(CX(i)) * ux + A(CY(i)) * uy;
        const A u2 = ux * ux + uy * uy;
        return A(WD(i)) * (drho + r * (A(3.0) * eu + A(4.5) * eu * eu - A(1.5) * u2));
    } else {
        return feq_full<A>(i, rho0, ux, uy);
    }
}

// Stores the 18 populations of node k (stochastic rounding when `sr` and
// the format rounds stochastically).  With BACK, f and g are replaced by the
// stored (rounded) values, computed in registers rather than re-read.
template <class St, bool BACK = false>
__device__ __forceinline__ void store_pops(St* __restrict__ dst, int n, int k, typename Fmt<St>::A (&f)[Q],
                                           typename Fmt<St>::A (&g)[Q], bool sr, uint32_t seed, long long key,
                                           long long node) {
    if constexpr (Fmt<St>::HW_SR_F) {
        // pairs of binary16 / bfloat16 planes by one cvt.rs (enc2_sr), fed
        // the bits the software rounding below takes from the same draw
        if (sr) {
            NodeRng rng(seed, key, node);
            const float sf = p2(Fmt<St>::EF), sg = p2(Fmt<St>::EG);
#pragma unroll
            for (int q = 0; q < NPLANES; q += 2) {
                const uint32_t r = rng.next();
                typename Fmt<St>::A& xa = q < Q ? f[q] : g[q - Q];
                typename Fmt<St>::A& xb = q + 1 < Q ? f[q + 1] : g[q + 1 - Q];
                const bool ha = q < Q || Fmt<St>::HW_SR_G, hb = q + 1 < Q || Fmt<St>::HW_SR_G;
                St va, vb;
                if (ha && hb) {
                    const uint32_t d = Fmt<St>::enc2_sr(xa * (q < Q ? sf : sg), xb * (q + 1 < Q ? sf : sg), r);
                    va.bits = (unsigned short)(d >> 16);
                    vb.bits = (unsigned short)(d & 0xffffu);
                } else {
                    if (ha)
                        va.bits = (unsigned short)(Fmt<St>::enc2_sr(xa * sf, 0.0f, r) >> 16);
                    else
                        va = Fmt<St>::store_sr(xa, q, r & 0xffff0000u);
                    vb = Fmt<St>::store_sr(xb, q + 1, r << 16);
                }
                dst[q * n + k] = va;
                dst[(q + 1) * n + k] = vb;
                if (BACK) {
                    xa = Fmt<St>::load(va, q);
                    xb = Fmt<St>::load(vb, q + 1);
                }
            }
            return;
        }
    } else if constexpr (Fmt<St>::SR) {
        if (sr) {
            NodeRng rng(seed, key, node);
            uint32_t r = 0;
#pragma unroll
            for (int q = 0; q < NPLANES; ++q) {
                if ((q & 1) == 0) r = rng.next();
                const uint32_t bits = (q & 1) == 0 ? (r & 0xffff0000u) : (r << 16);
                typename Fmt<St>::A& x = q < Q ? f[q] : g[q - Q];
                const St v = Fmt<St>::store_sr(x, q, bits);
                dst[q * n + k] = v;
                if (BACK) x = Fmt<St>::load(v, q);
            }
            return;
        }
    }
#pragma unroll
    for (int q = 0; q < NPLANES; ++q) {
        typename Fmt<St>::A& x = q < Q ? f[q] : g[q - Q];
        const St v = Fmt<St>::store(x, q, RN_BITS);
        dst[q * n + k] = v;
        if (BACK) x = Fmt<St>::load(v, q);
    }
}

// The planes of one half of store_pops (G: the g planes Q..2Q-1 from x,
// else the f planes 0..Q-1), each with the bits store_pops gives it: the
// node's draws are generated in full and this half's share of each pair used.
// A binary16 / bfloat16 pair that store_pops rounds by one cvt.rs is rounded
// here with the other half zero (the two halves are rounded independently).
template <class St, bool G>
__device__ __forceinline__ void store_half(St* __restrict__ dst, int n, int k, const typename Fmt<St>::A (&x)[Q],
                                           bool sr, uint32_t seed, long long key, long long node) {
    constexpr int Q0 = G ? Q : 0;
    if constexpr (Fmt<St>::HW_SR_F) {
        if (sr) {
            NodeRng rng(seed, key, node);
            const float sf = p2(Fmt<St>::EF), sg = p2(Fmt<St>::EG);
#pragma unroll
            for (int q = 0; q < NPLANES; q += 2) {
                const uint32_t r = rng.next();
                const bool ha = q < Q || Fmt<St>::HW_SR_G, hb = q + 1 < Q || Fmt<St>::HW_SR_G;
                if (q >= Q0 && q < Q0 + Q) {  // plane q (the pair's first) is this half's
                    const float xa = x[q - Q0];
                    St va;
                    if (ha && hb)
                        va.bits = (unsigned short)(Fmt<St>::enc2_sr(xa * (q < Q ? sf : sg), 0.0f, r) >> 16);
                    else if (ha)
                        va.bits = (unsigned short)(Fmt<St>::enc2_sr(xa * sf, 0.0f, r) >> 16);
                    else
                        va = Fmt<St>::store_sr(xa, q, r & 0xffff0000u);
                    dst[q * n + k] = va;
                }
                if (q + 1 >= Q0 && q + 1 < Q0 + Q) {  // plane q + 1 is this half's
                    const float xb = x[q + 1 - Q0];
                    St vb;
                    if (ha && hb)
                        vb.bits = (unsigned short)(Fmt<St>::enc2_sr(0.0f, xb * (q + 1 < Q ? sf : sg), r) & 0xffffu);
                    else
                        vb = Fmt<St>::store_sr(xb, q + 1, r << 16);
                    dst[(q + 1) * n + k] = vb;
                }
            }
            return;
        }
    } else if constexpr (Fmt<St>::SR) {
        if (sr) {
            NodeRng rng(seed, key, node);
            uint32_t r = 0;
#pragma unroll
            for (int q = 0; q < NPLANES; ++q) {
                if ((q & 1) == 0) r = rng.next();
                if (q < Q0 || q >= Q0 + Q) continue;
                const uint32_t bits = (q & 1) == 0 ? (r & 0xffff0000u) : (r << 16);
                dst[q * n + k] = Fmt<St>::store_sr(x[q - Q0], q, bits);
            }
            return;
        }
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) dst[(Q0 + i) * n + k] = Fmt<St>::store(x[i], Q0 + i, RN_BITS);
}

template <class St>
__device__ __forceinline__ void load_pops(const St* __restrict__ src, int n, int k, typename Fmt<St>::A (&f)[Q],
                                          typename Fmt<St>::A (&g)[Q]) {
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = Fmt<St>::load(src[i * n + k], i);
#pragma unroll
    for (int i = 0; i < Q; ++i) g[i] = Fmt<St>::load(src[(Q + i) * n + k], Q + i);
}

// ---------------------------------------------------------------------------
// Streaming sources.  L0 (stream, src/octree/lbm.rs:152-180): pull inside
// the grid, bounce-back (f) / keep (g) outside.  L1/L2 blocks
// (stream_cavity_block, src/octree/cavity.rs:393-495, wall_bottom =
// wall_top = true): interior nodes only; a source in a wall-side ghost line
// bounces back, a source in an interface ghost column is pulled from REF
// (the injected value), any other source from PC.
// The per-node neighbour classes are computed once (Src), so that each of
// the 18 loads costs a select and an address; all loads are in flight
// together.
// ---------------------------------------------------------------------------
struct Src {
    int k, nx;
    bool bb_xm, bb_xp, bb_ym, bb_yp;  // source x-1 / x+1 / y-1 / y+1 bounces back
    bool gh_xm, gh_xp;                // source x-1 / x+1 is an interface ghost (REF)
};

template <bool COARSE, class St>
__device__ __forceinline__ Src src_of(const LvlIO<St>& L, int x, int y) {
    Src r;
    r.k = y * L.nx + x;
    r.nx = L.nx;
    if constexpr (COARSE) {
        r.bb_xm = x == 0;
        r.bb_xp = x == L.nx - 1;
        r.bb_ym = y == 0;
        r.bb_yp = y == L.ny - 1;
        r.gh_xm = r.gh_xp = false;
    } else {
        r.bb_ym = y - 1 == 0;
        r.bb_yp = y + 1 == L.ny - 1;
        const bool xm_edge = x - 1 == 0, xp_edge = x + 1 == L.nx - 1;
        r.bb_xm = xm_edge && L.hot;
        r.bb_xp = xp_edge && L.cold;
        r.gh_xm = xm_edge && !L.hot;
        r.gh_xp = xp_edge && !L.cold;
    }
    return r;
}

// Population q_plane (plane i of f, or Q + i of g) streamed into the node.
template <class St>
__device__ __forceinline__ typename Fmt<St>::A pull_one(const LvlIO<St>& L, const Src& r, int q_plane, int i) {
    const int cx = CX(i), cy = CY(i);
    const bool bb = (cx > 0 && r.bb_xm) || (cx < 0 && r.bb_xp) || (cy > 0 && r.bb_ym) || (cy < 0 && r.bb_yp);
    const bool ghost = !bb && ((cx > 0 && r.gh_xm) || (cx < 0 && r.gh_xp));
    const St* base = ghost ? L.ref_in : L.pc_in;
    const int qs = (bb && q_plane < Q) ? OPP(i) : q_plane;
    const int ks = bb ? r.k : r.k - cx - cy * r.nx;
    return Fmt<St>::load(base[qs * L.n + ks], qs);
}

// Post-boundary-condition g of node (x, y).  L0
// (apply_thermal_boundary_conditions, src/octree/cavity.rs:501-534): wall
// columns geq(T_w, 0, 0), rows 0 / ny-1 copy rows 1 / ny-2.  Blocks
// (apply_thermal_boundary_conditions_block, :543-605): wall column 1 / nx-2
// geq(T_w); rows 1 / ny-2 copy rows 2 / ny-3 (columns 1..nx-2); ghost
// columns copy columns 1 / nx-2; ghost rows copy rows 1 / ny-2.  Resolving
// the copy chain: g(x, y) is the post-stream g of (x', y'') with x' the
// column clamped to 1..nx-2 and y'' the row clamped to 2..ny-3, or the wall
// equilibrium when x' is a wall column.
template <class St, bool COARSE>
__device__ __forceinline__ void bc_g(const LvlIO<St>& L, int x, int y, const Src& own, typename Fmt<St>::A (&g)[Q]) {
    using A = typename Fmt<St>::A;
    int xs, ys;
    bool wall;
    A tw;
    if constexpr (COARSE) {
        wall = x == 0 || x == L.nx - 1;
        tw = x == 0 ? A(T_HOT_C) : A(T_COLD_C);
        xs = x;
        ys = y < 1 ? 1 : (y > L.ny - 2 ? L.ny - 2 : y);
    } else {
        xs = x < 1 ? 1 : (x > L.nx - 2 ? L.nx - 2 : x);
        const int y1 = y < 1 ? 1 : (y > L.ny - 2 ? L.ny - 2 : y);
        ys = y1 == 1 ? 2 : (y1 == L.ny - 2 ? L.ny - 3 : y1);
        wall = (L.hot && xs == 1) || (L.cold && xs == L.nx - 2);
        tw = (L.hot && xs == 1) ? A(T_HOT_C) : A(T_COLD_C);
    }
    if (wall) {
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = geq_full<A>(i, tw, A(0.0), A(0.0), 2);
    } else {
        const Src r = (xs == x && ys == y) ? own : src_of<COARSE>(L, xs, ys);
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = pull_one<St>(L, r, Q + i, i);
    }
}

// Row and column of node k of a level with nx columns (exact for k < 2^22).
__device__ __forceinline__ void split_k(int k, int nx, float inv_nx, int& x, int& y) {
    y = int((float(k) + 0.5f) * inv_nx);
    x = k - y * nx;
}

// One (sub-)step of a level: pull + BC + macroscopic (update_macroscopic_guo,
// src/octree/cavity.rs:252-325) + no-slip (enforce_wall_velocity[_block],
// :609-656) -> REF; then the level's next collision -> PC.
template <class St, bool COARSE>
__global__ void __launch_bounds__(OT) k_oct_step(LvlPair<St> P, const OctScal<typename Fmt<St>::A>* __restrict__ tab,
                                                 int S, const long long* __restrict__ step_dev, int off, int lvl,
                                                 uint32_t seed, int phase, float inv_nx, int collide) {
    pdl_wait();
    pdl_trigger();
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const LvlIO<St> L = P.b[blockIdx.y];
    const int k = blockIdx.x * OT + threadIdx.x;
    if (k >= L.n) return;
    // the step index and the collision constants first: the stores below
    // may alias them as far as the compiler knows
    long long s;
    const LvlScal<A> sc = row_of<A>(tab, S, step_dev, off, &s).l[lvl];
    int x, y;
    split_k(k, L.nx, inv_nx, x, y);
    const bool ghost = !COARSE && (x == 0 || x == L.nx - 1 || y == 0 || y == L.ny - 1);
    const Src own = src_of<COARSE>(L, x, y);
    A f[Q], g[Q];
    if (ghost) {
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = Fmt<St>::load(L.ref_in[i * L.n + k], i);
    } else {
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = pull_one<St>(L, own, i, i);
    }
    bc_g<St, COARSE>(L, x, y, own, g);
    bool wall;
    if constexpr (COARSE)
        wall = x == 0 || x == L.nx - 1 || y == 0 || y == L.ny - 1;
    else
        wall = (L.hot && x == 1) || (L.cold && x == L.nx - 2) || y == 1 || y == L.ny - 2;
    const A fy_prev = L.fy[k];
    const Macro<A, SH> m = macro_node<A, SH>(f, g, fy_prev, wall);
    store_pops<St>(L.ref_out, L.n, k, f, g, false, 0, 0, 0);
    L.mac[k] = SH ? m.drho : m.rho;
    L.mac[L.n + k] = m.ux;
    L.mac[2 * L.n + k] = m.uy;
    L.mac[3 * L.n + k] = m.t;
    if (ghost || !collide) return;
    A fy_new;
    oct_collide<A, SH>(f, g, m, sc, fy_new);
    L.fy[k] = fy_new;
    store_pops<St>(L.pc_out, L.n, k, f, g, true, seed, s * 16 + phase, (long long)L.node_off + k);
}

// One (sub-)step of a fine level (L1 / L2) with each node's f and g halves
// on two threads, for the shifted formats without the fixed-Cs extension:
// OCT_FG nodes per CTA; the first OCT_FG threads take the f halves (pull of
// f, rho and u with the Guo half force and no-slip, the f REF planes and the
// moments, the TRT update with the Guo force, the f PC planes, fy), the
// others the g halves (pull of g at its boundary-condition source, T, the g
// REF planes, the BGK update, the g PC planes); they exchange u, v, u^2 and
// T through shared memory at one barrier.  Same bits as k_oct_step.
constexpr int OCT_FG = 64;
template <class St>
__global__ void __launch_bounds__(2 * OCT_FG) k_oct_step_fg(LvlPair<St> P, const OctScal<float>* __restrict__ tab,
                                                           int S, const long long* __restrict__ step_dev, int off,
                                                           int lvl, uint32_t seed, int phase, float inv_nx) {
    static_assert(Fmt<St>::SHIFT, "the split step runs the shifted formats");
    pdl_wait();
    pdl_trigger();
    __shared__ float xu[OCT_FG], xv[OCT_FG], xq[OCT_FG], xt[OCT_FG];
    const LvlIO<St> L = P.b[blockIdx.y];
    const bool g_half = threadIdx.x >= OCT_FG;
    const int j = g_half ? threadIdx.x - OCT_FG : threadIdx.x;
    const int k = blockIdx.x * OCT_FG + j;
    const bool act = k < L.n;
    long long s;
    const LvlScal<float> sc = row_of<float>(tab, S, step_dev, off, &s).l[lvl];
    int x = 0, y = 0;
    if (act) split_k(k, L.nx, inv_nx, x, y);
    const bool ghost = x == 0 || x == L.nx - 1 || y == 0 || y == L.ny - 1;
    const long long key = s * 16 + phase, node = (long long)L.node_off + k;
    if (!g_half) {
        float f[Q];
        float r = 0.0f, drho = 0.0f, u = 0.0f, v = 0.0f, u2 = 0.0f;
        if (act) {
            const Src own = src_of<false>(L, x, y);
            if (ghost) {
#pragma unroll
                for (int i = 0; i < Q; ++i) f[i] = Fmt<St>::load(L.ref_in[i * L.n + k], i);
            } else {
#pragma unroll
                for (int i = 0; i < Q; ++i) f[i] = pull_one<St>(L, own, i, i);
            }
            const bool wall = (L.hot && x == 1) || (L.cold && x == L.nx - 2) || y == 1 || y == L.ny - 2;
            const Macro<float, true> m = macro_f<float, true>(f, L.fy[k], wall);
            store_half<St, false>(L.ref_out, L.n, k, f, false, 0, 0, 0);
            L.mac[k] = m.drho;
            L.mac[L.n + k] = m.ux;
            L.mac[2 * L.n + k] = m.uy;
            r = m.rho;
            drho = m.drho;
            u = m.ux;
            v = m.uy;
            u2 = oct_u2(u, v);
        }
        xu[j] = u;
        xv[j] = v;
        xq[j] = u2;
        named_bar_sync(1, 2 * OCT_FG);
        if (act && !ghost) {
            float fy_new;
            oct_collide_f_sh(f, r, drho, u, v, u2, xt[j], sc, fy_new);
            L.fy[k] = fy_new;
            store_half<St, false>(L.pc_out, L.n, k, f, true, seed, key, node);
        }
    } else {
        float g[Q];
        float t = 0.0f;
        if (act) {
            const Src own = src_of<false>(L, x, y);
            bc_g<St, false>(L, x, y, own, g);
            t = sum_g<float>(g);
            store_half<St, true>(L.ref_out, L.n, k, g, false, 0, 0, 0);
            L.mac[3 * L.n + k] = t;
        }
        xt[j] = t;
        named_bar_sync(1, 2 * OCT_FG);
        if (act && !ghost) {
            oct_collide_g_sh(g, xu[j], xv[j], xq[j], t, sc);
            store_half<St, true>(L.pc_out, L.n, k, g, true, seed, key, node);
        }
    }
}

// Collision of the REF state into PC: the first collision after the state
// was set from the host, and every collision of the dynamic model (with the
// per-node nu_t / alpha_t of D).
template <class St, bool COARSE>
__global__ void __launch_bounds__(OT) k_oct_collide(LvlPair<St> P, const OctScal<typename Fmt<St>::A>* __restrict__ tab,
                                                    int S, const long long* __restrict__ step_dev, int lvl,
                                                    uint32_t seed, int phase, DynPtr<typename Fmt<St>::A> D) {
    pdl_wait();
    pdl_trigger();
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const LvlIO<St> L = P.b[blockIdx.y];
    const int k = blockIdx.x * OT + threadIdx.x;
    if (k >= L.n) return;
    const int x = k % L.nx, y = k / L.nx;
    if (!COARSE && (x == 0 || x == L.nx - 1 || y == 0 || y == L.ny - 1)) return;
    long long s;
    const LvlScal<A> sc = row_of<A>(tab, S, step_dev, 0, &s).l[lvl];
    A f[Q], g[Q];
    load_pops<St>(L.ref_in, L.n, k, f, g);
    Macro<A, SH> m;
    const A r0 = L.mac[k];
    m.rho = SH ? A(1.0) + r0 : r0;
    m.drho = SH ? r0 : r0 - A(1.0);
    m.ux = L.mac[L.n + k];
    m.uy = L.mac[2 * L.n + k];
    m.t = L.mac[3 * L.n + k];
    m.inv_rho = A(1.0) / m.rho;
    const A* nut = D.nut[blockIdx.y];
    const A* at = D.at[blockIdx.y];
    A fy_new;
    oct_collide<A, SH>(f, g, m, sc, fy_new, nut ? nut + k : nullptr, at ? at + k : nullptr);
    L.fy[k] = fy_new;
    store_pops<St>(L.pc_out, L.n, k, f, g, true, seed, s * 16 + phase, (long long)L.node_off + k);
}

// Moments of a node whose populations were just injected
// (refresh_moments, src/octree/interface.rs:209-227, unguarded, and
// refresh_moments_nodes, src/octree/solver.rs:1183-1206, guarded).
template <class A, bool SHIFT, bool GUARD>
__device__ __forceinline__ Macro<A, SHIFT> refresh(const A (&f)[Q], const A (&g)[Q]) {
    Macro<A, SHIFT> m;
    A rho = A(0.0), mx = A(0.0), my = A(0.0), t = A(0.0);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        rho = rho + f[i];
        mx = mx + f[i] * A(CX(i));
        my = my + f[i] * A(CY(i));
        t = t + g[i];
    }
    if (SHIFT) {
        m.drho = rho;
        m.rho = A(1.0) + rho;
    } else {
        m.rho = rho;
        m.drho = rho - A(1.0);
    }
    m.t = t;
    if (GUARD && !(m.rho > A(2.220446049250313e-16))) {
        m.ux = A(0.0);
        m.uy = A(0.0);
    } else {
        m.ux = mx / m.rho;
        m.uy = my / m.rho;
    }
    m.inv_rho = A(1.0) / m.rho;
    return m;
}

// even/odd split of f^neq and its rescaling (split_odd_even, rescale_fneq,
// rescale_fneq_inverse, src/octree/interface.rs:68-102).
template <class A, bool SHIFT, bool INVERSE>
__device__ __forceinline__ void rescale(const A (&fn)[Q], const Xi<A>& xi, A (&out)[Q]) {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const A even = A(0.5) * (fn[i] + fn[OPP(i)]);
        const A odd = A(0.5) * (fn[i] - fn[OPP(i)]);
        if constexpr (!INVERSE)
            out[i] = xi.even * even + xi.odd * odd;
        else if constexpr (SHIFT)
            out[i] = even * xi.inv_even + odd * xi.inv_odd;
        else
            out[i] = even / xi.even + odd / xi.odd;
    }
}

// Weighted contribution of one stencil node to a coupling: c[0..3] = w *
// (rho, ux, uy, T), c[4..12] = w * f^neq_i, c[13..21] = w * g^neq_i.
constexpr int NC = 22;
template <class St>
__device__ __forceinline__ void stencil_term(const LvlIO<St>& L, int k, typename Fmt<St>::A w,
                                             typename Fmt<St>::A (&c)[NC]) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const A r0 = L.mac[k], u = L.mac[L.n + k], v = L.mac[2 * L.n + k], t = L.mac[3 * L.n + k];
    A f[Q], g[Q];
    load_pops<St>(L.ref_out, L.n, k, f, g);
    c[0] = w * r0;
    c[1] = w * u;
    c[2] = w * v;
    c[3] = w * t;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        c[4 + i] = w * (f[i] - feq_st<A, SH>(i, r0, u, v));
        c[13 + i] = w * (g[i] - geq_full<A>(i, t, u, v, 2));
    }
}

// Sum of the group's contributions in lane order (the reference's stencil
// order, so that FP64 sums are bit-identical); every lane gets the sums.
template <class A, int GW, int NS>
__device__ __forceinline__ void group_sum(A (&c)[NC]) {
    const int base = (threadIdx.x & 31) & ~(GW - 1);
#pragma unroll
    for (int m = 0; m < NC; ++m) {
        A acc = __shfl_sync(0xffffffffu, c[m], base);
#pragma unroll
        for (int j = 1; j < NS; ++j) acc = acc + __shfl_sync(0xffffffffu, c[m], base + j);
        c[m] = acc;
    }
}

// coarse_to_fine (src/octree/interface.rs:137-170): every ghost node of the
// finer level gets the bilinear moments of the coarser level plus the
// interpolated, rescaled non-equilibrium parts; then its moments are
// refreshed from the injected populations.  Four lanes per ghost, one per
// stencil node.
template <class StC, class StF>
__global__ void __launch_bounds__(OT) k_oct_c2f(LvlPair<StC> C, LvlPair<StF> F,
                                                const GhostE<typename Fmt<StF>::A>* __restrict__ tab, int n_ghost,
                                                Xi<typename Fmt<StF>::A> xi_h,
                                                const Xi<typename Fmt<StF>::A>* __restrict__ xi_dev,
                                                const long long* __restrict__ step_dev, uint32_t seed, int phase) {
    pdl_wait();
    pdl_trigger();
    using A = typename Fmt<StF>::A;
    constexpr bool SH = Fmt<StF>::SHIFT;
    static_assert(Fmt<StC>::SHIFT == SH, "levels share one convention");
    const int t = blockIdx.x * OT + threadIdx.x;
    const int j = t >> 2, s = t & 3;
    if ((t & ~31) >= 4 * n_ghost) return;  // whole warp past the end
    const bool act = j < n_ghost;
    const LvlIO<StC> Lc = C.b[blockIdx.y];
    const LvlIO<StF> Lf = F.b[blockIdx.y];
    const long long key = *step_dev * 16 + phase;
    A c[NC];
    int kf = 0;
    if (act) {
        const GhostE<A>& e = tab[blockIdx.y * n_ghost + j];
        kf = e.kf;
        stencil_term<StC>(Lc, e.kc[s], e.w[s], c);
    } else {
#pragma unroll
        for (int m = 0; m < NC; ++m) c[m] = A(0.0);
    }
    group_sum<A, 4, 4>(c);
    if (!act || s != 0) return;
    const Xi<A> xi = xi_dev ? xi_dev[blockIdx.y] : xi_h;
    const A rho = c[0], ux = c[1], uy = c[2], tt = c[3];
    A fn[Q], fr[Q], f[Q], g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) fn[i] = c[4 + i];
    rescale<A, SH, false>(fn, xi, fr);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        f[i] = feq_st<A, SH>(i, rho, ux, uy) + fr[i];
        g[i] = geq_full<A>(i, tt, ux, uy, 2) + xi.th * c[13 + i];
    }
    store_pops<StF, true>(Lf.ref_out, Lf.n, kf, f, g, true, seed, key, (long long)Lf.node_off + kf);
    const Macro<A, SH> m = refresh<A, SH, false>(f, g);
    Lf.mac[kf] = SH ? m.drho : m.rho;
    Lf.mac[Lf.n + kf] = m.ux;
    Lf.mac[2 * Lf.n + kf] = m.uy;
    Lf.mac[3 * Lf.n + kf] = m.t;
}

// fine_to_coarse (src/octree/interface.rs:175-206) + refresh of the
// coincident node (src/octree/solver.rs:874-876, 936-942) + that node's next
// collision into the coarser level's PC (not with the dynamic model, whose
// collisions run after its own model evaluation).  Three lanes per
// coincident node (F2C_NPW nodes per warp): lane l takes the stencil nodes l,
// l + 3 and l + 6 in three rounds, and the terms are added in stencil order.
constexpr int F2C_NPW = 10;
template <class StF, class StC>
__global__ void __launch_bounds__(OT) k_oct_f2c(LvlPair<StF> F, LvlPair<StC> C, const CoinE* __restrict__ tab, int n0,
                                                int n1, Xi<typename Fmt<StF>::A> xi_h,
                                                const Xi<typename Fmt<StF>::A>* __restrict__ xi_dev,
                                                const OctScal<typename Fmt<StF>::A>* __restrict__ stab, int S,
                                                const long long* __restrict__ step_dev, int off, int lvl_c,
                                                uint32_t seed, int phase, int collide) {
    pdl_wait();
    pdl_trigger();
    using A = typename Fmt<StF>::A;
    constexpr bool SH = Fmt<StF>::SHIFT;
    // F2C_NPW coincident nodes per warp, three lanes each (lanes 30, 31 idle)
    const int t = blockIdx.x * OT + threadIdx.x;
    const int wi = t >> 5, lane = t & 31;
    const int j = wi * F2C_NPW + lane / 3, l = lane - 3 * (lane / 3);
    const int blk = blockIdx.y;
    const int nb = blk == 0 ? n0 : n1;
    if (wi * F2C_NPW >= nb) return;  // whole warp past the end
    const bool act_e = lane < 3 * F2C_NPW && j < nb;
    const LvlIO<StF> Lf = F.b[blk];
    const LvlIO<StC> Lc = C.b[blk];
    CoinE e{0, 0, 0};
    if (act_e) e = tab[(blk == 0 ? 0 : n0) + j];
    long long sidx;
    const LvlScal<A> sc = row_of<A>(stab, S, step_dev, off, &sidx).l[lvl_c];
    const int base = lane < 3 * F2C_NPW ? lane - l : 3 * (F2C_NPW - 1);
    const A ww[3] = {A(0.25), A(0.5), A(0.25)};
    A c[NC];
#pragma unroll
    for (int m = 0; m < NC; ++m) c[m] = A(0.0);
#pragma unroll
    for (int round = 0; round < 3; ++round) {
        const int st = 3 * round + l;  // this lane's stencil node in this round
        A term[NC];
        if (act_e) {
            const int jb = st / 3, ja = st - 3 * jb;
            const int kf = (e.b + jb - 1) * Lf.nx + (e.a + ja - 1);
            stencil_term<StF>(Lf, kf, ww[ja] * ww[jb], term);
        } else {
#pragma unroll
            for (int m = 0; m < NC; ++m) term[m] = A(0.0);
        }
#pragma unroll
        for (int m = 0; m < NC; ++m)
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                    const A v = __shfl_sync(0xffffffffu, term[m], base + q);
                    c[m] = (round == 0 && q == 0) ? v : c[m] + v;
                }
    }
    if (!act_e || l != 0) return;
    const Xi<A> xi = xi_dev ? xi_dev[blk] : xi_h;
    const A rho = c[0], ux = c[1], uy = c[2], tt = c[3];
    A fn[Q], fr[Q], f[Q], g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) fn[i] = c[4 + i];
    rescale<A, SH, true>(fn, xi, fr);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        f[i] = feq_st<A, SH>(i, rho, ux, uy) + fr[i];
        if constexpr (SH)
            g[i] = geq_full<A>(i, tt, ux, uy, 2) + c[13 + i] * xi.inv_th;
        else
            g[i] = geq_full<A>(i, tt, ux, uy, 2) + c[13 + i] / xi.th;
    }
    store_pops<StC, true>(Lc.ref_out, Lc.n, e.kc, f, g, true, seed, sidx * 16 + phase, (long long)Lc.node_off + e.kc);
    const Macro<A, SH> m = refresh<A, SH, true>(f, g);
    Lc.mac[e.kc] = SH ? m.drho : m.rho;
    Lc.mac[Lc.n + e.kc] = m.ux;
    Lc.mac[2 * Lc.n + e.kc] = m.uy;
    Lc.mac[3 * Lc.n + e.kc] = m.t;
    if (!collide) return;
    A fy_new;
    oct_collide<A, SH>(f, g, m, sc, fy_new);
    Lc.fy[e.kc] = fy_new;
    store_pops<StC>(Lc.pc_out, Lc.n, e.kc, f, g, true, seed, sidx * 16 + phase + 1, (long long)Lc.node_off + e.kc);
}

// ---------------------------------------------------------------------------
// Dynamic model: rescaling factors from the mean effective relaxation times
// (step_cavity, src/octree/solver.rs:690-711 for xi A and :808-829 for xi B):
// tau_eff = RelaxTimes::from_nu_alpha(nu + mean nu_t, alpha + mean alpha_t),
// xi = rescaling_factors_multilevel(tau_eff coarser, tau_eff finer, 2,
// odd_exact).  One CTA: each view's means in a fixed order, then thread 0.
// ---------------------------------------------------------------------------
template <class A>
struct MeanView {
    const A* nut;
    const A* at;
    int n;
};
template <class A>
struct XiJob {
    MeanView<A> v[4];
    int mode;  // 0: xi A from v0 (L0) and v1 + v2 (both L1 blocks); 1: xi B of block b from v[b] (L1), v[2 + b] (L2)
    double nu_c, al_c, nu_f, al_f;  // molecular nu / alpha of the coarser and finer level (ramped)
    int odd_exact;
};

__device__ __forceinline__ void relax_of(double nu, double al, double& tp, double& tm, double& tt) {
    tp = 0.5 + 3.0 * nu;
    tm = 0.5 + LAMBDA_TRT / (tp - 0.5);
    tt = 0.5 + 3.0 * al;
}

constexpr int DYN_PARTS = 64;  // CTAs of the dynamic model's reductions (fixed partition)

// Fixed-order sum of a CTA's 256 values (deterministic).
__device__ __forceinline__ double cta_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}
__device__ __forceinline__ double cta_max(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// Partial sums of nu_t and alpha_t: CTA (b, v) sums chunk b of view v into
// part[(v * DYN_PARTS + b) * 2 + {0, 1}].
template <class A>
__global__ void __launch_bounds__(256) k_oct_mean_parts(XiJob<A> J, double* __restrict__ part) {
    __shared__ double sh[256];
    const MeanView<A> V = J.v[blockIdx.y];
    const int chunk = (V.n + DYN_PARTS - 1) / DYN_PARTS;
    const int k0 = blockIdx.x * chunk, k1 = min(V.n, k0 + chunk);
    double a = 0.0, b = 0.0;
    for (int k = k0 + threadIdx.x; k < k1; k += 256) {
        a += double(V.nut[k]);
        b += double(V.at[k]);
    }
    a = cta_sum(a, sh);
    b = cta_sum(b, sh);
    if (threadIdx.x == 0) {
        part[(blockIdx.y * DYN_PARTS + blockIdx.x) * 2 + 0] = a;
        part[(blockIdx.y * DYN_PARTS + blockIdx.x) * 2 + 1] = b;
    }
}

template <class A>
__global__ void k_oct_xi(XiJob<A> J, const double* __restrict__ part, Xi<A>* __restrict__ xi_out,
                         double* __restrict__ xi_log) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nv = J.mode == 0 ? 3 : 4;
    double mean[4][2];
    for (int v = 0; v < nv; ++v) {
        double a = 0.0, b = 0.0;
        for (int c = 0; c < DYN_PARTS; ++c) {
            a += part[(v * DYN_PARTS + c) * 2 + 0];
            b += part[(v * DYN_PARTS + c) * 2 + 1];
        }
        mean[v][0] = a / double(J.v[v].n);
        mean[v][1] = b / double(J.v[v].n);
    }
    const int nxi = J.mode == 0 ? 1 : 2;
    for (int b = 0; b < nxi; ++b) {
        double ntc, atc, ntf, atf;
        if (J.mode == 0) {
            ntc = mean[0][0];
            atc = mean[0][1];
            ntf = (0.0 + mean[1][0] + mean[2][0]) / 2.0;
            atf = (0.0 + mean[1][1] + mean[2][1]) / 2.0;
        } else {
            ntc = mean[b][0];
            atc = mean[b][1];
            ntf = mean[2 + b][0];
            atf = mean[2 + b][1];
        }
        double tpc, tmc, ttc, tpf, tmf, ttf;
        relax_of(J.nu_c + ntc, J.al_c + atc, tpc, tmc, ttc);
        relax_of(J.nu_f + ntf, J.al_f + atf, tpf, tmf, ttf);
        const double dt = 1.0 / 2.0;
        const double x[3] = {dt * tpf / tpc, J.odd_exact ? dt * tmf / tmc : dt, dt * ttf / ttc};
        Xi<A> o;
        o.even = A(x[0]);
        o.odd = A(x[1]);
        o.th = A(x[2]);
        o.inv_even = A(1.0 / x[0]);
        o.inv_odd = A(1.0 / x[1]);
        o.inv_th = A(1.0 / x[2]);
        const int slot = J.mode == 0 ? 0 : b;
        xi_out[slot] = o;
        if (J.mode == 0) xi_out[1] = o;
        for (int i = 0; i < 3; ++i) xi_log[3 * slot + i] = x[i];
    }
}

// Partial statistics of the L0 model's Lilly coefficients (cs_dyn_mean /
// _max, kappa_dyn_mean / _max, src/octree/smag.rs:369-378): CTA b writes
// sum / max of C_nu and of C_kappa over chunk b; the host adds the parts in
// order.
static __global__ void __launch_bounds__(256) k_oct_sgs_parts(const double* __restrict__ W, int n,
                                                              double* __restrict__ part) {
    __shared__ double sh[256];
    const long long P = n;
    const int chunk = (n + DYN_PARTS - 1) / DYN_PARTS;
    const int k0 = blockIdx.x * chunk, k1 = min(n, k0 + chunk);
    double s0 = 0.0, m0 = 0.0, s1 = 0.0, m1 = 0.0;
    for (int k = k0 + threadIdx.x; k < k1; k += 256) {
        const double a = W[S_CNU * P + k], b = W[S_CK * P + k];
        s0 += a;
        m0 = fmax(m0, a);
        s1 += b;
        m1 = fmax(m1, b);
    }
    s0 = cta_sum(s0, sh);
    m0 = cta_max(m0, sh);
    s1 = cta_sum(s1, sh);
    m1 = cta_max(m1, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 4 + 0] = s0;
        part[blockIdx.x * 4 + 1] = m0;
        part[blockIdx.x * 4 + 2] = s1;
        part[blockIdx.x * 4 + 3] = m1;
    }
}

// nu_t_max (src/octree/solver.rs:918-933): max |nu_t| over every level.
template <class A>
__global__ void __launch_bounds__(256) k_oct_nutmax(MeanView<A> v0, MeanView<A> v1, MeanView<A> v2, MeanView<A> v3,
                                                    MeanView<A> v4, int nv, double* __restrict__ out) {
    __shared__ double sh[256];
    const MeanView<A> V[5] = {v0, v1, v2, v3, v4};
    double m = 0.0;
    for (int v = 0; v < nv; ++v)
        for (int k = threadIdx.x; k < V[v].n; k += 256) m = fmax(m, fabs(double(V[v].nut[k])));
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// ---------------------------------------------------------------------------
// Diagnostics (FP64, deterministic: fixed CTA partition, sequential final sums).
// ---------------------------------------------------------------------------
template <class A>
struct StatView {
    const A* mac;
    int n;
};
template <class A>
struct StatViews {
    StatView<A> v[5];
};

// Per CTA of view blockIdx.y: min / max of rho, max max(|ux|, |uy|) (max_u,
// src/octree/cavity.rs:743-748), count of non-finite moments
// (check_finite_levels, :751-789), sum of the rho plane.
template <class A, bool SHIFT>
__global__ void __launch_bounds__(256) k_oct_stats(StatViews<A> V, double* __restrict__ part) {
    const StatView<A> W = V.v[blockIdx.y];
    double mn = 1e300, mx = -1e300, mu = 0.0, nf = 0.0, sm = 0.0;
    for (int k = blockIdx.x * 256 + threadIdx.x; k < W.n; k += gridDim.x * 256) {
        const double r0 = double(W.mac[k]);
        const double r = SHIFT ? 1.0 + r0 : r0;
        const double u = double(W.mac[W.n + k]), v = double(W.mac[2 * W.n + k]), t = double(W.mac[3 * W.n + k]);
        mn = fmin(mn, r);
        mx = fmax(mx, r);
        mu = fmax(mu, fmax(fabs(u), fabs(v)));
        if (!(isfinite(r) && isfinite(u) && isfinite(v) && isfinite(t))) nf += 1.0;
        sm += r0;
    }
    __shared__ double sh[OSTAT][256];
    sh[0][threadIdx.x] = mn;
    sh[1][threadIdx.x] = mx;
    sh[2][threadIdx.x] = mu;
    sh[3][threadIdx.x] = nf;
    sh[4][threadIdx.x] = sm;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            const int o = threadIdx.x + h;
            sh[0][threadIdx.x] = fmin(sh[0][threadIdx.x], sh[0][o]);
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][o]);
            sh[2][threadIdx.x] = fmax(sh[2][threadIdx.x], sh[2][o]);
            sh[3][threadIdx.x] += sh[3][o];
            sh[4][threadIdx.x] += sh[4][o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* p = part + (size_t(blockIdx.y) * gridDim.x + blockIdx.x) * OSTAT;
        for (int q = 0; q < 5; ++q) p[q] = sh[q][0];
        p[5] = 0.0;
    }
}

// min / max of rho over the interface nodes (noise_stats, src/octree/
// solver.rs:954-1003): ghosts of each finer level and coincident nodes of
// each coarser level.  One CTA per (list, block).
template <class A, bool SHIFT>
__global__ void __launch_bounds__(256) k_oct_iface(const A* mac_f0, const A* mac_f1, const A* mac_c0, const A* mac_c1,
                                                   const GhostE<A>* __restrict__ gh, int n_ghost,
                                                   const CoinE* __restrict__ co, int n0, int n1,
                                                   double* __restrict__ out) {
    const int blk = blockIdx.x;
    const A* mf = blk == 0 ? mac_f0 : mac_f1;
    const A* mc = blk == 0 ? mac_c0 : mac_c1;
    double mn = 1e300, mx = -1e300;
    for (int j = threadIdx.x; j < n_ghost; j += 256) {
        const double r0 = double(mf[gh[blk * n_ghost + j].kf]);
        const double r = SHIFT ? 1.0 + r0 : r0;
        mn = fmin(mn, r);
        mx = fmax(mx, r);
    }
    const int nc = blk == 0 ? n0 : n1;
    const CoinE* cb = co + (blk == 0 ? 0 : n0);
    for (int j = threadIdx.x; j < nc; j += 256) {
        const double r0 = double(mc[cb[j].kc]);
        const double r = SHIFT ? 1.0 + r0 : r0;
        mn = fmin(mn, r);
        mx = fmax(mx, r);
    }
    __shared__ double s0[256], s1[256];
    s0[threadIdx.x] = mn;
    s1[threadIdx.x] = mx;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            s0[threadIdx.x] = fmin(s0[threadIdx.x], s0[threadIdx.x + h]);
            s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * blk] = s0[0];
        out[2 * blk + 1] = s1[0];
    }
}

// Per-row terms of the Nusselt and y+ estimators, one thread per row, into
// rows[5][R] (summed in row order by k_oct_final).
template <class A>
__global__ void __launch_bounds__(256) k_oct_rows(const A* __restrict__ mac0, int nx0, int ny0,
                                                  const A* __restrict__ mac_h1, int nx1, int ny1,
                                                  const A* __restrict__ mac_fin, int nxf, int nyf, double nu_fin,
                                                  double* __restrict__ rows, int R) {
    const int r = blockIdx.x * 256 + threadIdx.x;
    if (r < ny0) {
        const A* T0 = mac0 + 3 * (size_t)nx0 * ny0;
        const double t0 = T0[r * nx0], t1 = T0[r * nx0 + 1], t2 = T0[r * nx0 + 2];
        const double tc2 = T0[r * nx0 + nx0 - 2], tc3 = T0[r * nx0 + nx0 - 3];
        rows[r] = fabs(t1 - t2);
        rows[R + r] = fabs(t1 - t0);
        rows[2 * R + r] = fabs(tc2 - tc3);
    }
    if (r >= 1 && r < ny1 - 1) {
        const A* T1 = mac_h1 + 3 * (size_t)nx1 * ny1;
        rows[3 * R + r] = fabs(double(T1[r * nx1 + 1]) - double(T1[r * nx1 + 2])) * 2.0;
    }
    if (r >= 2 && r < nyf - 2) {
        const A* Uy = mac_fin + 2 * (size_t)nxf * nyf;
        const double tw = nu_fin * fabs(double(Uy[r * nxf + 2]) - double(Uy[r * nxf + 1]));
        rows[4 * R + r] = 0.5 * sqrt(fmax(tw, 0.0)) / nu_fin;
    }
}

// Final reduction.  out: nu_hot, nu_hot_link0, nu_cold (nusselt_hot /
// nusselt_hot_link0 / nusselt_cold, src/octree/cavity.rs:672-715, Lx
// scale), nu_hot_fine (:728-741), max_u, mass (mean coarse rho), max_rho_dev,
// max_rho_dev_ifaces, finite, y_plus (post.rs:182-199 formula on the finest
// hot-wall level: wall column 1, first fluid column 2, rows 2..ny-3).
// Row sums in row order, as the reference.
// Sum of a[lo..hi) in index order, computed by a whole warp: coalesced
// loads of 32 values, then every lane adds them one by one.
__device__ __forceinline__ double warp_ordered_sum(const double* __restrict__ a, int lo, int hi) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    bool first = true;
    for (int b = lo; b < hi; b += 32) {
        const double v = b + lane < hi ? a[b + lane] : 0.0;
        const int nv = hi - b < 32 ? hi - b : 32;
        for (int j = 0; j < nv; ++j) {
            const double x = __shfl_sync(0xffffffffu, v, j);
            s = first ? x : s + x;
            first = false;
        }
    }
    return s;
}

template <bool SHIFT>
__global__ void k_oct_final(const double* __restrict__ rows, int R, int nx0, int ny0, int ny1, int nyf, int n0,
                            const double* __restrict__ part, int n_views, int n_ctas,
                            const double* __restrict__ iface, int n_iface, double* __restrict__ out) {
    // one warp; FP64 row sums in row order (bit-identical to the reference's loops)
    const double sh = warp_ordered_sum(rows, 0, ny0);
    const double s0 = warp_ordered_sum(rows + R, 0, ny0);
    const double sc = warp_ordered_sum(rows + 2 * R, 0, ny0);
    const double sf = warp_ordered_sum(rows + 3 * R, 1, ny1 - 1);
    const double sy = warp_ordered_sum(rows + 4 * R, 2, nyf - 2);
    if (threadIdx.x != 0) return;
    const double lx = double(nx0 - 1);
    out[0] = sh / double(ny0) * lx / 1.0;
    out[1] = s0 / double(ny0) * lx / 1.0;
    out[2] = sc / double(ny0) * lx / 1.0;
    out[3] = sf / double(ny1 - 2) * lx / 1.0;
    double mn = 1e300, mx = -1e300, mu = 0.0, nf = 0.0, sum0 = 0.0;
    for (int v = 0; v < n_views; ++v)
        for (int c = 0; c < n_ctas; ++c) {
            const double* p = part + (size_t(v) * n_ctas + c) * OSTAT;
            mn = fmin(mn, p[0]);
            mx = fmax(mx, p[1]);
            mu = fmax(mu, p[2]);
            nf += p[3];
            if (v == 0) sum0 += p[4];
        }
    out[4] = mu;
    const double rb = SHIFT ? 1.0 + sum0 / double(n0) : sum0 / double(n0);
    out[5] = rb;
    out[6] = fmax(mx - rb, rb - mn);
    double imn = 1e300, imx = -1e300;
    for (int j = 0; j < n_iface; ++j) {
        imn = fmin(imn, iface[2 * j]);
        imx = fmax(imx, iface[2 * j + 1]);
    }
    out[7] = fmax(imx - rb, rb - imn);
    out[8] = nf == 0.0 ? 1.0 : 0.0;
    out[9] = sy / double(nyf - 4);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------

// The octree behind cav_octree_*; OctImpl<StC, StF> holds the buffers.
struct Octree {
    virtual ~Octree() = default;
    virtual void setup(const cav_octree_params& p) = 0;
    virtual void step(int64_t n) = 0;
    virtual void get_level(int lvl, double* rho, double* ux, double* uy, double* t, double* f, double* g) = 0;
    virtual void set_level(int lvl, const double* rho, const double* ux, const double* uy, const double* t,
                           const double* f, const double* g) = 0;
    virtual void diag(double* out10) = 0;
    virtual void debug_phase(int phase) = 0;
    virtual void restart_level(int lvl, const double* rho, const double* ux, const double* uy, const double* t) = 0;
    virtual void set_time_step(int64_t t) = 0;
    virtual void sync() = 0;
    virtual void set_dynamic_sgs(bool on, double smag_alpha, double nu_sm_min, double eta_test) = 0;
    virtual void dynamic_stats(double* out14) = 0;
    virtual void get_nut(int lvl, double* nut, double* at) = 0;
    virtual void set_level_kernel(int kind) = 0;
    virtual int get_level_kernel() const = 0;

    cav_octree_params p{};
    int levels = 2, nx0 = 0, ny0 = 0, nx1 = 0, ny1 = 0, nx2 = 0, ny2 = 0;
    double nu = 0, alpha = 0, beta_c = 0, nu_start_mult = 1.0;
    double tau_p[3] = {0, 0, 0};
    double xiA[3] = {0, 0, 0}, xiB[3] = {0, 0, 0};
    int64_t time_step = 0, spin_up = 0;
    int n_ghost = 0, n_co0 = 0, n_co1 = 0, n_ghost2 = 0, n_co2_0 = 0, n_co2_1 = 0;
    cudaStream_t stream = nullptr;
    int64_t launches = 0;
    std::string err;
};

// Host restatement of the grid tables (OctreeGrid::build, grid.rs:103-204,
// bilinear_stencil :218-229), in FP64.
struct HostGrid {
    int nx0, ny0, bx0, by0, bx1, by1, nx1, ny1;
    struct G {
        int kf;
        int kc[4];
        double w[4];
    };
    std::vector<G> ghosts;
    std::vector<CoinE> coin;
    static void bilinear(double x, double y, int nx0, int ny0, int kc[4], double w[4]) {
        long ix = (long)std::floor(x), iy = (long)std::floor(y);
        ix = std::min<long>(std::max<long>(ix, 0), nx0 - 2);
        iy = std::min<long>(std::max<long>(iy, 0), ny0 - 2);
        const double fx = x - double(ix), fy = y - double(iy);
        kc[0] = int(iy * nx0 + ix);
        w[0] = (1.0 - fx) * (1.0 - fy);
        kc[1] = int(iy * nx0 + ix + 1);
        w[1] = fx * (1.0 - fy);
        kc[2] = int((iy + 1) * nx0 + ix);
        w[2] = (1.0 - fx) * fy;
        kc[3] = int((iy + 1) * nx0 + ix + 1);
        w[3] = fx * fy;
    }
    void build(int nx0_, int ny0_, int bx0_, int by0_, int bx1_, int by1_, bool wl, bool wr, bool wb, bool wt) {
        nx0 = nx0_;
        ny0 = ny0_;
        bx0 = bx0_;
        by0 = by0_;
        bx1 = bx1_;
        by1 = by1_;
        nx1 = 2 * (bx1 - bx0) + 3;
        ny1 = 2 * (by1 - by0) + 3;
        ghosts.clear();
        coin.clear();
        for (int b = 0; b < ny1; ++b)
            for (int a = 0; a < nx1; ++a)
                if (a == 0 || b == 0 || a == nx1 - 1 || b == ny1 - 1) {
                    G e;
                    e.kf = b * nx1 + a;
                    bilinear(double(bx0) - 0.5 + 0.5 * a, double(by0) - 0.5 + 0.5 * b, nx0, ny0, e.kc, e.w);
                    ghosts.push_back(e);
                }
        for (int cy = by0; cy < by1; ++cy)
            for (int cx = bx0; cx < bx1; ++cx) {
                if (cx == 0 || cx + 1 == nx0 || cy == 0 || cy + 1 == ny0) continue;
                if ((wl && cx == bx0) || (wr && cx + 1 == bx1) || (wb && cy == by0) || (wt && cy + 1 == by1)) continue;
                coin.push_back(CoinE{cy * nx0 + cx, 2 * (cx - bx0) + 1, 2 * (cy - by0) + 1});
            }
    }
};

template <class StC, class StF>
struct OctImpl final : Octree {
    using A = typename Fmt<StC>::A;
    static_assert(std::is_same<A, typename Fmt<StF>::A>::value, "one arithmetic type");
    static constexpr bool SH = Fmt<StC>::SHIFT;

    template <class St>
    struct Lvl {
        int nx = 0, ny = 0, n = 0;
        St* ref[2] = {nullptr, nullptr};
        St* pc[2] = {nullptr, nullptr};
        A* mac = nullptr;
        A* fy = nullptr;
        int hot = 0, cold = 0, node_off = 0;
        int cur = 0;  // REF and PC buffers flip together
        LvlIO<St> io() const {
            LvlIO<St> o;
            o.ref_in = ref[cur];
            o.ref_out = ref[cur ^ 1];
            o.pc_in = pc[cur];
            o.pc_out = pc[cur ^ 1];
            o.mac = mac;
            o.fy = fy;
            o.nx = nx;
            o.ny = ny;
            o.n = n;
            o.hot = hot;
            o.cold = cold;
            o.node_off = node_off;
            return o;
        }
        // The current state: REF and PC written by the last step (the
        // couplings read and write this one).
        LvlIO<St> io_cur() const {
            LvlIO<St> o = io();
            o.ref_in = ref[cur];
            o.ref_out = ref[cur];
            o.pc_in = pc[cur];
            o.pc_out = pc[cur];
            return o;
        }
    };

    Lvl<StC> L0;
    Lvl<StF> L1[2], L2[2];
    GhostE<A>* gh1 = nullptr;
    GhostE<A>* gh2 = nullptr;
    CoinE* co1 = nullptr;
    CoinE* co2 = nullptr;
    OctScal<A>* tab = nullptr;
    int S = 0;
    long long* step_dev = nullptr;
    long long step_dev_val = -1;
    double* part = nullptr;
    double* iface = nullptr;
    double* dout = nullptr;
    double* rowbuf = nullptr;
    uint32_t seed32 = 0;
    bool pc_valid = false;
    Xi<A> xa{}, xb{};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int level_kernel = CAV_OCT_LEVEL_FG;  // fine-level step form (step_fine)
    // dynamic mixed-scale SGS model (set_dynamic_sgs, src/octree/solver.rs:476-481)
    bool dyn = false;
    double dyn_alpha = 0.5, dyn_min = -0.1, dyn_eta = 2.0;
    double* sgs_w = nullptr;              // 2 x S_NPLANES work planes of the largest level
    size_t sgs_stride = 0;                // elements of one block's work planes
    A* nut0 = nullptr;                    // nu_t_pre, then alpha_t_pre, of L0
    A* nut1[2] = {nullptr, nullptr};      // of the L1 blocks
    A* nut2[2] = {nullptr, nullptr};      // of the L2 strips
    Xi<A>* xi_dev = nullptr;              // xi A (slots 0, 1), xi B hot / cold (slots 2, 3)
    bool xi_dyn = false;                  // xi_dev holds the factors in use (a dynamic step ran)
    double* dstat = nullptr;              // cs / kappa mean, max; nu_t_max; xi A, xi B hot, xi B cold
    double* mpart = nullptr;              // partial sums of the xi means (4 views x DYN_PARTS x 2)
    double* spart = nullptr;              // partial statistics of the L0 model (DYN_PARTS x 4)
    cudaGraphExec_t dgraph[2] = {nullptr, nullptr};  // OCT_GRAPH_STEPS dynamic coarse steps
    std::vector<void*> allocs;

    ~OctImpl() override {
        for (auto& gx : graph)
            if (gx) cudaGraphExecDestroy(gx);
        for (auto& gx : dgraph)
            if (gx) cudaGraphExecDestroy(gx);
        for (void* b : allocs) cudaFree(b);
        if (stream) cudaStreamDestroy(stream);
    }

    template <class T>
    T* dalloc(size_t n) {
        void* p = nullptr;
        CK(cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)));
        allocs.push_back(p);
        CK(cudaMemsetAsync(p, 0, sizeof(T) * std::max<size_t>(n, 1), stream));
        return static_cast<T*>(p);
    }

    template <class St>
    void alloc_level(Lvl<St>& L, int nx, int ny, int hot, int cold, int node_off) {
        L.nx = nx;
        L.ny = ny;
        L.n = nx * ny;
        L.hot = hot;
        L.cold = cold;
        L.node_off = node_off;
        for (int b = 0; b < 2; ++b) {
            L.ref[b] = dalloc<St>(size_t(NPLANES) * L.n);
            L.pc[b] = dalloc<St>(size_t(NPLANES) * L.n);
        }
        L.mac = dalloc<A>(size_t(4) * L.n);
        L.fy = dalloc<A>(L.n);
    }

    static Xi<A> make_xi(const double* x) {
        Xi<A> o;
        o.even = A(x[0]);
        o.odd = A(x[1]);
        o.th = A(x[2]);
        o.inv_even = A(1.0 / x[0]);
        o.inv_odd = A(1.0 / x[1]);
        o.inv_th = A(1.0 / x[2]);
        return o;
    }

    // RelaxTimes::from_nu_alpha (lbm.rs:90-98) + collision coefficients.
    LvlScal<A> lvl_scal(double nu_l, double al_l, double beta) const {
        const double tp = 0.5 + 3.0 * nu_l;
        const double tm = 0.5 + LAMBDA_TRT / (tp - 0.5);
        const double tt = 0.5 + 3.0 * al_l;
        LvlScal<A> c;
        c.a_f = A(0.5 * (1.0 / tp + 1.0 / tm));
        c.b_f = A(0.5 * (1.0 / tp - 1.0 / tm));
        c.a_g = A(1.0 / tt);
        c.c_m = A(1.0 - 0.5 / tm);
        c.c_p = A(1.0 - 0.5 / tp);
        c.om_p = A(1.0 / tp);
        c.om_m = A(1.0 / tm);
        c.om_g = A(1.0 / tt);
        c.k_p = A(1.0 - 0.5 / tp);
        c.k_m = A(1.0 - 0.5 / tm);
        c.beta = A(beta);
        c.tp = A(tp);
        c.tt = A(tt);
        const double ts = 0.5 + 3.0 * std::fmax(nu_l, 0.002 / 3.0);
        c.cs = A(p.cs);
        c.nu = A(nu_l);
        c.alpha = A(al_l);
        c.tau_s = A(ts);
        c.inv_tau_s = A(1.0 / ts);
        c.pr_t = A(p.pr_t);
        c.inv_pr_t = A(1.0 / p.pr_t);
        return c;
    }

    // ramp_nu_alpha / ramp_beta_factor (src/octree/solver.rs:596-617) and the
    // per-level tau / beta of step_cavity (:653-656, 718, 751-753).
    OctScal<A> row(int64_t s) const {
        double nu_eff = nu, al_eff = alpha, br = 1.0;
        if (nu_start_mult != 1.0) {
            const double m = 1.0 + (nu_start_mult - 1.0) * std::exp(-double(s) / 1000.0);
            nu_eff = nu * m;
            al_eff = alpha * m;
            if (s < spin_up) br = double(s) / double(spin_up);
        }
        OctScal<A> r;
        r.l[0] = lvl_scal(nu_eff, al_eff, beta_c * br);
        r.l[1] = lvl_scal(2.0 * nu_eff, 2.0 * al_eff, (0.5 * beta_c) * br);
        r.l[2] = lvl_scal(4.0 * nu_eff, 4.0 * al_eff, 0.25 * beta_c * br);
        return r;
    }

    void setup(const cav_octree_params& pp) override {
        p = pp;
        if (p.bl_width < 2) throw ArgError{CAV_ERR_ARG, "bl_width >= 2 required"};
        if (!(2 * p.bl_width < p.nx0)) throw ArgError{CAV_ERR_ARG, "2 * bl_width < nx0 required (coarse core)"};
        if (p.levels != 2 && p.levels != 3) throw ArgError{CAV_ERR_ARG, "levels must be 2 or 3"};
        if (p.ny0 < 4) throw ArgError{CAV_ERR_ARG, "ny0 >= 4 required"};
        // node kernels split k into (x, y) in FP32 (exact below 2^22 nodes)
        if ((long long)p.nx0 * p.ny0 >= (1ll << 22) || (long long)p.ny0 * 4 * (2 * p.bl_width + 3) >= (1ll << 22))
            throw ArgError{CAV_ERR_ARG, "grid too large: every level must stay below 2^22 nodes"};
        if (!(p.ra > 0 && p.pr > 0 && p.utarget > 0)) throw ArgError{CAV_ERR_ARG, "ra, pr, utarget must be > 0"};
        if (!(p.cs >= 0.0 && p.cs < 1.0) || !(p.pr_t > 0.0)) throw ArgError{CAV_ERR_ARG, "cs in [0, 1), pr_t > 0"};
        levels = p.levels;
        nx0 = p.nx0;
        ny0 = p.ny0;
        // CavitySolver::new, src/octree/solver.rs:298-336.
        const double lz = double(ny0 - 1);
        const double nu_cal = std::pow(p.utarget * std::sqrt(p.pr) * lz / (1.7 * std::sqrt(p.ra)), 2.0 / 3.0);
        if (p.has_nu_override) {
            if (!(p.nu_override > 0.0 && std::isfinite(p.nu_override)))
                throw ArgError{CAV_ERR_ARG, "nu must be > 0 and finite"};
            nu = p.nu_override;
        } else {
            nu = std::fmax(nu_cal, 0.002);
        }
        alpha = nu / p.pr;
        beta_c = p.ra * nu * alpha / (lz * lz * lz);
        nu_start_mult = std::max(p.nu_start_mult, 1.0);
        spin_up = std::max<int64_t>(ny0 / 10, 2000);
        for (int l = 0; l < 3; ++l) tau_p[l] = 0.5 + 3.0 * (double(1 << l) * nu);
        auto xi_of = [&](int lc) {
            // rescaling_factors_multilevel(tau(lc), tau(lc + 1), 2, odd_exact)
            const double nc = lc == 0 ? nu : 2.0 * nu, ncf = lc == 0 ? 2.0 * nu : 4.0 * nu;
            const double ac = lc == 0 ? alpha : 2.0 * alpha, acf = lc == 0 ? 2.0 * alpha : 4.0 * alpha;
            const double tpc = 0.5 + 3.0 * nc, tpf = 0.5 + 3.0 * ncf;
            const double tmc = 0.5 + LAMBDA_TRT / (tpc - 0.5), tmf = 0.5 + LAMBDA_TRT / (tpf - 0.5);
            const double ttc = 0.5 + 3.0 * ac, ttf = 0.5 + 3.0 * acf;
            const double dt = 1.0 / 2.0;
            std::array<double, 3> x{dt * tpf / tpc, p.odd_exact ? dt * tmf / tmc : dt, dt * ttf / ttc};
            return x;
        };
        const auto a = xi_of(0), b = xi_of(1);
        for (int i = 0; i < 3; ++i) {
            xiA[i] = a[i];
            xiB[i] = b[i];
        }
        xa = make_xi(xiA);
        xb = make_xi(xiB);
        seed32 = uint32_t(p.seed) ^ uint32_t(p.seed >> 32) ^ 0x27d4eb2fu;

        // grids (src/octree/solver.rs:356-431)
        const int blw = p.bl_width;
        HostGrid g1[2], g2[2];
        const int spec[2][2] = {{0, blw}, {nx0 - 1 - blw, nx0 - 1}};
        for (int b = 0; b < 2; ++b) g1[b].build(nx0, ny0, spec[b][0], 0, spec[b][1], ny0 - 1, false, false, false, false);
        nx1 = g1[0].nx1;
        ny1 = g1[0].ny1;
        if (levels == 3) {
            for (int b = 0; b < 2; ++b) {
                const int sbx0 = b == 0 ? 1 : nx1 - 4, sbx1 = b == 0 ? 3 : nx1 - 2;
                g2[b].build(nx1, ny1, sbx0, 1, sbx1, ny1 - 2, true, false, true, false);
            }
            nx2 = g2[0].nx1;
            ny2 = g2[0].ny1;
        }

        CK(cudaSetDevice(p.device));
        CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        alloc_level(L0, nx0, ny0, 1, 1, 0);
        int off = nx0 * ny0;
        for (int b = 0; b < 2; ++b) {
            alloc_level(L1[b], nx1, ny1, b == 0, b == 1, off);
            off += nx1 * ny1;
        }
        if (levels == 3)
            for (int b = 0; b < 2; ++b) {
                alloc_level(L2[b], nx2, ny2, b == 0, b == 1, off);
                off += nx2 * ny2;
            }

        // tables
        auto upload_ghosts = [&](HostGrid* g, GhostE<A>*& dst, int& ng) {
            ng = int(g[0].ghosts.size());
            std::vector<GhostE<A>> h(2 * size_t(ng));
            for (int b = 0; b < 2; ++b)
                for (int j = 0; j < ng; ++j) {
                    const auto& e = g[b].ghosts[j];
                    GhostE<A>& o = h[size_t(b) * ng + j];
                    o.kf = e.kf;
                    for (int s = 0; s < 4; ++s) {
                        o.kc[s] = e.kc[s];
                        o.w[s] = A(e.w[s]);
                    }
                }
            dst = dalloc<GhostE<A>>(h.size());
            CK(cudaMemcpyAsync(dst, h.data(), sizeof(GhostE<A>) * h.size(), cudaMemcpyHostToDevice, stream));
            CK(cudaStreamSynchronize(stream));
        };
        auto upload_coin = [&](HostGrid* g, CoinE*& dst, int& c0, int& c1) {
            c0 = int(g[0].coin.size());
            c1 = int(g[1].coin.size());
            std::vector<CoinE> h(g[0].coin);
            h.insert(h.end(), g[1].coin.begin(), g[1].coin.end());
            dst = dalloc<CoinE>(h.size());
            CK(cudaMemcpyAsync(dst, h.data(), sizeof(CoinE) * h.size(), cudaMemcpyHostToDevice, stream));
            CK(cudaStreamSynchronize(stream));
        };
        upload_ghosts(g1, gh1, n_ghost);
        upload_coin(g1, co1, n_co0, n_co1);
        if (levels == 3) {
            upload_ghosts(g2, gh2, n_ghost2);
            upload_coin(g2, co2, n_co2_0, n_co2_1);
        }

        // per-step table: rows until the ramps have converged bit for bit
        std::vector<OctScal<A>> rows;
        rows.push_back(row(0));
        if (nu_start_mult != 1.0) {
            for (int64_t s = 1;; ++s) {
                const double m = 1.0 + (nu_start_mult - 1.0) * std::exp(-double(s) / 1000.0);
                rows.push_back(row(s));
                if (m == 1.0 && s >= spin_up) break;
                if (s > 4000000) throw ArgError{CAV_ERR_ARG, "viscosity ramp does not converge"};
            }
        }
        S = int(rows.size()) - 1;
        tab = dalloc<OctScal<A>>(rows.size());
        CK(cudaMemcpyAsync(tab, rows.data(), sizeof(OctScal<A>) * rows.size(), cudaMemcpyHostToDevice, stream));
        step_dev = dalloc<long long>(1);
        part = dalloc<double>(size_t(5) * OSTAT_CTAS * OSTAT);
        iface = dalloc<double>(8);
        dout = dalloc<double>(16);
        rowbuf = dalloc<double>(size_t(5) * std::max(std::max(ny0, ny1), levels == 3 ? ny2 : 0));
        CK(cudaStreamSynchronize(stream));
        init_cavity();
    }

    // init_cavity, src/octree/solver.rs:504-578.
    void init_cavity() {
        Rng rng(p.seed);
        const size_t n0 = size_t(nx0) * ny0;
        std::vector<double> t0(n0);
        for (int iy = 0; iy < ny0; ++iy)
            for (int ix = 0; ix < nx0; ++ix) {
                const double xf = double(ix) / double(nx0 - 1);
                const double t_lin = T_HOT_C + (T_COLD_C - T_HOT_C) * xf;
                const double pert = 1.0e-3 * (2.0 * rng.next_f64() - 1.0);
                t0[size_t(iy) * nx0 + ix] = t_lin + pert;
            }
        upload_eq(L0, t0);
        auto interp = [&](double x, double y) {
            int kc[4];
            double w[4];
            HostGrid::bilinear(x, y, nx0, ny0, kc, w);
            double t = 0.0;
            for (int s = 0; s < 4; ++s) t += w[s] * t0[kc[s]];
            return t;
        };
        const int blw = p.bl_width;
        const int bx0s[2] = {0, nx0 - 1 - blw};
        for (int b = 0; b < 2; ++b) {
            std::vector<double> t1(size_t(nx1) * ny1);
            for (int yb = 0; yb < ny1; ++yb)
                for (int a = 0; a < nx1; ++a)
                    t1[size_t(yb) * nx1 + a] = interp(double(bx0s[b]) - 0.5 + 0.5 * a, -0.5 + 0.5 * yb);
            upload_eq(L1[b], t1);
            if (levels == 3) {
                const int sbx0 = b == 0 ? 1 : nx1 - 4;
                std::vector<double> t2(size_t(nx2) * ny2);
                for (int b2 = 0; b2 < ny2; ++b2)
                    for (int a2 = 0; a2 < nx2; ++a2) {
                        const double x = double(bx0s[b]) - 0.5 + 0.5 * (double(sbx0) - 0.5 + 0.5 * a2);
                        const double y = 0.0 - 0.5 + 0.5 * (1.0 - 0.5 + 0.5 * b2);
                        t2[size_t(b2) * nx2 + a2] = interp(x, y);
                    }
                upload_eq(L2[b], t2);
            }
        }
        time_step = 0;
        pc_valid = false;
    }

    // f = feq(1, 0, 0), g = geq(T, 0, 0), rho = 1, u = 0, fy = 0.
    template <class St>
    void upload_eq(Lvl<St>& L, const std::vector<double>& t) {
        const size_t n = size_t(L.n);
        std::vector<double> f(n * Q), g(n * Q), r(n, 1.0), z(n, 0.0);
        for (size_t k = 0; k < n; ++k)
            for (int i = 0; i < Q; ++i) {
                f[k * Q + i] = feq_full<double>(i, 1.0, 0.0, 0.0);
                g[k * Q + i] = geq_full<double>(i, t[k], 0.0, 0.0, 2);
            }
        upload_state(L, r.data(), z.data(), z.data(), t.data(), f.data(), g.data());
        CK(cudaMemsetAsync(L.fy, 0, sizeof(A) * n, stream));
        CK(cudaStreamSynchronize(stream));
    }

    template <class St>
    void upload_state(Lvl<St>& L, const double* r, const double* u, const double* v, const double* t, const double* f,
                      const double* g) {
        const size_t n = size_t(L.n);
        if (f || g) {
            std::vector<St> hp(NPLANES * n);
            CK(cudaMemcpyAsync(hp.data(), L.ref[L.cur], sizeof(St) * hp.size(), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            for (size_t k = 0; k < n; ++k)
                for (int i = 0; i < Q; ++i) {
                    if (f) hp[size_t(i) * n + k] = Fmt<St>::store(A(f[k * Q + i] - (SH ? WD(i) : 0.0)), i, RN_BITS);
                    if (g) hp[size_t(Q + i) * n + k] = Fmt<St>::store(A(g[k * Q + i]), Q + i, RN_BITS);
                }
            CK(cudaMemcpyAsync(L.ref[L.cur], hp.data(), sizeof(St) * hp.size(), cudaMemcpyHostToDevice, stream));
        }
        std::vector<A> hm(4 * n);
        CK(cudaMemcpyAsync(hm.data(), L.mac, sizeof(A) * hm.size(), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (size_t k = 0; k < n; ++k) {
            if (r) hm[k] = A(SH ? r[k] - 1.0 : r[k]);
            if (u) hm[n + k] = A(u[k]);
            if (v) hm[2 * n + k] = A(v[k]);
            if (t) hm[3 * n + k] = A(t[k]);
        }
        CK(cudaMemcpyAsync(L.mac, hm.data(), sizeof(A) * hm.size(), cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));
        pc_valid = false;
    }

    template <class St>
    void download_state(const Lvl<St>& L, double* r, double* u, double* v, double* t, double* f, double* g) {
        const size_t n = size_t(L.n);
        if (f || g) {
            std::vector<St> hp(NPLANES * n);
            CK(cudaMemcpyAsync(hp.data(), L.ref[L.cur], sizeof(St) * hp.size(), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            for (size_t k = 0; k < n; ++k)
                for (int i = 0; i < Q; ++i) {
                    if (f) f[k * Q + i] = double(Fmt<St>::load(hp[size_t(i) * n + k], i)) + (SH ? WD(i) : 0.0);
                    if (g) g[k * Q + i] = double(Fmt<St>::load(hp[size_t(Q + i) * n + k], Q + i));
                }
        }
        std::vector<A> hm(4 * n);
        CK(cudaMemcpyAsync(hm.data(), L.mac, sizeof(A) * hm.size(), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (size_t k = 0; k < n; ++k) {
            if (r) r[k] = SH ? 1.0 + double(hm[k]) : double(hm[k]);
            if (u) u[k] = double(hm[n + k]);
            if (v) v[k] = double(hm[2 * n + k]);
            if (t) t[k] = double(hm[3 * n + k]);
        }
    }

    void check_launch() {
        ++launches;
        CK(cudaGetLastError());
    }

    template <class St>
    static LvlPair<St> pair(const Lvl<St>& a, const Lvl<St>& b) {
        LvlPair<St> q;
        q.b[0] = a.io();
        q.b[1] = b.io();
        return q;
    }
    template <class St>
    static LvlPair<St> pair_cur(const Lvl<St>& a, const Lvl<St>& b) {
        LvlPair<St> q;
        q.b[0] = a.io_cur();
        q.b[1] = b.io_cur();
        return q;
    }
    static dim3 grid_of(int n, int nb) { return dim3((n + OT - 1) / OT, nb); }
    // fine_to_coarse: a warp per F2C_NPW coincident nodes, both blocks
    static dim3 f2c_grid(int n) { return grid_of(32 * ((n + F2C_NPW - 1) / F2C_NPW), 2); }

    // Launch with programmatic dependent launch (the kernels start with
    // pdl_wait(), so a launch overlaps only the tail of its predecessor).
    template <typename... KArgs, typename... Args>
    void launch(void (*kern)(KArgs...), dim3 grid, Args... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = dim3(OT);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, kern, args...));
        check_launch();
    }

    void set_step_dev() {
        if (step_dev_val != time_step) {
            k_set_step<<<1, 1, 0, stream>>>(step_dev, time_step);
            check_launch();
            step_dev_val = time_step;
        }
    }

    // The first collision of every level from the REF state.
    void collide_all() {
        set_step_dev();
        {
            LvlPair<StC> q = pair_cur(L0, L0);
            launch(k_oct_collide<StC, true>, grid_of(L0.n, 1), q, (const OctScal<A>*)tab, S,
                   (const long long*)step_dev, 0, seed32, 10, DynPtr<A>{});
        }
        {
            LvlPair<StF> q = pair_cur(L1[0], L1[1]);
            launch(k_oct_collide<StF, false>, grid_of(L1[0].n, 2), q, (const OctScal<A>*)tab, S,
                   (const long long*)step_dev, 1, seed32, 11, DynPtr<A>{});
        }
        if (levels == 3) {
            LvlPair<StF> q = pair_cur(L2[0], L2[1]);
            launch(k_oct_collide<StF, false>, grid_of(L2[0].n, 2), q, (const OctScal<A>*)tab, S,
                   (const long long*)step_dev, 2, seed32, 12, DynPtr<A>{});
        }
        pc_valid = true;
    }

    // The dynamic model's rescaling factors live on the device (xi_dev); the
    // molecular ones are launch arguments.  Once a dynamic step has run, the
    // device factors stay in use with the model off too: the reference never
    // rewrites xi in that mode (src/octree/solver.rs:690-698).
    const Xi<A>* xi_a_dev() const { return xi_dyn ? xi_dev : nullptr; }
    const Xi<A>* xi_b_dev() const { return xi_dyn ? xi_dev + 2 : nullptr; }

    void c2f_L1() {
        LvlPair<StC> c = pair_cur(L0, L0);
        LvlPair<StF> f = pair_cur(L1[0], L1[1]);
        launch(k_oct_c2f<StC, StF>, grid_of(4 * n_ghost, 2), c, f, (const GhostE<A>*)gh1, n_ghost, xa, xi_a_dev(),
               (const long long*)step_dev, seed32, 2);
    }
    void c2f_L2() {
        LvlPair<StF> c = pair_cur(L1[0], L1[1]);
        LvlPair<StF> f = pair_cur(L2[0], L2[1]);
        launch(k_oct_c2f<StF, StF>, grid_of(4 * n_ghost2, 2), c, f, (const GhostE<A>*)gh2, n_ghost2, xb, xi_b_dev(),
               (const long long*)step_dev, seed32, 4);
    }
    void f2c_L2(int off) {
        LvlPair<StF> f = pair_cur(L2[0], L2[1]);
        LvlPair<StF> c = pair_cur(L1[0], L1[1]);
        launch(k_oct_f2c<StF, StF>, f2c_grid(std::max(n_co2_0, n_co2_1)), f, c, (const CoinE*)co2, n_co2_0,
               n_co2_1, xb, xi_b_dev(), (const OctScal<A>*)tab, S, (const long long*)step_dev, off, 1, seed32, 7,
               int(!dyn));
    }
    void f2c_L1(int off) {
        LvlPair<StF> f = pair_cur(L1[0], L1[1]);
        LvlPair<StC> c = pair_cur(L0, L0);
        launch(k_oct_f2c<StF, StC>, f2c_grid(std::max(n_co0, n_co1)), f, c, (const CoinE*)co1, n_co0, n_co1,
               xa, xi_a_dev(), (const OctScal<A>*)tab, S, (const long long*)step_dev, off, 0, seed32, 13, int(!dyn));
    }
    void step_L0() {
        LvlPair<StC> q = pair(L0, L0);
        launch(k_oct_step<StC, true>, grid_of(L0.n, 1), q, (const OctScal<A>*)tab, S, (const long long*)step_dev, 1,
               0, seed32, 1, 1.0f / float(L0.nx), int(!dyn));
        L0.cur ^= 1;
    }
    // A fine level's (sub-)step: the f and g halves of a node on two threads
    // where that form exists (shifted formats, no fixed-Cs extension, not the
    // dynamic model's step, which collides separately), else one thread.
    bool split_fg() const { return level_kernel == CAV_OCT_LEVEL_FG && Fmt<StF>::SHIFT && !dyn && p.cs == 0.0; }
    void step_fine(Lvl<StF>* Lv, int lvl, int off, int phase) {
        LvlPair<StF> q = pair(Lv[0], Lv[1]);
        if constexpr (Fmt<StF>::SHIFT) {
            if (split_fg()) {
                launch(k_oct_step_fg<StF>, dim3((Lv[0].n + OCT_FG - 1) / OCT_FG, 2), q, (const OctScal<float>*)tab, S,
                       (const long long*)step_dev, off, lvl, seed32, phase, 1.0f / float(Lv[0].nx));
                Lv[0].cur ^= 1;
                Lv[1].cur ^= 1;
                return;
            }
        }
        launch(k_oct_step<StF, false>, grid_of(Lv[0].n, 2), q, (const OctScal<A>*)tab, S, (const long long*)step_dev,
               off, lvl, seed32, phase, 1.0f / float(Lv[0].nx), int(!dyn));
        Lv[0].cur ^= 1;
        Lv[1].cur ^= 1;
    }
    void step_L1(int off, int phase) { step_fine(L1, 1, off, phase); }
    void step_L2(int off, int phase) { step_fine(L2, 2, off, phase); }

    void set_level_kernel(int kind) override {
        if (kind != CAV_OCT_LEVEL_NODE && kind != CAV_OCT_LEVEL_FG)
            throw ArgError{CAV_ERR_ARG, "unknown octree level kernel"};
        if (kind == level_kernel) return;
        CK(cudaStreamSynchronize(stream));
        for (auto* gs : {graph, dgraph})
            for (int i = 0; i < 2; ++i)
                if (gs[i]) {
                    CK(cudaGraphExecDestroy(gs[i]));
                    gs[i] = nullptr;
                }
        level_kernel = kind;
    }
    int get_level_kernel() const override { return level_kernel; }

    // ---- dynamic mixed-scale SGS model ------------------------------------
    void set_dynamic_sgs(bool on, double smag_alpha, double nu_sm_min, double eta_test) override {
        if (!(smag_alpha >= 0.0 && smag_alpha <= 1.0) || !(eta_test >= 1.0) || !std::isfinite(nu_sm_min))
            throw ArgError{CAV_ERR_ARG, "dynamic SGS: smag_alpha in [0, 1], eta_test >= 1, finite nu_sm_min"};
        if (on && p.cs != 0.0)
            throw ArgError{CAV_ERR_ARG, "dynamic SGS and the fixed-Cs extension (cs != 0) are exclusive"};
        CK(cudaStreamSynchronize(stream));
        if (on && !sgs_w) {
            const int nmax = std::max(std::max(L0.n, L1[0].n), levels == 3 ? L2[0].n : 0);
            sgs_stride = size_t(S_NPLANES) * nmax;
            sgs_w = dalloc<double>(2 * sgs_stride);
            nut0 = dalloc<A>(2 * size_t(L0.n));
            for (int b = 0; b < 2; ++b) {
                nut1[b] = dalloc<A>(2 * size_t(L1[b].n));
                if (levels == 3) nut2[b] = dalloc<A>(2 * size_t(L2[b].n));
            }
            xi_dev = dalloc<Xi<A>>(4);
            dstat = dalloc<double>(16);
            mpart = dalloc<double>(size_t(4) * DYN_PARTS * 2);
            spart = dalloc<double>(size_t(DYN_PARTS) * 4);
            // before the first dynamic step: the molecular factors
            double h[16] = {0, 0, 0, 0, 0, xiA[0], xiA[1], xiA[2], xiB[0], xiB[1], xiB[2], xiB[0], xiB[1], xiB[2], 0, 0};
            CK(cudaMemcpyAsync(dstat, h, sizeof(h), cudaMemcpyHostToDevice, stream));
            const Xi<A> x4[4] = {xa, xa, xb, xb};
            CK(cudaMemcpyAsync(xi_dev, x4, sizeof(x4), cudaMemcpyHostToDevice, stream));
            CK(cudaStreamSynchronize(stream));
        }
        // new model constants: the dynamic graphs are captured anew
        for (auto& gx : dgraph)
            if (gx) {
                CK(cudaGraphExecDestroy(gx));
                gx = nullptr;
            }
        // leaving the model: the molecular path collides from REF again, and
        // its graphs are captured anew with the device factors
        if (dyn && !on) {
            pc_valid = false;
            for (auto& gx : graph)
                if (gx) {
                    CK(cudaGraphExecDestroy(gx));
                    gx = nullptr;
                }
        }
        dyn = on;
        dyn_alpha = smag_alpha;
        dyn_min = nu_sm_min;
        dyn_eta = eta_test;
    }

    // The model on nb (1 or 2) blocks of one level shape in one launch per
    // kernel (blockIdx.z = block).
    template <class St>
    void sgs_levels(const Lvl<St>* Ls, int nb, A* const* nuts, double tau_mol, double nu_l, double al_l) {
        const Lvl<St>& L = Ls[0];
        const Geom G{L.nx, L.ny, L.nx, (long long)L.n};
        SgsParams sp;
        const double eta = std::max(dyn_eta, 1.0);
        sp.width = std::max((int)std::llround(eta), 1);
        sp.dtest = eta * 1.0;
        sp.alpha_exp = dyn_alpha;
        sp.tau_s = tau_mol;
        sp.nu_mol = nu_l;
        sp.alpha_mol = al_l;
        sp.nu_sm_min = dyn_min;
        sp.rho_off = SH ? 1.0 : 0.0;
        SgsGrids<St> S{};
        for (int b = 0; b < nb; ++b) {
            const A* mac = Ls[b].mac;
            S.g[b] = SgsGrid<St>{Ls[b].ref[Ls[b].cur], mac,       mac + L.n, mac + 2 * L.n, mac + 3 * L.n,
                                 sgs_w + b * sgs_stride, nuts[b], nuts[b] + L.n};
        }
        const dim3 blk(32, 4), grd((L.nx + 31) / 32, (L.ny + 3) / 4, nb);
        k_sgs_b<St><<<grd, blk, 0, stream>>>(S, G, sp);
        check_launch();
        k_sgs_c<St><<<grd, blk, 0, stream>>>(S, G, sp);
        check_launch();
        k_sgs_d<St><<<grd, blk, 0, stream>>>(S, G, sp);
        check_launch();
    }

    template <class St>
    static MeanView<A> mview(const Lvl<St>& L, const A* nut) {
        return MeanView<A>{nut, nut + L.n, L.n};
    }

    void ramp_of(int64_t s, double& nu_eff, double& al_eff) const {
        nu_eff = nu;
        al_eff = alpha;
        if (nu_start_mult != 1.0) {
            const double m = 1.0 + (nu_start_mult - 1.0) * std::exp(-double(s) / 1000.0);
            nu_eff = nu * m;
            al_eff = alpha * m;
        }
    }

    // step_cavity with the dynamic model (src/octree/solver.rs:647-947): each
    // level's model on its REF state, then its collision with the per-node
    // nu_t / alpha_t (REF -> PC), then pull + BC + macroscopic + no-slip
    // without the fused next collision; xi A / xi B from the mean effective
    // taus.  Host-driven launches (the model's constants follow the ramp).
    void dyn_coarse_step() {
        xi_dyn = true;
        double nu_eff, al_eff;
        ramp_of(time_step, nu_eff, al_eff);
        // L0 model, its coefficient statistics, xi A (L1 nu_t of the previous step)
        sgs_levels(&L0, 1, &nut0, 0.5 + 3.0 * nu_eff, nu_eff, al_eff);
        k_oct_sgs_parts<<<DYN_PARTS, 256, 0, stream>>>(sgs_w, L0.n, spart);
        check_launch();
        {
            XiJob<A> J{};
            J.v[0] = mview(L0, nut0);
            J.v[1] = mview(L1[0], nut1[0]);
            J.v[2] = mview(L1[1], nut1[1]);
            J.mode = 0;
            J.nu_c = nu_eff;
            J.al_c = al_eff;
            J.nu_f = 2.0 * nu_eff;
            J.al_f = 2.0 * al_eff;
            J.odd_exact = p.odd_exact ? 1 : 0;
            k_oct_mean_parts<A><<<dim3(DYN_PARTS, 3), 256, 0, stream>>>(J, mpart);
            check_launch();
            k_oct_xi<A><<<1, 32, 0, stream>>>(J, (const double*)mpart, xi_dev, dstat + 5);
            check_launch();
        }
        const DynPtr<A> d0{{nut0, nut0}, {nut0 + L0.n, nut0 + L0.n}};
        const DynPtr<A> d1{{nut1[0], nut1[1]}, {nut1[0] + L1[0].n, nut1[1] + L1[1].n}};
        launch(k_oct_collide<StC, true>, grid_of(L0.n, 1), pair_cur(L0, L0), (const OctScal<A>*)tab, S,
               (const long long*)step_dev, 0, seed32, 1, d0);
        step_L0();
        c2f_L1();
        const double tau_mol_l1 = 0.5 + 3.0 * 2.0 * nu_eff, tau_mol_l2 = 0.5 + 3.0 * 4.0 * nu_eff;
        sgs_levels(L1, 2, nut1, tau_mol_l1, 2.0 * nu_eff, 2.0 * al_eff);
        launch(k_oct_collide<StF, false>, grid_of(L1[0].n, 2), pair_cur(L1[0], L1[1]), (const OctScal<A>*)tab, S,
               (const long long*)step_dev, 1, seed32, 3, d1);
        step_L1(0, 3);
        if (levels == 3) {
            XiJob<A> J{};
            J.v[0] = mview(L1[0], nut1[0]);
            J.v[1] = mview(L1[1], nut1[1]);
            J.v[2] = mview(L2[0], nut2[0]);
            J.v[3] = mview(L2[1], nut2[1]);
            J.mode = 1;
            J.nu_c = 2.0 * nu_eff;
            J.al_c = 2.0 * al_eff;
            J.nu_f = 4.0 * nu_eff;
            J.al_f = 4.0 * al_eff;
            J.odd_exact = p.odd_exact ? 1 : 0;
            k_oct_mean_parts<A><<<dim3(DYN_PARTS, 4), 256, 0, stream>>>(J, mpart);
            check_launch();
            k_oct_xi<A><<<1, 32, 0, stream>>>(J, (const double*)mpart, xi_dev + 2, dstat + 8);
            check_launch();
            c2f_L2();
            const DynPtr<A> d2{{nut2[0], nut2[1]}, {nut2[0] + L2[0].n, nut2[1] + L2[1].n}};
            for (int sp = 0; sp < 2; ++sp) {
                sgs_levels(L2, 2, nut2, tau_mol_l2, 4.0 * nu_eff, 4.0 * al_eff);
                launch(k_oct_collide<StF, false>, grid_of(L2[0].n, 2), pair_cur(L2[0], L2[1]),
                       (const OctScal<A>*)tab, S, (const long long*)step_dev, 2, seed32, 5 + sp, d2);
                step_L2(0, 5 + sp);
            }
            f2c_L2(0);
        }
        // the second L1 model takes the unramped nu / alpha (src/octree/solver.rs:882-890)
        sgs_levels(L1, 2, nut1, tau_mol_l1, 2.0 * nu, 2.0 * alpha);
        launch(k_oct_collide<StF, false>, grid_of(L1[0].n, 2), pair_cur(L1[0], L1[1]), (const OctScal<A>*)tab, S,
               (const long long*)step_dev, 1, seed32, 9, d1);
        step_L1(0, 9);
        f2c_L1(0);
        k_add_step<<<1, 1, 0, stream>>>(step_dev, 1);
        check_launch();
    }

    int64_t dyn_launches = 0;  // launches of one dynamic coarse step

    void dynamic_stats(double* out) override {
        if (!dstat) {
            for (int i = 0; i < 5; ++i) out[i] = 0.0;
            for (int i = 0; i < 3; ++i) out[5 + i] = xiA[i];
            for (int b = 0; b < 2; ++b)
                for (int i = 0; i < 3; ++i) out[8 + 3 * b + i] = levels == 3 ? xiB[i] : 0.0;
            return;
        }
        const bool l3 = levels == 3;
        k_oct_nutmax<A><<<1, 256, 0, stream>>>(mview(L0, nut0), mview(L1[0], nut1[0]), mview(L1[1], nut1[1]),
                                               l3 ? mview(L2[0], nut2[0]) : MeanView<A>{},
                                               l3 ? mview(L2[1], nut2[1]) : MeanView<A>{}, l3 ? 5 : 3, dstat + 4);
        check_launch();
        double h[14], sp[DYN_PARTS * 4];
        CK(cudaMemcpyAsync(h, dstat, sizeof(h), cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(sp, spart, sizeof(sp), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (int i = 0; i < 14; ++i) out[i] = h[i];
        if (xi_dyn) {
            double s0 = 0.0, m0 = 0.0, s1 = 0.0, m1 = 0.0;
            for (int c = 0; c < DYN_PARTS; ++c) {
                s0 += sp[c * 4 + 0];
                m0 = std::fmax(m0, sp[c * 4 + 1]);
                s1 += sp[c * 4 + 2];
                m1 = std::fmax(m1, sp[c * 4 + 3]);
            }
            out[0] = s0 / double(L0.n);
            out[1] = m0;
            out[2] = s1 / double(L0.n);
            out[3] = m1;
        }
        if (!l3)
            for (int i = 8; i < 14; ++i) out[i] = 0.0;
    }

    void get_nut(int lvl, double* nt, double* at) override {
        const A* src = nullptr;
        int n = 0;
        if (lvl == 0) {
            src = nut0;
            n = L0.n;
        } else if (lvl == 1 || lvl == 2) {
            src = nut1[lvl - 1];
            n = L1[lvl - 1].n;
        } else if (levels == 3 && (lvl == 3 || lvl == 4)) {
            src = nut2[lvl - 3];
            n = L2[lvl - 3].n;
        } else {
            throw ArgError{CAV_ERR_ARG, "no such level"};
        }
        if (!src) throw ArgError{CAV_ERR_STATE, "the dynamic model was never enabled"};
        std::vector<A> h(2 * size_t(n));
        CK(cudaMemcpyAsync(h.data(), src, sizeof(A) * h.size(), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (int k = 0; k < n; ++k) {
            if (nt) nt[k] = double(h[k]);
            if (at) at[k] = double(h[size_t(n) + k]);
        }
    }

    // One step_cavity (src/octree/solver.rs:647-947), all launches on `stream`,
    // with the step index taken from *step_dev (advanced at the end).
    void launch_coarse_step() {
        step_L0();
        c2f_L1();
        step_L1(0, 3);
        if (levels == 3) {
            c2f_L2();
            step_L2(0, 5);
            step_L2(1, 6);
            f2c_L2(0);
        }
        step_L1(1, 9);
        f2c_L1(1);
        k_add_step<<<1, 1, 0, stream>>>(step_dev, 1);
        check_launch();
    }

    cudaGraphExec_t get_graph() {
        cudaGraphExec_t& gx = graph[L0.cur];
        if (gx) return gx;
        const int c0 = L0.cur, c1 = L1[0].cur, c2 = L2[0].cur;
        const int64_t l0 = launches;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < OCT_GRAPH_STEPS; ++j) launch_coarse_step();
        cudaGraph_t gr;
        CK(cudaStreamEndCapture(stream, &gr));
        L0.cur = c0;
        L1[0].cur = L1[1].cur = c1;
        L2[0].cur = L2[1].cur = c2;
        launches = l0;
        CK(cudaGraphInstantiate(&gx, gr, 0));
        cudaGraphDestroy(gr);
        return gx;
    }

    int per_step_launches() const { return levels == 3 ? 10 : 6; }

    // OCT_GRAPH_STEPS dynamic coarse steps in one graph: valid once the
    // viscosity ramp has converged (the model's constants no longer change).
    cudaGraphExec_t get_dyn_graph() {
        cudaGraphExec_t& gx = dgraph[L0.cur];
        if (gx) return gx;
        const int c0 = L0.cur, c1 = L1[0].cur, c2 = L2[0].cur;
        const int64_t l0 = launches;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < OCT_GRAPH_STEPS; ++j) dyn_coarse_step();
        cudaGraph_t gr;
        CK(cudaStreamEndCapture(stream, &gr));
        dyn_launches = (launches - l0) / OCT_GRAPH_STEPS;
        L0.cur = c0;
        L1[0].cur = L1[1].cur = c1;
        L2[0].cur = L2[1].cur = c2;
        launches = l0;
        CK(cudaGraphInstantiate(&gx, gr, 0));
        cudaGraphDestroy(gr);
        return gx;
    }

    void step(int64_t n) override {
        if (n <= 0) return;
        if (dyn) {
            set_step_dev();
            while (n > 0) {
                if (n >= OCT_GRAPH_STEPS && time_step >= S) {
                    const int64_t l0 = launches;
                    cudaGraphExec_t gx = get_dyn_graph();
                    CK(cudaGraphLaunch(gx, stream));
                    launches = l0 + int64_t(OCT_GRAPH_STEPS) * dyn_launches;
                    xi_dyn = true;
                    time_step += OCT_GRAPH_STEPS;
                    n -= OCT_GRAPH_STEPS;
                } else {
                    dyn_coarse_step();
                    time_step += 1;
                    n -= 1;
                }
                step_dev_val = time_step;
            }
            CK(cudaGetLastError());
            return;
        }
        if (!pc_valid) collide_all();
        set_step_dev();
        while (n > 0) {
            if (n >= OCT_GRAPH_STEPS) {
                cudaGraphExec_t gx = get_graph();
                CK(cudaGraphLaunch(gx, stream));
                launches += int64_t(OCT_GRAPH_STEPS) * per_step_launches();
                time_step += OCT_GRAPH_STEPS;
                n -= OCT_GRAPH_STEPS;
            } else {
                launch_coarse_step();
                time_step += 1;
                n -= 1;
            }
            step_dev_val = time_step;
        }
        CK(cudaGetLastError());
    }

    void get_level(int lvl, double* r, double* u, double* v, double* t, double* f, double* g) override {
        CK(cudaStreamSynchronize(stream));
        if (lvl == 0) return download_state(L0, r, u, v, t, f, g);
        if (lvl == 1 || lvl == 2) return download_state(L1[lvl - 1], r, u, v, t, f, g);
        if (levels == 3 && (lvl == 3 || lvl == 4)) return download_state(L2[lvl - 3], r, u, v, t, f, g);
        throw ArgError{CAV_ERR_ARG, "no such level"};
    }

    void set_level(int lvl, const double* r, const double* u, const double* v, const double* t, const double* f,
                   const double* g) override {
        CK(cudaStreamSynchronize(stream));
        if (lvl == 0) return upload_state(L0, r, u, v, t, f, g);
        if (lvl == 1 || lvl == 2) return upload_state(L1[lvl - 1], r, u, v, t, f, g);
        if (levels == 3 && (lvl == 3 || lvl == 4)) return upload_state(L2[lvl - 3], r, u, v, t, f, g);
        throw ArgError{CAV_ERR_ARG, "no such level"};
    }

    // set_from_snapshot's per-level injection (src/octree/solver.rs:1113-1153):
    // fields as given, f = feq(rho, u), g = geq(T, u), then the level's
    // no-slip on the stored velocity (the populations keep the given u).
    void restart_level(int lvl, const double* r, const double* u, const double* v, const double* t) override {
        CK(cudaStreamSynchronize(stream));
        int nx, ny, hot = 0, cold = 0;
        bool coarse = lvl == 0;
        if (lvl == 0) {
            nx = nx0;
            ny = ny0;
        } else if (lvl == 1 || lvl == 2) {
            nx = nx1;
            ny = ny1;
            hot = lvl == 1;
            cold = lvl == 2;
        } else if (levels == 3 && (lvl == 3 || lvl == 4)) {
            nx = nx2;
            ny = ny2;
            hot = lvl == 3;
            cold = lvl == 4;
        } else {
            throw ArgError{CAV_ERR_ARG, "no such level"};
        }
        const size_t n = size_t(nx) * ny;
        std::vector<double> f(n * Q), g(n * Q), uu(u, u + n), vv(v, v + n);
        for (size_t k = 0; k < n; ++k)
            for (int i = 0; i < Q; ++i) {
                f[k * Q + i] = feq_full<double>(i, r[k], u[k], v[k]);
                g[k * Q + i] = geq_full<double>(i, t[k], u[k], v[k], 2);
            }
        for (int b = 0; b < ny; ++b)
            for (int a = 0; a < nx; ++a) {
                const bool wall = coarse ? (a == 0 || a == nx - 1 || b == 0 || b == ny - 1)
                                         : ((hot && a == 1) || (cold && a == nx - 2) || b == 1 || b == ny - 2);
                if (wall) uu[size_t(b) * nx + a] = vv[size_t(b) * nx + a] = 0.0;
            }
        set_level(lvl, r, uu.data(), vv.data(), t, f.data(), g.data());
    }

    void set_time_step(int64_t t) override {
        if (t < 0) throw ArgError{CAV_ERR_ARG, "negative time step"};
        time_step = t;
        pc_valid = false;
    }

    // Single couplings on the current state (for the interface tests):
    // 0 = coarse_to_fine L0 -> L1, 1 = fine_to_coarse L1 -> L0 (+ refresh),
    // 2 = coarse_to_fine L1 -> L2, 3 = fine_to_coarse L2 -> L1 (+ refresh).
    void debug_phase(int phase) override {
        set_step_dev();
        if (phase == 0) c2f_L1();
        else if (phase == 1) f2c_L1(0);
        else if (levels == 3 && phase == 2) c2f_L2();
        else if (levels == 3 && phase == 3) f2c_L2(0);
        else throw ArgError{CAV_ERR_ARG, "no such coupling phase"};
        pc_valid = false;
        CK(cudaStreamSynchronize(stream));
    }

    void diag(double* out) override {
        StatViews<A> V{};
        int nv = 0;
        V.v[nv++] = StatView<A>{L0.mac, L0.n};
        for (int b = 0; b < 2; ++b) V.v[nv++] = StatView<A>{L1[b].mac, L1[b].n};
        if (levels == 3)
            for (int b = 0; b < 2; ++b) V.v[nv++] = StatView<A>{L2[b].mac, L2[b].n};
        k_oct_stats<A, SH><<<dim3(OSTAT_CTAS, nv), 256, 0, stream>>>(V, part);
        check_launch();
        k_oct_iface<A, SH><<<2, 256, 0, stream>>>(L1[0].mac, L1[1].mac, L0.mac, L0.mac, gh1, n_ghost, co1, n_co0,
                                                 n_co1, iface);
        check_launch();
        int n_if = 2;
        if (levels == 3) {
            k_oct_iface<A, SH><<<2, 256, 0, stream>>>(L2[0].mac, L2[1].mac, L1[0].mac, L1[1].mac, gh2, n_ghost2, co2,
                                                     n_co2_0, n_co2_1, iface + 4);
            check_launch();
            n_if = 4;
        }
        const bool l3 = levels == 3;
        const A* mf = l3 ? L2[0].mac : L1[0].mac;
        const int nxf = l3 ? nx2 : nx1, nyf = l3 ? ny2 : ny1;
        const double nu_f = (l3 ? 4.0 : 2.0) * nu;
        const int R = std::max(std::max(ny0, ny1), nyf);
        k_oct_rows<A><<<(R + 255) / 256, 256, 0, stream>>>(L0.mac, nx0, ny0, L1[0].mac, nx1, ny1, mf, nxf, nyf, nu_f,
                                                          rowbuf, R);
        check_launch();
        k_oct_final<SH><<<1, 32, 0, stream>>>(rowbuf, R, nx0, ny0, ny1, nyf, nx0 * ny0, part, nv, OSTAT_CTAS, iface, n_if,
                                              dout);
        check_launch();
        CK(cudaMemcpyAsync(out, dout, sizeof(double) * 10, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    void sync() override { CK(cudaStreamSynchronize(stream)); }
};

}  // namespace oct
}  // namespace cav
