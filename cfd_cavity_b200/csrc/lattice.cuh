// lattice.cuh -- D2Q9 constants, storage formats and the per-node physics of
// the differentially heated cavity step (bbrangeo/cfd_cavity
// src/uniform/solver.rs), shared by every kernel of the library.
//
// Populations live on the device as 18 SoA planes (9 for f, 9 for g) of
// ny rows x pitch columns.  Four storage formats:
//   double         FP64 arithmetic, unshifted (the parity variant);
//   float          FP32 arithmetic, f stored as f_i - w_i;
//   Half16         FP32 arithmetic, f_i - w_i and g_i scaled by 2^15 into
//                  IEEE binary16 (Lehmann et al. 2022, "FP16S" storage);
//   Bf16           FP32 arithmetic, f_i - w_i and g_i in bfloat16;
//   Mix16          FP32 arithmetic, f_i - w_i in binary16 and g_i in 16-bit
//                  fixed point;
//   *SR            the same 16-bit encodings with stochastic rounding.
// g is shifted by w_i * T0 with T0 = 0, i.e. stored as is: theta is centred
// on zero in this problem (walls at +-0.5).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

namespace cav {

constexpr int Q = 9;
constexpr int NPLANES = 18;  // f planes 0..8, g planes 9..17

// Direction order: rest, E, N, NE, NW, W, S, SW, SE  (OPP[i] = i +- 4).
__host__ __device__ constexpr int CX(int i) {
    return i == 1 || i == 3 || i == 8 ? 1 : (i == 4 || i == 5 || i == 7 ? -1 : 0);
}
__host__ __device__ constexpr int CY(int i) {
    return i == 2 || i == 3 || i == 4 ? 1 : (i == 6 || i == 7 || i == 8 ? -1 : 0);
}
__host__ __device__ constexpr int OPP(int i) { return i == 0 ? 0 : (i <= 4 ? i + 4 : i - 4); }
__host__ __device__ constexpr double WD(int i) {
    return i == 0 ? 4.0 / 9.0 : (i == 1 || i == 2 || i == 5 || i == 6 ? 1.0 / 9.0 : 1.0 / 36.0);
}
constexpr double CS2 = 1.0 / 3.0;
constexpr double LAMBDA_TRT = 3.0 / 16.0;

// ---------------------------------------------------------------------------
// Storage formats.  load(v, q) / store(x, q, r) take the plane index q
// (0..8 f, 9..17 g) so that a format may encode f and g differently; every
// plane keeps one encoding, so raw copies between planes of one population
// set stay exact.  r carries 32 random bits for the stochastically rounded
// formats (ignored by the others); r = RN_BITS asks for round-to-nearest.
// Every load -> store round trip is exact, so moved (streamed) values are
// never re-rounded.
// ---------------------------------------------------------------------------
constexpr uint32_t RN_BITS = 0x80000000u;

template <class St>
struct Fmt;

template <>
struct Fmt<double> {
    using A = double;
    static constexpr bool SHIFT = false, SR = false;
    __host__ __device__ static A load(double v, int) { return v; }
    __host__ __device__ static double store(A v, int, uint32_t) { return v; }
};
template <>
struct Fmt<float> {
    using A = float;
    static constexpr bool SHIFT = true, SR = false;
    __host__ __device__ static A load(float v, int) { return v; }
    __host__ __device__ static float store(A v, int, uint32_t) { return v; }
};

// binary16 of x * 2^15 (the 2^15 keeps |f - w| >= 2e-9 out of the subnormals).
constexpr float H_SCALE = 32768.0f, H_INV = 1.0f / 32768.0f;

__host__ __device__ __forceinline__ float h16_load(unsigned short bits) {
    __half_raw r;
    r.x = bits;
    return __half2float(__half(r)) * H_INV;
}
// Round to nearest (ties to even), or stochastically: add 13 random bits
// below binary16's last mantissa bit to the binary32 magnitude, then
// truncate (Croci et al., "Stochastic rounding: implementation, error
// analysis and applications", R. Soc. open sci. 2022).  Unbiased:
// E[round(x)] = x.
__host__ __device__ __forceinline__ unsigned short h16_store(float x, bool sr, uint32_t r) {
    float s = x * H_SCALE;
    __half h;
    if (sr) {
        // (a non-finite input stays non-finite: inf + dither becomes NaN)
        uint32_t u;
        memcpy(&u, &s, 4);
        u += (r >> 19);
        memcpy(&s, &u, 4);
        h = __float2half_rz(s);
    } else {
        h = __float2half_rn(s);
    }
    return __half_raw(h).x;
}

__host__ __device__ __forceinline__ float bf16_load(unsigned short bits) {
    uint32_t u = uint32_t(bits) << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}
__host__ __device__ __forceinline__ unsigned short bf16_store(float x, bool sr, uint32_t r) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (unsigned short)(u >> 16);  // inf / nan
    if (sr) return (unsigned short)((u + (r >> 16)) >> 16);
    return (unsigned short)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);        // nearest, ties to even
}

// 16-bit fixed point of g_i with a power-of-two scale per direction class:
// 2^16 on the rest population (|g_0| <= 4/9 |T| < 0.5), 2^17 on the axes
// (|g| <= 1/9 |T| (1 + 3|u| + ...) < 0.25), 2^19 on the diagonals
// (< 0.0625), for |T| <= 0.51 and |u| <= 0.1 (the driver's max_u guard).
// Saturates instead of wrapping.  Absolute error: 1.5e-5, 7.6e-6, 1.9e-6.
__host__ __device__ constexpr int fx_shift(int q) {
    return q == 9 ? 16 : (q == 10 || q == 11 || q == 14 || q == 15 ? 17 : 19);
}
__host__ __device__ __forceinline__ float fx_load(unsigned short bits, int q) {
    return float(short(bits)) * ldexpf(1.0f, -fx_shift(q));
}
__host__ __device__ __forceinline__ unsigned short fx_store(float x, int q, bool sr, uint32_t r) {
    float s = x * ldexpf(1.0f, fx_shift(q));
    s = fminf(fmaxf(s, -32767.0f), 32767.0f);
    float fl = floorf(s);
    float frac = s - fl;
    int iv;
    if (sr) {
        iv = int(fl) + ((float(r >> 8) * (1.0f / 16777216.0f)) < frac ? 1 : 0);
    } else {
        iv = int(fl) + (frac > 0.5f || (frac == 0.5f && (int(fl) & 1)) ? 1 : 0);
    }
    if (iv > 32767) iv = 32767;
    return (unsigned short)(short)iv;
}

// Tag types of the 16-bit formats (one distinct type per encoding).
template <int KIND, bool SRND>
struct P16 {
    unsigned short bits;
};
constexpr int K_HALF = 0, K_BF16 = 1, K_MIX = 2;  // MIX: binary16 f - w, fixed-point g

template <int KIND, bool SRND>
struct Fmt<P16<KIND, SRND>> {
    using A = float;
    using St = P16<KIND, SRND>;
    static constexpr bool SHIFT = true, SR = SRND;
    __host__ __device__ static A load(St v, int q) {
        if (KIND == K_BF16) return bf16_load(v.bits);
        if (KIND == K_MIX && q >= 9) return fx_load(v.bits, q);
        return h16_load(v.bits);
    }
    __host__ __device__ static St store(A x, int q, uint32_t r) {
        const bool sr = SRND && r != RN_BITS;
        St o;
        if (KIND == K_BF16) o.bits = bf16_store(x, sr, r);
        else if (KIND == K_MIX && q >= 9) o.bits = fx_store(x, q, sr, r);
        else o.bits = h16_store(x, sr, r);
        return o;
    }
    // Always stochastic (the collision's writes).
    __host__ __device__ static St store_sr(A x, int q, uint32_t r) {
        St o;
        if (KIND == K_BF16) o.bits = bf16_store(x, true, r);
        else if (KIND == K_MIX && q >= 9) o.bits = fx_store(x, q, true, r);
        else o.bits = h16_store(x, true, r);
        return o;
    }
};
using Half16 = P16<K_HALF, false>;
using Half16SR = P16<K_HALF, true>;
using Bf16 = P16<K_BF16, false>;
using Bf16SR = P16<K_BF16, true>;
using Mix16 = P16<K_MIX, false>;
using Mix16SR = P16<K_MIX, true>;

// Per-node stream of random words for the stochastic rounding: a MurmurHash3
// finaliser of (seed, step, node) seeds a 32-bit LCG (Numerical Recipes
// constants); the rounding uses the high bits.  Depends only on
// (seed, step, node), so every run, graph replay or not, is reproducible.
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
struct NodeRng {
    uint32_t s;
    __host__ __device__ NodeRng(uint32_t seed, long long step, long long node)
        : s(mix32(uint32_t(node) * 0x9E3779B1u + mix32(uint32_t(step) ^ seed))) {}
    __host__ __device__ uint32_t next() {
        s = s * 1664525u + 1013904223u;
        return s;
    }
};

// Grid geometry of one cavity.
struct Geom {
    int nx, ny, pitch;
    long long plane;  // ny * pitch
};

// Per-launch scalars of collide (CollideCtx, src/uniform/solver.rs:1034-1043)
// plus the boundary data.  Computed on the host in FP64 for each step, then
// converted to the arithmetic type.
template <class A>
struct StepScalars {
    A tau_s;   // tau used for |S|: 0.5 + 3*max(nu_eff, 0.002/3)  (solver.rs:442)
    A beta;    // ramped beta_eff                                   (solver.rs:433-437)
    A nu;      // ramped nu_eff                                     (solver.rs:390-400)
    A alpha;   // ramped alpha_eff                                  (solver.rs:401-408)
    A cs;      // Smagorinsky constant
    A pr_t;    // turbulent Prandtl number
    A inv_tau_s;  // 1 / tau_s
    A inv_pr_t;   // 1 / pr_t
    A t_cold;  // cold-wall theta
    int geq_order;
    const A* t_hot;  // [ny] hot-wall theta
    uint32_t sr_seed;  // seed of the stochastic rounding
    long long step;    // step index of this collision (used by the rounding)
    const long long* step_dev;  // if set, the step is *step_dev + step (graph replays)
};

// ---------------------------------------------------------------------------
// Equilibria.  In the unshifted (FP64) form the expressions are those of the
// reference (feq form restated at src/uniform/tests.rs:314-316); the shifted
// form returns feq_i - w_i from (drho = rho - 1, rho).
// ---------------------------------------------------------------------------
template <class A>
__host__ __device__ __forceinline__ A feq_full(int i, A rho, A ux, A uy) {
    const A cs2 = A(CS2);
    A eu = A(CX(i)) * ux + A(CY(i)) * uy;
    A u2 = ux * ux + uy * uy;
    return A(WD(i)) * rho * (A(1.0) + eu / cs2 + eu * eu / (A(2.0) * cs2 * cs2) - u2 / (A(2.0) * cs2));
}

template <class A>
__host__ __device__ __forceinline__ A geq_full(int i, A t, A ux, A uy, int order) {
    const A cs2 = A(CS2);
    A eu = A(CX(i)) * ux + A(CY(i)) * uy;
    if (order == 1) return A(WD(i)) * t * (A(1.0) + eu / cs2);
    A u2 = ux * ux + uy * uy;
    return A(WD(i)) * t * (A(1.0) + eu / cs2 + eu * eu / (A(2.0) * cs2 * cs2) - u2 / (A(2.0) * cs2));
}

// FP32 shifted equilibrium: feq_i - w_i = w_i*(drho + rho*P_i),
// P_i = 3 e.u + 4.5 (e.u)^2 - 1.5 u^2.
__device__ __forceinline__ float feq_shift_f32(int i, float drho, float rho, float ux, float uy) {
    float eu = float(CX(i)) * ux + float(CY(i)) * uy;
    float u2 = ux * ux + uy * uy;
    float P = 3.0f * eu + 4.5f * eu * eu - 1.5f * u2;
    return float(WD(i)) * (drho + rho * P);
}
__device__ __forceinline__ float geq_f32(int i, float t, float ux, float uy, int order) {
    float eu = float(CX(i)) * ux + float(CY(i)) * uy;
    if (order == 1) return float(WD(i)) * t * (1.0f + 3.0f * eu);
    float u2 = ux * ux + uy * uy;
    return float(WD(i)) * t * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * u2);
}

// ---------------------------------------------------------------------------
// Macroscopic update of one node (update_macroscopic, src/uniform/solver.rs:
// 298-367, then enforce_wall_velocity :992-1009 when `wall`).  Sums run in
// the reference's direction order so that FP64 results are bit-identical.
// ---------------------------------------------------------------------------
template <class A, bool SHIFT>
struct Macro {
    A rho, drho, ux, uy, t, inv_rho;
};

template <class A>
__device__ __forceinline__ A sum_g(const A (&g)[Q]) {
    A tn = g[0];
#pragma unroll
    for (int j = 1; j < Q; ++j) tn = tn + g[j];
    return tn;
}

// rho and u of the node (t left 0): the f part of macro_node.
template <class A, bool SHIFT>
__device__ __forceinline__ Macro<A, SHIFT> macro_f(const A (&f)[Q], A fy_prev, bool wall) {
    Macro<A, SHIFT> m;
    A s = f[0];
#pragma unroll
    for (int j = 1; j < Q; ++j) s = s + f[j];
    A un = ((((f[1] + f[3]) - f[4]) - f[5]) - f[7]) + f[8];
    A vn = ((((f[2] + f[3]) + f[4]) - f[6]) - f[7]) - f[8];
    A r;
    m.inv_rho = A(0.0);
    if (SHIFT) {
        m.drho = s;
        r = A(1.0) + s;
    } else {
        r = s;
        m.drho = s - A(1.0);
    }
    if constexpr (SHIFT) {
        const A inv = __fdividef(1.0f, r);
        m.inv_rho = inv;
        un = un * inv;
        vn = (vn + A(0.5) * fy_prev) * inv;
    } else if (r > A(2.220446049250313e-16)) {
        un = un / r;
        vn = vn / r;
        vn = vn + A(0.5) * fy_prev / r;
    }
    m.rho = r;
    m.ux = wall ? A(0.0) : un;
    m.uy = wall ? A(0.0) : vn;
    m.t = A(0.0);
    return m;
}

template <class A, bool SHIFT>
__device__ __forceinline__ Macro<A, SHIFT> macro_node(const A (&f)[Q], const A (&g)[Q], A fy_prev, bool wall) {
    Macro<A, SHIFT> m = macro_f<A, SHIFT>(f, fy_prev, wall);
    m.t = sum_g<A>(g);
    return m;
}

// ---------------------------------------------------------------------------
// Collision of one node: TRT + Smagorinsky + Guo forcing for f, BGK for g
// (collide_node, src/uniform/solver.rs:1054-1185, fixed-Cs branch).
// f and g are updated in place; returns fy and nu_t.
// FP64 follows the reference expression by expression; the FP32 variant
// works on f_i - w_i and replaces divisions by constants with products.
// ---------------------------------------------------------------------------
// The collision in three parts: collide_f_pre (everything of f that does
// not need T: non-equilibrium parts, pi_neq, nu_t, relaxation rates),
// collide_f_post (the f update, with the Guo force rho beta T) and collide_g
// (BGK of g, needs T, u and nu_t).  collide_node runs the three.
template <class A>
struct CollF {
    A d[Q];                // FP64: f - feq
    A d0, dS[5], dD[5];    // FP32: rest part, symmetric / antisymmetric pair parts
    A nut, w1, w2, k1, k2; // FP64 a_f, b_f, k-, k+;  FP32 om+, om-, k+, k-
};

// nut_ovr: nu_t given per node (the dynamic subgrid model, solver.rs:1118-1121)
// instead of Cs^2 |S|.
template <class A, bool SHIFT>
__device__ __forceinline__ CollF<A> collide_f_pre(const A (&f)[Q], const Macro<A, SHIFT>& m, const StepScalars<A>& c,
                                                  const A* nut_ovr = nullptr) {
    CollF<A> o;
    const A r = m.rho, u = m.ux, v = m.uy;
    if constexpr (!SHIFT) {
        // ---- FP64: expression order of the reference ----------------------
        const double cs2 = CS2;
#pragma unroll
        for (int i = 0; i < Q; ++i) o.d[i] = f[i] - feq_full<double>(i, r, u, v);
        const double* d_f = o.d;
        // pi_neq, solver.rs:1096-1106 (terms with c = 0 add +-0).
        double pxx = ((((d_f[1] + d_f[3]) + d_f[4]) + d_f[5]) + d_f[7]) + d_f[8];
        double pxy = ((d_f[3] - d_f[4]) + d_f[7]) - d_f[8];
        double pyy = ((((d_f[2] + d_f[3]) + d_f[4]) + d_f[6]) + d_f[7]) + d_f[8];
        double pi2 = pxx * pxx + 2.0 * pxy * pxy + pyy * pyy;
        double rho_m = r > 1e-12 ? r : 1e-12;
        double s_mag = sqrt(pi2) / (2.0 * cs2 * c.tau_s * rho_m);
        double nut = nut_ovr ? double(*nut_ovr) : c.cs * c.cs * s_mag;
        o.nut = nut;
        double tau_plus = 0.5 + 3.0 * (c.nu + nut);
        double tau_minus = 0.5 + LAMBDA_TRT / (tau_plus - 0.5);
        o.w1 = 0.5 * (1.0 / tau_plus + 1.0 / tau_minus);
        o.w2 = 0.5 * (1.0 / tau_plus - 1.0 / tau_minus);
        o.k1 = 1.0 - 0.5 / tau_minus;
        o.k2 = 1.0 - 0.5 / tau_plus;
    } else {
        // ---- FP32 on h_i = f_i - w_i, pairwise (i, opp(i)) form --------------
        // For each pair p = (i, i+4), i = 1..4, split populations and
        // equilibria into symmetric / antisymmetric parts: the TRT update
        //   f_i += -a d_i - b d_opp + (1 - 1/2tau-) S-_i + (1 - 1/2tau+) S+_i
        // with a = (w+ + w-)/2, b = (w+ - w-)/2 is exactly
        //   f_p += E + O, f_opp += E - O,
        //   E = -w+ (d_p + d_opp)/2 + k+ S+_p,  O = -w- (d_p - d_opp)/2 + k- S-_p,
        // and pi_neq only needs the symmetric parts.  Same arithmetic as the
        // reference up to rounding (FP32), a third of the operations.
        const float u2 = u * u + v * v;
        const float inv_r = m.inv_rho;
        const float feq0 = float(WD(0)) * (m.drho - 1.5f * r * u2);
        o.d0 = f[0] - feq0;
#pragma unroll
        for (int p = 1; p <= 4; ++p) {
            const float cx = CX(p), cy = CY(p);
            const float eu = cx * u + cy * v;
            const float feS = float(WD(p)) * (m.drho + r * (4.5f * eu * eu - 1.5f * u2));
            const float feA = float(WD(p)) * (r * 3.0f * eu);
            o.dS[p] = (f[p] + f[p + 4]) - 2.0f * feS;
            o.dD[p] = (f[p] - f[p + 4]) - 2.0f * feA;
        }
        // pi_neq (solver.rs:1096-1106) from the symmetric parts.
        const float pxx = o.dS[1] + o.dS[3] + o.dS[4];
        const float pxy = o.dS[3] - o.dS[4];
        const float pyy = o.dS[2] + o.dS[3] + o.dS[4];
        const float pi2 = pxx * pxx + 2.0f * pxy * pxy + pyy * pyy;
        // |S| = sqrt(pi:pi) / (2 cs^2 tau rho) = sqrt(pi:pi) * (1.5 / tau) / rho
        const float s_mag = __fsqrt_rn(pi2) * (1.5f * c.inv_tau_s) * inv_r;
        const float nut = nut_ovr ? float(*nut_ovr) : c.cs * c.cs * s_mag;
        o.nut = nut;
        const float e = 3.0f * (c.nu + nut);             // tau+ - 1/2
        o.w1 = __fdividef(1.0f, 0.5f + e);                // 1/tau+
        o.w2 = __fdividef(e, 0.5f * e + float(LAMBDA_TRT));  // 1/tau-, tau- = 1/2 + Lambda/e
        o.k1 = 1.0f - 0.5f * o.w1;
        o.k2 = 1.0f - 0.5f * o.w2;
    }
    return o;
}

// The f update with the Guo force fy = rho beta (T - 0) (solver.rs:1084,
// 1159-1179); returns fy.
template <class A, bool SHIFT>
__device__ __forceinline__ A collide_f_post(A (&f)[Q], const CollF<A>& o, const Macro<A, SHIFT>& m,
                                            const StepScalars<A>& c, A temp) {
    const A r = m.rho, u = m.ux, v = m.uy;
    if constexpr (!SHIFT) {
        const double cs2 = CS2;
        const double fyv = r * c.beta * 1.0 * (temp - 0.0);
        const double* d_f = o.d;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const double cx = CX(i), cy = CY(i);
            double ei_u = cx * u + cy * v;
            double s_i = WD(i) * ((cy - v) / cs2 + ei_u * cy / (cs2 * cs2)) * fyv;
            double s_minus = WD(i) * (cy / cs2) * fyv;
            double s_plus = s_i - s_minus;
            f[i] = f[i] + (-o.w1 * d_f[i] - o.w2 * d_f[OPP(i)] + o.k1 * s_minus + o.k2 * s_plus);
        }
        return fyv;
    } else {
        const float fyv = r * c.beta * temp;
        const float om_p = o.w1, om_m = o.w2, k_p = o.k1, k_m = o.k2;
        // Guo source: S+_p = w_p (-3 u_y + 9 (e.u) c_y) fy, S-_p = w_p 3 c_y fy.
        f[0] = f[0] - om_p * o.d0 + k_p * float(WD(0)) * (-3.0f * v) * fyv;
#pragma unroll
        for (int p = 1; p <= 4; ++p) {
            const float cx = CX(p), cy = CY(p);
            const float eu = cx * u + cy * v;
            const float E = -0.5f * om_p * o.dS[p] + k_p * float(WD(p)) * (-3.0f * v + 9.0f * eu * cy) * fyv;
            const float O = -0.5f * om_m * o.dD[p] + k_m * float(WD(p)) * (3.0f * cy) * fyv;
            f[p] = f[p] + (E + O);
            f[p + 4] = f[p + 4] + (E - O);
        }
        return fyv;
    }
}

// BGK collision of g (solver.rs:1136-1144, 1181-1184); at_ovr: alpha_t given
// per node (dynamic subgrid model) instead of nu_t / Pr_t.
template <class A, bool SHIFT>
__device__ __forceinline__ void collide_g(A (&g)[Q], A temp, A u, A v, A nut, const StepScalars<A>& c,
                                          const A* at_ovr = nullptr) {
    if constexpr (!SHIFT) {
        double d_g[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) d_g[i] = g[i] - geq_full<double>(i, temp, u, v, c.geq_order);
        double alpha_t = at_ovr ? double(*at_ovr) : nut / c.pr_t;
        double tau_t_plus = 0.5 + 3.0 * (c.alpha + alpha_t);
        double tau_t_minus = tau_t_plus;
        double a_g = 0.5 * (1.0 / tau_t_plus + 1.0 / tau_t_minus);
        double b_g = 0.5 * (1.0 / tau_t_plus - 1.0 / tau_t_minus);
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = g[i] + (-a_g * d_g[i] - b_g * d_g[OPP(i)]);
    } else {
        const float u2 = u * u + v * v;
        const float alpha_t = at_ovr ? float(*at_ovr) : nut * c.inv_pr_t;
        const float om_g = __fdividef(1.0f, 0.5f + 3.0f * (c.alpha + alpha_t));  // BGK g
        // g: BGK towards geq (quadratic or linear in u).
        const float one_m = 1.0f - om_g;
        const float q2 = c.geq_order == 1 ? 0.0f : 1.0f;
        g[0] = one_m * g[0] + om_g * float(WD(0)) * temp * (1.0f - q2 * 1.5f * u2);
#pragma unroll
        for (int p = 1; p <= 4; ++p) {
            const float cx = CX(p), cy = CY(p);
            const float eu = cx * u + cy * v;
            const float gS = om_g * float(WD(p)) * temp * (1.0f + q2 * (4.5f * eu * eu - 1.5f * u2));
            const float gA = om_g * float(WD(p)) * temp * (3.0f * eu);
            g[p] = one_m * g[p] + (gS + gA);
            g[p + 4] = one_m * g[p + 4] + (gS - gA);
        }
    }
}

// ---------------------------------------------------------------------------
// Collision of one node: TRT + Smagorinsky + Guo forcing for f, BGK for g
// (collide_node, src/uniform/solver.rs:1054-1185, fixed-Cs branch).
// f and g are updated in place; returns fy and nu_t.
// FP64 follows the reference expression by expression; the FP32 variant
// works on f_i - w_i and replaces divisions by constants with products.
// ---------------------------------------------------------------------------
template <class A, bool SHIFT>
__device__ __forceinline__ void collide_node(A (&f)[Q], A (&g)[Q], const Macro<A, SHIFT>& m,
                                             const StepScalars<A>& c, A& fy_out, A& nut_out,
                                             const A* nut_ovr = nullptr, const A* at_ovr = nullptr) {
    const CollF<A> o = collide_f_pre<A, SHIFT>(f, m, c, nut_ovr);
    nut_out = o.nut;
    fy_out = collide_f_post<A, SHIFT>(f, o, m, c, m.t);
    collide_g<A, SHIFT>(g, m.t, m.ux, m.uy, o.nut, c, at_ovr);
}

// Wall-node equilibrium of g (apply_thermal_boundary_conditions,
// src/uniform/solver.rs:957-970): geq(T_wall, 0, 0) = w_i T_wall.
template <class A>
__device__ __forceinline__ A geq_rest(int i, A t, int order) {
    return geq_full<A>(i, t, A(0.0), A(0.0), order);
}

}  // namespace cav
