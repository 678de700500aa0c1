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

#include <type_traits>

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

// 2^e as a float constant (|e| < 64).
__host__ __device__ constexpr float p2(int e) {
    return e >= 0 ? float(1ull << e) : 1.0f / float(1ull << -e);
}

// Lane units.  The fused step works on the f planes scaled by 2^EF and the g
// planes by 2^EG (the formats' own power-of-two scales, so that lload is a
// bare decode and lstore a bare encode); power-of-two scaling commutes with
// rounding, and the physics folds the factors into its constants.

template <class St>
struct Fmt;

template <>
struct Fmt<double> {
    using A = double;
    static constexpr bool SHIFT = false, SR = false, HW_SR_F = false, HW_SR_G = false;
    static constexpr bool KIND_BF16 = false, FIXED_G = false;
    static constexpr int EF = 0, EG = 0;
    __host__ __device__ static A load(double v, int) { return v; }
    __host__ __device__ static double store(A v, int, uint32_t) { return v; }
    __host__ __device__ static A lload(double v, int) { return v; }
    __host__ __device__ static double lstore(A v, int, uint32_t) { return v; }
};
template <>
struct Fmt<float> {
    using A = float;
    static constexpr bool SHIFT = true, SR = false, HW_SR_F = false, HW_SR_G = false;
    static constexpr bool KIND_BF16 = false, FIXED_G = false;
    static constexpr int EF = 0, EG = 0;
    __host__ __device__ static A load(float v, int) { return v; }
    __host__ __device__ static float store(A v, int, uint32_t) { return v; }
    __host__ __device__ static A lload(float v, int) { return v; }
    __host__ __device__ static float lstore(A v, int, uint32_t) { return v; }
};

// binary16 of x * 2^15 (the 2^15 keeps |f - w| >= 2e-9 out of the subnormals).
constexpr float H_SCALE = 32768.0f, H_INV = 1.0f / 32768.0f;

__host__ __device__ __forceinline__ float h16_raw(unsigned short bits) {
    __half_raw r;
    r.x = bits;
    return __half2float(__half(r));
}
__host__ __device__ __forceinline__ float h16_load(unsigned short bits) { return h16_raw(bits) * H_INV; }
// Round to nearest (ties to even), or stochastically: add 13 random bits
// below binary16's last mantissa bit to the binary32 magnitude, then
// truncate (Croci et al., "Stochastic rounding: implementation, error
// analysis and applications", R. Soc. open sci. 2022).  Unbiased:
// E[round(x)] = x.
// h16_enc takes x already scaled by 2^15.
__host__ __device__ __forceinline__ unsigned short h16_enc(float s, bool sr, uint32_t r) {
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
__host__ __device__ __forceinline__ unsigned short h16_store(float x, bool sr, uint32_t r) {
    return h16_enc(x * H_SCALE, sr, r);
}
#ifdef __CUDACC__
// Two h16_enc stochastic roundings in one instruction (cvt.rs.f16x2.f32):
// the hardware adds the low 13 bits of rbits[31:16] (for a) and of
// rbits[15:0] (for b) below binary16's last mantissa bit and truncates (the
// layout checked on a B200 with an in-bounds probe).  With rbits = r >> 3
// those are r's bits 31..19 and 15..3, the bits h16_enc takes from the
// draws r & 0xffff0000 and r << 16.  Checked against h16_enc on 2^21 random
// values: the same bits for normal binary16 results (33 differences, all at
// the overflow edge above 65504); results in the subnormal range differ,
// where the hardware dithers at the subnormal's last bit (unbiased) and the
// 13-bit software dither does not.  Returns (a << 16) | b.
__device__ __forceinline__ uint32_t h16x2_enc_sr(float a, float b, uint32_t r) {
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(r >> 3));
    return d;
}
#endif

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
#ifdef __CUDACC__
// Two bf16_store stochastic roundings in one instruction
// (cvt.rs.bf16x2.f32): r[31:16] dithers a, r[15:0] dithers b, the bits
// bf16_store takes from the draws r & 0xffff0000 and r << 16.  Returns
// (a << 16) | b.
__device__ __forceinline__ uint32_t bf16x2_enc_sr(float a, float b, uint32_t r) {
    uint32_t d;
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(r));
    return d;
}
#endif

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
template <class St>
struct is_p16 : std::false_type {};
template <int KIND, bool SRND>
struct is_p16<P16<KIND, SRND>> : std::true_type {};

template <int KIND, bool SRND>
struct Fmt<P16<KIND, SRND>> {
    using A = float;
    using St = P16<KIND, SRND>;
    static constexpr bool SHIFT = true, SR = SRND;
    // stochastic rounding of the binary16 (bfloat16) planes by the hardware
    // cvt.rs: the f planes of every 16-bit format, the g planes unless they
    // are fixed point.  enc2_sr rounds two planes of one node (the octree's
    // stores); the uniform solver rounds one plane of two nodes (kernels.cuh)
    static constexpr bool HW_SR_F = SRND, HW_SR_G = SRND && KIND != K_MIX;
    static constexpr bool KIND_BF16 = KIND == K_BF16, FIXED_G = KIND == K_MIX;
#ifdef __CUDACC__
    __device__ static uint32_t enc2_sr(float a, float b, uint32_t r) {
        if constexpr (KIND == K_BF16)
            return bf16x2_enc_sr(a, b, r);
        else
            return h16x2_enc_sr(a, b, r);
    }
#endif
    static constexpr int EF = KIND == K_BF16 ? 0 : 15, EG = KIND == K_HALF ? 15 : 0;
    // lane units: binary16 planes undecoded by the 2^15 (see EF / EG)
    __host__ __device__ static A lload(St v, int q) {
        if (KIND == K_BF16) return bf16_load(v.bits);
        if (KIND == K_MIX && q >= 9) return fx_load(v.bits, q);
        return h16_raw(v.bits);
    }
    __host__ __device__ static St lstore(A x, int q, uint32_t r) {
        const bool sr = SRND && r != RN_BITS;
        St o;
        if (KIND == K_BF16) o.bits = bf16_store(x, sr, r);
        else if (KIND == K_MIX && q >= 9) o.bits = fx_store(x, q, sr, r);
        else o.bits = h16_enc(x, sr, r);
        return o;
    }
    __host__ __device__ static St lstore_sr(A x, int q, uint32_t r) {
        St o;
        if (KIND == K_BF16) o.bits = bf16_store(x, true, r);
        else if (KIND == K_MIX && q >= 9) o.bits = fx_store(x, q, true, r);
        else o.bits = h16_enc(x, true, r);
        return o;
    }
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
    // Advances by K draws in one multiply-add: s <- a^K s + c (a^(K-1) + ... + 1).
    template <int K>
    __host__ __device__ void skip() {
        uint32_t a = 1u, c = 0u;
        for (int j = 0; j < K; ++j) {
            c = c * 1664525u + 1013904223u;
            a = a * 1664525u;
        }
        s = s * a + c;
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

// ---------------------------------------------------------------------------
// Lane arithmetic of the FP32 physics.  The FP32 macroscopic update and
// collision are written once over a lane type L: float (one node) or float2
// (two nodes in one thread, on Blackwell's packed FP32x2 add / mul / fma:
// one instruction for both nodes).  Every operation is an explicitly rounded
// intrinsic, so the compiler contracts nothing and a node gets the same bits
// from either lane type, in whichever kernel it runs.
// ---------------------------------------------------------------------------
struct Mask2 {
    bool x, y;
};
template <class L>
struct LaneMask;
template <>
struct LaneMask<float> {
    using T = bool;
};
template <>
struct LaneMask<float2> {
    using T = Mask2;
};

__device__ __forceinline__ float ladd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float lsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float lmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float lfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float2 ladd(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as fma(b, -1, a): b * -1 is exact, so this is the one rounding of
// a - b that __fsub_rn gives.
__device__ __forceinline__ float2 lsub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 lmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 lfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <class L>
__device__ __forceinline__ L lbc(float s);
template <>
__device__ __forceinline__ float lbc<float>(float s) {
    return s;
}
template <>
__device__ __forceinline__ float2 lbc<float2>(float s) {
    return make_float2(s, s);
}

// 1/x and sqrt(x) from the special-function unit (rcp.approx / sqrt.approx,
// about one ulp); the arguments here are normal numbers or zero.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float lrcp(float x) { return rcp_approx(x); }
__device__ __forceinline__ float2 lrcp(float2 x) { return make_float2(rcp_approx(x.x), rcp_approx(x.y)); }
__device__ __forceinline__ float lsqrt(float x) { return sqrt_approx(x); }
__device__ __forceinline__ float2 lsqrt(float2 x) { return make_float2(sqrt_approx(x.x), sqrt_approx(x.y)); }
__device__ __forceinline__ float lsel(bool m, float a, float b) { return m ? a : b; }
__device__ __forceinline__ float2 lsel(Mask2 m, float2 a, float2 b) {
    return make_float2(m.x ? a.x : b.x, m.y ? a.y : b.y);
}

// c_i . u for the directions p = 1..4 of the (p, p + 4) pairs:
// E (1, 0), N (0, 1), NE (1, 1), NW (-1, 1).
template <class L>
__device__ __forceinline__ L eu_pair(int p, L u, L v) {
    return p == 1 ? u : (p == 2 ? v : (p == 3 ? ladd(u, v) : lsub(v, u)));
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

// T = sum of g: the reference's order in FP64; a balanced tree in the FP32
// lane arithmetic.
template <class A>
__device__ __forceinline__ A sum_g(const A (&g)[Q]) {
    if constexpr (std::is_same<A, double>::value) {
        A tn = g[0];
#pragma unroll
        for (int j = 1; j < Q; ++j) tn = tn + g[j];
        return tn;
    } else {
        return ladd(ladd(g[0], ladd(ladd(g[1], g[5]), ladd(g[2], g[6]))), ladd(ladd(g[3], g[7]), ladd(g[4], g[8])));
    }
}

// FP32 rho and u on the shifted populations h_i = f_i - w_i, from the pair
// sums a_p = h_p + h_opp and differences d_p = h_p - h_opp (p = 1..4; the
// collision reuses them): rho - 1 = h_0 + sum a_p, rho u_x = d_E + d_NE - d_NW,
// rho u_y = d_N + d_NE + d_NW, plus half the previous Guo force in u_y.
// f in lane units (h 2^EF): drho comes out scaled by 2^EF, rho and u not.
template <class L, int EF = 0>
__device__ __forceinline__ Macro<L, true> macro_f_lane(const L (&f)[Q], L fy_prev, typename LaneMask<L>::T wall) {
    L a[5], d[5];
#pragma unroll
    for (int p = 1; p <= 4; ++p) {
        a[p] = ladd(f[p], f[p + 4]);
        d[p] = lsub(f[p], f[p + 4]);
    }
    Macro<L, true> m;
    m.drho = ladd(ladd(f[0], ladd(a[1], a[2])), ladd(a[3], a[4]));
    if constexpr (EF == 0)
        m.rho = ladd(lbc<L>(1.0f), m.drho);
    else
        m.rho = lfma(m.drho, lbc<L>(p2(-EF)), lbc<L>(1.0f));
    m.inv_rho = lrcp(m.rho);
    const L inv_s = EF == 0 ? m.inv_rho : lmul(m.inv_rho, lbc<L>(p2(-EF)));
    const L un = lmul(lsub(ladd(d[1], d[3]), d[4]), inv_s);
    const L vn = lmul(lfma(lbc<L>(0.5f * p2(EF)), fy_prev, ladd(ladd(d[2], d[3]), d[4])), inv_s);
    m.ux = lsel(wall, lbc<L>(0.0f), un);
    m.uy = lsel(wall, lbc<L>(0.0f), vn);
    m.t = lbc<L>(0.0f);
    return m;
}

// rho and u of the node (t left 0): the f part of macro_node.
template <class A, bool SHIFT>
__device__ __forceinline__ Macro<A, SHIFT> macro_f(const A (&f)[Q], A fy_prev, bool wall) {
    if constexpr (SHIFT) {
        return macro_f_lane<A>(f, fy_prev, wall);
    } else {
        Macro<A, SHIFT> m;
        A s = f[0];
#pragma unroll
        for (int j = 1; j < Q; ++j) s = s + f[j];
        A un = ((((f[1] + f[3]) - f[4]) - f[5]) - f[7]) + f[8];
        A vn = ((((f[2] + f[3]) + f[4]) - f[6]) - f[7]) - f[8];
        const A r = s;
        m.drho = s - A(1.0);
        m.inv_rho = A(0.0);
        if (r > A(2.220446049250313e-16)) {
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
    A q[5];                // FP32: 4.5 (c_p.u)^2 - 1.5 u^2 (shared with the g equilibrium)
    A nut, w1, w2, k1, k2; // FP64 a_f, b_f, k-, k+;  FP32 om+, om-, k+, k-
};

// ---- FP32 collision over a lane type (float: one node, float2: two) --------
// On h_i = f_i - w_i, pairwise: for each pair p = (i, i+4), i = 1..4, split
// populations and equilibria into symmetric / antisymmetric parts.  The TRT
// update f_i += -a d_i - b d_opp + (1 - 1/2tau-) S-_i + (1 - 1/2tau+) S+_i
// with a = (w+ + w-)/2, b = (w+ - w-)/2 is exactly
//   f_p += E + O, f_opp += E - O,
//   E = -w+ (d_p + d_opp)/2 + k+ S+_p,  O = -w- (d_p - d_opp)/2 + k- S-_p,
// and pi_neq only needs the symmetric parts.  Same arithmetic as the
// reference up to rounding, a third of the operations.  f, drho and the
// non-equilibrium parts in lane units (scaled by 2^EF).
// The pieces of the pairwise split, each one expression so that every caller
// (whatever it keeps in registers and what it recomputes) gets the same bits.
template <class L>
__device__ __forceinline__ L m15u2_lane(L u, L v) {
    return lmul(lbc<L>(-1.5f), lfma(u, u, lmul(v, v)));
}
// q_p = 4.5 (c_p.u)^2 - 1.5 u^2
template <class L>
__device__ __forceinline__ L q_lane(int p, L u, L v, L m15u2) {
    const L eu = eu_pair<L>(p, u, v);
    return lfma(lbc<L>(4.5f), lmul(eu, eu), m15u2);
}
// (h_p + h_opp) - 2 w (drho + rho q)
template <class L>
__device__ __forceinline__ L dS_lane(int p, const L (&f)[Q], L r, L drho, L q) {
    return lfma(lbc<L>(-2.0f * float(WD(p))), lfma(r, q, drho), ladd(f[p], f[p + 4]));
}
// (h_p - h_opp) - 2 w rho 3 e.u
template <class L>
__device__ __forceinline__ L dD_lane(int p, const L (&f)[Q], L r, L u, L v) {
    return lfma(lbc<L>(-6.0f * float(WD(p))), lmul(r, eu_pair<L>(p, u, v)), lsub(f[p], f[p + 4]));
}
// rest: h_0 - (feq_0 - w_0) = h_0 - w_0 (drho - 1.5 rho u^2)
template <class L>
__device__ __forceinline__ L d0_lane(const L (&f)[Q], L r, L drho, L m15u2) {
    return lfma(lbc<L>(-float(WD(0))), lfma(r, m15u2, drho), f[0]);
}
template <class L, int EF>
__device__ __forceinline__ L rho_scaled(const Macro<L, true>& m) {
    return EF == 0 ? m.rho : lmul(m.rho, lbc<L>(p2(EF)));  // rho 2^EF
}

// The relaxation coefficients alone (nu_t from pi_neq, 1/tau+-, k+-): what
// collide_f_pre_lane computes besides the non-equilibrium parts.
template <class L>
struct CollCoef {
    L nut, w1, w2, k1, k2;
};
template <class L, int EF = 0>
__device__ __forceinline__ CollCoef<L> collide_f_coef_lane(const L (&f)[Q], const Macro<L, true>& m,
                                                           const StepScalars<float>& c, const L* nut_ovr) {
    CollCoef<L> o;
    const L u = m.ux, v = m.uy, r = rho_scaled<L, EF>(m), m15u2 = m15u2_lane<L>(u, v);
    L dS[5];
#pragma unroll
    for (int p = 1; p <= 4; ++p) dS[p] = dS_lane<L>(p, f, r, m.drho, q_lane<L>(p, u, v, m15u2));
    // pi_neq (solver.rs:1096-1106) from the symmetric parts.
    const L s34 = ladd(dS[3], dS[4]);
    const L pxx = ladd(dS[1], s34), pyy = ladd(dS[2], s34), pxy = lsub(dS[3], dS[4]);
    const L pi2 = lfma(pxx, pxx, lfma(lmul(lbc<L>(2.0f), pxy), pxy, lmul(pyy, pyy)));
    // nu_t = Cs^2 |S|, |S| = sqrt(pi:pi) / (2 cs^2 tau rho) = sqrt(pi:pi) (1.5 / tau) / rho
    const float kS = c.cs * c.cs * (1.5f * c.inv_tau_s) * p2(-EF);
    o.nut = nut_ovr ? *nut_ovr : lmul(lmul(lsqrt(pi2), lbc<L>(kS)), m.inv_rho);
    const L e = lfma(lbc<L>(3.0f), o.nut, lbc<L>(3.0f * c.nu));          // tau+ - 1/2
    o.w1 = lrcp(ladd(lbc<L>(0.5f), e));                                     // 1/tau+
    o.w2 = lmul(e, lrcp(lfma(lbc<L>(0.5f), e, lbc<L>(float(LAMBDA_TRT)))));  // 1/tau-, tau- = 1/2 + Lambda/e
    o.k1 = lfma(lbc<L>(-0.5f), o.w1, lbc<L>(1.0f));
    o.k2 = lfma(lbc<L>(-0.5f), o.w2, lbc<L>(1.0f));
    return o;
}

// The non-equilibrium parts (d0, dS, dD) and q, around given coefficients.
template <class L, int EF = 0>
__device__ __forceinline__ CollF<L> collide_f_parts_lane(const L (&f)[Q], const Macro<L, true>& m,
                                                         const CollCoef<L>& k) {
    CollF<L> o;
    const L u = m.ux, v = m.uy, r = rho_scaled<L, EF>(m), m15u2 = m15u2_lane<L>(u, v);
    o.d0 = d0_lane<L>(f, r, m.drho, m15u2);
#pragma unroll
    for (int p = 1; p <= 4; ++p) {
        o.q[p] = q_lane<L>(p, u, v, m15u2);
        o.dS[p] = dS_lane<L>(p, f, r, m.drho, o.q[p]);
        o.dD[p] = dD_lane<L>(p, f, r, u, v);
    }
    o.nut = k.nut;
    o.w1 = k.w1;
    o.w2 = k.w2;
    o.k1 = k.k1;
    o.k2 = k.k2;
    return o;
}

template <class L, int EF = 0>
__device__ __forceinline__ CollF<L> collide_f_pre_lane(const L (&f)[Q], const Macro<L, true>& m,
                                                       const StepScalars<float>& c, const L* nut_ovr) {
    return collide_f_parts_lane<L, EF>(f, m, collide_f_coef_lane<L, EF>(f, m, c, nut_ovr));
}

// The f update with the Guo force fy = rho beta T: S+_p = w_p (-3 u_y +
// 9 (c_p.u) c_py) fy, S-_p = w_p 3 c_py fy.  f in lane units (2^EF), temp
// in g lane units (2^EG); returns fy unscaled.
template <class L, int EF = 0, int EG = 0>
__device__ __forceinline__ L collide_f_post_lane(L (&f)[Q], const CollF<L>& o, const Macro<L, true>& m,
                                                 const StepScalars<float>& c, L temp) {
    const L u = m.ux, v = m.uy;
    const L fyv = lmul(lmul(m.rho, lbc<L>(c.beta * p2(-EG))), temp);
    const L fys = EF == 0 ? fyv : lmul(fyv, lbc<L>(p2(EF)));
    const L gp = lmul(o.k1, fys), gm = lmul(o.k2, fys);       // k+ fy, k- fy
    const L hp = lmul(lbc<L>(-0.5f), o.w1), hm = lmul(lbc<L>(-0.5f), o.w2);
    const L m3v = lmul(lbc<L>(-3.0f), v);
    f[0] = lfma(lmul(lbc<L>(float(WD(0))), m3v), gp, lsub(f[0], lmul(o.w1, o.d0)));
    const L sa = lmul(lbc<L>(float(WD(1))), m3v), sd = lmul(lbc<L>(float(WD(3))), m3v);
    const L oa = lmul(lbc<L>(3.0f * float(WD(2))), gm), od = lmul(lbc<L>(3.0f * float(WD(3))), gm);
#pragma unroll
    for (int p = 1; p <= 4; ++p) {
        const float w = float(WD(p));
        const L w3v = p <= 2 ? sa : sd;
        const L sp = p == 1 ? w3v : lfma(lbc<L>(9.0f * w), eu_pair<L>(p, u, v), w3v);
        const L E = lfma(sp, gp, lmul(hp, o.dS[p]));
        const L O = p == 1 ? lmul(hm, o.dD[p]) : lfma(hm, o.dD[p], p == 2 ? oa : od);
        f[p] = ladd(f[p], ladd(E, O));
        f[p + 4] = ladd(f[p + 4], lsub(E, O));
    }
    return fyv;
}

// BGK of g towards geq (quadratic, or linear in u when c.geq_order == 1).
// q_p = 4.5 (c_p.u)^2 - 1.5 u^2 comes from the f collision (same u).  g and
// temp in the same (lane) units: the update is linear in both.
template <class L, bool LINEAR>
__device__ __forceinline__ void collide_g_lane_o(L (&g)[Q], L temp, L u, L v, L om, const L (&q)[5]) {
    const L one_m = lsub(lbc<L>(1.0f), om);
    const L B = lmul(om, temp);
    const L b0 = lmul(B, lbc<L>(float(WD(0))));
    const L ba = lmul(B, lbc<L>(float(WD(1)))), bd = lmul(B, lbc<L>(float(WD(3))));
    const L ba3 = lmul(lbc<L>(3.0f), ba), bd3 = lmul(lbc<L>(3.0f), bd);
    const L u2 = lfma(u, u, lmul(v, v));
    g[0] = lfma(one_m, g[0], LINEAR ? b0 : lfma(b0, lmul(lbc<L>(-1.5f), u2), b0));
#pragma unroll
    for (int p = 1; p <= 4; ++p) {
        const L bw = p <= 2 ? ba : bd;
        const L gS = LINEAR ? bw : lfma(bw, q[p], bw);
        const L gA = lmul(p <= 2 ? ba3 : bd3, eu_pair<L>(p, u, v));
        g[p] = lfma(one_m, g[p], ladd(gS, gA));
        g[p + 4] = lfma(one_m, g[p + 4], lsub(gS, gA));
    }
}
template <class L>
__device__ __forceinline__ void collide_g_lane(L (&g)[Q], L temp, L u, L v, L nut, const L (&q)[5],
                                               const StepScalars<float>& c, const L* at_ovr) {
    const L at = at_ovr ? *at_ovr : lmul(nut, lbc<L>(c.inv_pr_t));
    const L om = lrcp(lfma(lbc<L>(3.0f), at, lbc<L>(0.5f + 3.0f * c.alpha)));
    if (c.geq_order == 1)
        collide_g_lane_o<L, true>(g, temp, u, v, om, q);
    else
        collide_g_lane_o<L, false>(g, temp, u, v, om, q);
}

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
        o = collide_f_pre_lane<A>(f, m, c, nut_ovr);
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
        return collide_f_post_lane<A>(f, o, m, c, temp);
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
        A q[5];
        const A m15u2 = lmul(lbc<A>(-1.5f), lfma(u, u, lmul(v, v)));
#pragma unroll
        for (int p = 1; p <= 4; ++p) {
            const A eu = eu_pair<A>(p, u, v);
            q[p] = lfma(lbc<A>(4.5f), lmul(eu, eu), m15u2);
        }
        collide_g_lane<A>(g, temp, u, v, nut, q, c, at_ovr);
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
    if constexpr (SHIFT)
        collide_g_lane<A>(g, m.t, m.ux, m.uy, o.nut, o.q, c, at_ovr);
    else
        collide_g<A, SHIFT>(g, m.t, m.ux, m.uy, o.nut, c, at_ovr);
}

// The same collision on a lane type and in lane units (f scaled by 2^EF,
// g and m.t by 2^EG, m.drho by 2^EF).
template <class L, int EF, int EG>
__device__ __forceinline__ void collide_node_lane(L (&f)[Q], L (&g)[Q], const Macro<L, true>& m,
                                                  const StepScalars<float>& c, L& fy_out, L& nut_out) {
    const CollF<L> o = collide_f_pre_lane<L, EF>(f, m, c, nullptr);
    nut_out = o.nut;
    fy_out = collide_f_post_lane<L, EF, EG>(f, o, m, c, m.t);
    collide_g_lane<L>(g, m.t, m.ux, m.uy, o.nut, o.q, c, nullptr);
}

// Wall-node equilibrium of g (apply_thermal_boundary_conditions,
// src/uniform/solver.rs:957-970): geq(T_wall, 0, 0) = w_i T_wall.
template <class A>
__device__ __forceinline__ A geq_rest(int i, A t, int order) {
    return geq_full<A>(i, t, A(0.0), A(0.0), order);
}

}  // namespace cav
