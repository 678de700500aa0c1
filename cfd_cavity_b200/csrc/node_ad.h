// node_ad.h -- one node of the cavity step as a generic function of its
// inputs, and its hand-written reverse (adjoint).
//
// Forward: the node's pulled populations (f_i - w_i, g_i), the Guo force of
// the previous collision and the Smagorinsky constant Cs give the
// post-collision populations and the new Guo force.  It is the macroscopic
// update with the Guo half-force correction and no-slip
// (src/uniform/solver.rs:298-367, 992-1009) followed by collide_node
// (:1054-1185: TRT Lambda = 3/16 with nu_t = (Cs dx)^2 |S| from pi_neq, Guo
// forcing with per-mode factors, BGK for g), written per direction pair
// (i, opp(i)).  The reverse propagates adjoints of the outputs back to the
// inputs and to Cs; every intermediate is recomputed, nothing is stored.
// Non-smooth point: |S| = sqrt(pi:pi) at pi = 0 takes the subgradient 0.
//
// Plain C++ (host and device) so that the same code runs in double, float
// and dual numbers: the CPU tests check the reverse against forward-mode
// derivatives (dot-product test) without a GPU.
#pragma once

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#define __device__
#define __forceinline__ inline
#endif
#endif

#include <math.h>

namespace cav {
namespace ad {

__host__ __device__ constexpr int cx(int i) {
    return i == 1 || i == 3 || i == 8 ? 1 : (i == 4 || i == 5 || i == 7 ? -1 : 0);
}
__host__ __device__ constexpr int cy(int i) {
    return i == 2 || i == 3 || i == 4 ? 1 : (i == 6 || i == 7 || i == 8 ? -1 : 0);
}
__host__ __device__ constexpr double wd(int i) {
    return i == 0 ? 4.0 / 9.0 : (i == 1 || i == 2 || i == 5 || i == 6 ? 1.0 / 9.0 : 1.0 / 36.0);
}

template <class T>
__host__ __device__ __forceinline__ T sqrt_(T x) {
    return sqrt(x);
}
// FP32 on the device: the special-function unit's square root, as the FP32
// forward step uses.
template <>
__host__ __device__ __forceinline__ float sqrt_<float>(float x) {
#ifdef __CUDA_ARCH__
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return sqrtf(x);
#endif
}

// Division; FP32 on the device uses the fast approximate division (2 ulp),
// as the FP32 forward step does.
template <class T>
__host__ __device__ __forceinline__ T div_(T a, T b) {
    return a / b;
}
template <>
__host__ __device__ __forceinline__ float div_<float>(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}

// Per-step scalars of the collision (CollideCtx, src/uniform/solver.rs:1034-1043).
template <class T>
struct NodeScal {
    T beta, nu, alpha, c1;  // c1 = 1.5 / tau_s (|S| = sqrt(pi:pi) * c1 / rho)
    T inv_pr_t, lambda;
    T q2;  // 1: quadratic g equilibrium, 0: linear
};

// Forward.  h[9] = f_i - w_i, g[9] pulled; fyp = fy of the previous
// collision; outputs overwrite ho[9], go[9] and return fy; *t_out = T.
template <class T>
__host__ __device__ __forceinline__ T node_forward(const T (&h)[9], const T (&g)[9], T fyp, bool wall, T cs,
                                                   const NodeScal<T>& c, T (&ho)[9], T (&go)[9], T* t_out) {
    T drho = h[0];
    for (int i = 1; i < 9; ++i) drho = drho + h[i];
    const T jx = h[1] + h[3] - h[4] - h[5] - h[7] + h[8];
    const T jy = h[2] + h[3] + h[4] - h[6] - h[7] - h[8];
    const T r = T(1.0) + drho;
    const T inv = div_(T(1.0), r);
    const T ux = wall ? T(0.0) : jx * inv;
    const T uy = wall ? T(0.0) : (jy + T(0.5) * fyp) * inv;
    T t = g[0];
    for (int i = 1; i < 9; ++i) t = t + g[i];
    if (t_out) *t_out = t;
    const T fy = r * c.beta * t;
    const T u2 = ux * ux + uy * uy;
    const T d0 = h[0] - T(wd(0)) * (drho - T(1.5) * r * u2);
    T dS[5], dD[5], eu[5];
    for (int p = 1; p <= 4; ++p) {
        eu[p] = T(double(cx(p))) * ux + T(double(cy(p))) * uy;
        const T feS = T(wd(p)) * (drho + r * (T(4.5) * eu[p] * eu[p] - T(1.5) * u2));
        const T feA = T(wd(p)) * (T(3.0) * r * eu[p]);
        dS[p] = h[p] + h[p + 4] - T(2.0) * feS;
        dD[p] = h[p] - h[p + 4] - T(2.0) * feA;
    }
    const T pxx = dS[1] + dS[3] + dS[4];
    const T pxy = dS[3] - dS[4];
    const T pyy = dS[2] + dS[3] + dS[4];
    const T pi2 = pxx * pxx + T(2.0) * pxy * pxy + pyy * pyy;
    const T sq = sqrt_(pi2);
    const T smag = sq * c.c1 * inv;
    const T nut = cs * cs * smag;
    const T e = T(3.0) * (c.nu + nut);
    const T om_p = div_(T(1.0), T(0.5) + e);
    const T om_m = div_(e, T(0.5) * e + c.lambda);
    const T om_g = div_(T(1.0), T(0.5) + T(3.0) * (c.alpha + nut * c.inv_pr_t));
    const T k_p = T(1.0) - T(0.5) * om_p, k_m = T(1.0) - T(0.5) * om_m;
    ho[0] = h[0] - om_p * d0 + k_p * T(wd(0)) * (T(-3.0) * uy) * fy;
    for (int p = 1; p <= 4; ++p) {
        const T A = T(-3.0) * uy + T(9.0) * eu[p] * T(double(cy(p)));
        const T E = T(-0.5) * om_p * dS[p] + k_p * T(wd(p)) * A * fy;
        const T O = T(-0.5) * om_m * dD[p] + k_m * T(wd(p)) * T(3.0 * cy(p)) * fy;
        ho[p] = h[p] + (E + O);
        ho[p + 4] = h[p + 4] + (E - O);
    }
    const T om1 = T(1.0) - om_g;
    go[0] = om1 * g[0] + om_g * T(wd(0)) * t * (T(1.0) - c.q2 * T(1.5) * u2);
    for (int p = 1; p <= 4; ++p) {
        const T B = T(1.0) + c.q2 * (T(4.5) * eu[p] * eu[p] - T(1.5) * u2);
        const T gS = om_g * T(wd(p)) * t * B;
        const T gA = om_g * T(wd(p)) * t * (T(3.0) * eu[p]);
        go[p] = om1 * g[p] + (gS + gA);
        go[p + 4] = om1 * g[p + 4] + (gS - gA);
    }
    return fy;
}

// Reverse.  Given the inputs and the adjoints of the outputs (af, ag, afy)
// plus a direct adjoint of T (at_obj, from an objective that reads T),
// writes the adjoints of the inputs (ah, agi, *afyp) and returns dJ/dCs.
template <class T>
__host__ __device__ __forceinline__ T node_reverse(const T (&h)[9], const T (&g)[9], T fyp, bool wall, T cs,
                                                   const NodeScal<T>& c, const T (&af)[9], const T (&ag)[9], T afy,
                                                   T at_obj, T (&ah)[9], T (&agi)[9], T* afyp) {
    // ---- forward recomputation -------------------------------------------
    T drho = h[0];
    for (int i = 1; i < 9; ++i) drho = drho + h[i];
    const T jx = h[1] + h[3] - h[4] - h[5] - h[7] + h[8];
    const T jy = h[2] + h[3] + h[4] - h[6] - h[7] - h[8];
    const T r = T(1.0) + drho;
    const T inv = div_(T(1.0), r);
    const T ux = wall ? T(0.0) : jx * inv;
    const T uy = wall ? T(0.0) : (jy + T(0.5) * fyp) * inv;
    T t = g[0];
    for (int i = 1; i < 9; ++i) t = t + g[i];
    const T fy = r * c.beta * t;
    const T u2 = ux * ux + uy * uy;
    const T d0 = h[0] - T(wd(0)) * (drho - T(1.5) * r * u2);
    T dS[5], dD[5], eu[5];
    for (int p = 1; p <= 4; ++p) {
        eu[p] = T(double(cx(p))) * ux + T(double(cy(p))) * uy;
        const T feS = T(wd(p)) * (drho + r * (T(4.5) * eu[p] * eu[p] - T(1.5) * u2));
        const T feA = T(wd(p)) * (T(3.0) * r * eu[p]);
        dS[p] = h[p] + h[p + 4] - T(2.0) * feS;
        dD[p] = h[p] - h[p + 4] - T(2.0) * feA;
    }
    const T pxx = dS[1] + dS[3] + dS[4];
    const T pxy = dS[3] - dS[4];
    const T pyy = dS[2] + dS[3] + dS[4];
    const T pi2 = pxx * pxx + T(2.0) * pxy * pxy + pyy * pyy;
    const T sq = sqrt_(pi2);
    const T smag = sq * c.c1 * inv;
    const T nut = cs * cs * smag;
    const T e = T(3.0) * (c.nu + nut);
    const T om_p = div_(T(1.0), T(0.5) + e);
    const T den_m = T(0.5) * e + c.lambda;
    const T om_m = div_(e, den_m);
    const T om_g = div_(T(1.0), T(0.5) + T(3.0) * (c.alpha + nut * c.inv_pr_t));
    const T k_p = T(1.0) - T(0.5) * om_p, k_m = T(1.0) - T(0.5) * om_m;
    const T om1 = T(1.0) - om_g;

    // ---- reverse -------------------------------------------------------------
    T b_t = at_obj, b_u2 = T(0.0), b_omg = T(0.0), b_om1 = T(0.0);
    T b_omp = T(0.0), b_omm = T(0.0), b_kp = T(0.0), b_km = T(0.0);
    T b_ux = T(0.0), b_uy = T(0.0), b_fy = afy, b_d0 = T(0.0);
    T b_eu[5], b_dS[5], b_dD[5];
    for (int p = 0; p < 5; ++p) b_eu[p] = b_dS[p] = b_dD[p] = T(0.0);
    for (int i = 0; i < 9; ++i) ah[i] = agi[i] = T(0.0);

    // g outputs
    {
        const T q0 = T(1.0) - c.q2 * T(1.5) * u2;
        agi[0] = agi[0] + om1 * ag[0];
        b_om1 = b_om1 + g[0] * ag[0];
        b_omg = b_omg + T(wd(0)) * t * q0 * ag[0];
        b_t = b_t + om_g * T(wd(0)) * q0 * ag[0];
        b_u2 = b_u2 - om_g * T(wd(0)) * t * c.q2 * T(1.5) * ag[0];
    }
    for (int p = 1; p <= 4; ++p) {
        const T s = ag[p] + ag[p + 4], d = ag[p] - ag[p + 4];
        const T B = T(1.0) + c.q2 * (T(4.5) * eu[p] * eu[p] - T(1.5) * u2);
        agi[p] = agi[p] + om1 * ag[p];
        agi[p + 4] = agi[p + 4] + om1 * ag[p + 4];
        b_om1 = b_om1 + g[p] * ag[p] + g[p + 4] * ag[p + 4];
        const T w = T(wd(p));
        b_omg = b_omg + w * t * B * s + w * t * T(3.0) * eu[p] * d;
        b_t = b_t + om_g * w * B * s + om_g * w * T(3.0) * eu[p] * d;
        const T b_B = om_g * w * t * s;
        b_eu[p] = b_eu[p] + om_g * w * t * T(3.0) * d + c.q2 * T(9.0) * eu[p] * b_B;
        b_u2 = b_u2 - c.q2 * T(1.5) * b_B;
    }
    b_omg = b_omg - b_om1;

    // f outputs
    ah[0] = ah[0] + af[0];
    b_omp = b_omp - d0 * af[0];
    b_d0 = b_d0 - om_p * af[0];
    b_kp = b_kp + T(wd(0)) * (T(-3.0) * uy) * fy * af[0];
    b_uy = b_uy + k_p * T(wd(0)) * T(-3.0) * fy * af[0];
    b_fy = b_fy + k_p * T(wd(0)) * (T(-3.0) * uy) * af[0];
    for (int p = 1; p <= 4; ++p) {
        const T bE = af[p] + af[p + 4], bO = af[p] - af[p + 4];
        const T w = T(wd(p));
        const T cyp = T(double(cy(p)));
        const T A = T(-3.0) * uy + T(9.0) * eu[p] * cyp;
        ah[p] = ah[p] + af[p];
        ah[p + 4] = ah[p + 4] + af[p + 4];
        b_omp = b_omp - T(0.5) * dS[p] * bE;
        b_dS[p] = b_dS[p] - T(0.5) * om_p * bE;
        b_kp = b_kp + w * A * fy * bE;
        const T b_A = k_p * w * fy * bE;
        b_fy = b_fy + k_p * w * A * bE;
        b_uy = b_uy - T(3.0) * b_A;
        b_eu[p] = b_eu[p] + T(9.0) * cyp * b_A;
        b_omm = b_omm - T(0.5) * dD[p] * bO;
        b_dD[p] = b_dD[p] - T(0.5) * om_m * bO;
        b_km = b_km + w * T(3.0) * cyp * fy * bO;
        b_fy = b_fy + k_m * w * T(3.0) * cyp * bO;
    }
    b_omp = b_omp - T(0.5) * b_kp;
    b_omm = b_omm - T(0.5) * b_km;

    // relaxation rates -> nut -> (Cs, |S|)
    T b_nut = b_omg * (T(-3.0) * c.inv_pr_t * om_g * om_g);
    const T b_e = b_omm * div_(c.lambda, den_m * den_m) - b_omp * om_p * om_p;
    b_nut = b_nut + T(3.0) * b_e;
    const T b_cs = T(2.0) * cs * smag * b_nut;
    const T b_smag = cs * cs * b_nut;
    T b_inv = sq * c.c1 * b_smag;
    const T b_sq = c.c1 * inv * b_smag;
    T b_pxx = T(0.0), b_pxy = T(0.0), b_pyy = T(0.0);
    if (pi2 > T(0.0)) {  // subgradient 0 at pi = 0
        const T k = div_(b_sq, sq);
        b_pxx = k * pxx;
        b_pxy = k * T(2.0) * pxy;
        b_pyy = k * pyy;
    }
    b_dS[1] = b_dS[1] + b_pxx;
    b_dS[3] = b_dS[3] + b_pxx + b_pxy + b_pyy;
    b_dS[4] = b_dS[4] + b_pxx - b_pxy + b_pyy;
    b_dS[2] = b_dS[2] + b_pyy;

    // equilibrium deviations
    T b_drho = T(0.0), b_r = T(0.0);
    for (int p = 1; p <= 4; ++p) {
        const T w = T(wd(p));
        ah[p] = ah[p] + b_dS[p] + b_dD[p];
        ah[p + 4] = ah[p + 4] + b_dS[p] - b_dD[p];
        const T b_feS = T(-2.0) * b_dS[p];
        const T b_feA = T(-2.0) * b_dD[p];
        b_drho = b_drho + w * b_feS;
        b_r = b_r + w * (T(4.5) * eu[p] * eu[p] - T(1.5) * u2) * b_feS + w * T(3.0) * eu[p] * b_feA;
        b_eu[p] = b_eu[p] + w * r * T(9.0) * eu[p] * b_feS + w * T(3.0) * r * b_feA;
        b_u2 = b_u2 - T(1.5) * w * r * b_feS;
    }
    ah[0] = ah[0] + b_d0;
    {
        const T b_feq0 = -b_d0;
        b_drho = b_drho + T(wd(0)) * b_feq0;
        b_r = b_r - T(1.5) * T(wd(0)) * u2 * b_feq0;
        b_u2 = b_u2 - T(1.5) * T(wd(0)) * r * b_feq0;
    }
    for (int p = 1; p <= 4; ++p) {
        b_ux = b_ux + T(double(cx(p))) * b_eu[p];
        b_uy = b_uy + T(double(cy(p))) * b_eu[p];
    }
    b_ux = b_ux + T(2.0) * ux * b_u2;
    b_uy = b_uy + T(2.0) * uy * b_u2;
    // fy = r beta T
    b_r = b_r + c.beta * t * b_fy;
    b_t = b_t + r * c.beta * b_fy;
    for (int i = 0; i < 9; ++i) agi[i] = agi[i] + b_t;
    // macroscopic update
    T b_jx = T(0.0), b_jy = T(0.0), b_fyp = T(0.0);
    if (!wall) {
        b_jx = inv * b_ux;
        b_inv = b_inv + jx * b_ux;
        b_jy = inv * b_uy;
        b_fyp = T(0.5) * inv * b_uy;
        b_inv = b_inv + (jy + T(0.5) * fyp) * b_uy;
    }
    b_r = b_r - inv * inv * b_inv;
    b_drho = b_drho + b_r;
    for (int i = 0; i < 9; ++i)
        ah[i] = ah[i] + b_drho + T(double(cx(i))) * b_jx + T(double(cy(i))) * b_jy;
    *afyp = b_fyp;
    return b_cs;
}

}  // namespace ad
}  // namespace cav
