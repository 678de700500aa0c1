// sgs.cuh -- the dynamic mixed-scale subgrid model of the uniform cavity
// (compute_dynamic_sgs, src/uniform/solver.rs:562-828; box_filter / ddx /
// ddy / lilly_coefficient :1195-1261), evaluated on the GPU before the
// collision of a step, on the REF state (post-stream populations and
// fields).  The octree runs the same kernels on each level
// (compute_dynamic_sgs_level, src/octree/smag.rs:144-416: the same
// algorithm with the level's tau, nu and alpha in its own lattice units).
//
// Three kernels, each one thread per node, every quantity in FP64 whatever
// the storage format (the reference's arithmetic); a launch covers
// gridDim.z grids of one shape (the two blocks of an octree level):
//   k_sgs_b  test-filter boxes of u_x, u_y, T (at the node and at the four
//            neighbours its central differences read, each box summed in
//            the reference's window order) and of the five products
//            (Leonard terms at the test level); grid-level S~ and |S~| from
//            pi_neq (the collision's formula), test-level S-bar and
//            temperature gradients by central differences, similarity scales
//            qsm^1/2 and Phi_sm^1/2, |T~|, |T-bar|;
//   k_sgs_c  box of qsm^1/2 and Phi_sm^1/2, the interpolated mixed forms
//            (a^alpha b^(1-alpha)), Germano tensors M and L, Lilly numerators
//            and denominators;
//   k_sgs_d  box of the numerators and denominators (regularisation),
//            Lilly coefficients clamped to [0, 0.04], nu_t and alpha_t bounded
//            below by the TRT floor, written for the collision.
// Sums run in the reference's order (box windows row by row), so every
// quantity but the a^alpha powers (CUDA's pow, within 2 ulp of the
// reference's) is bit-identical in FP64.
#pragma once

#include "kernels.cuh"

namespace cav {

constexpr double C_DYN_MAX = 0.04;       // src/uniform/solver.rs:25
constexpr double TAU_TRT_FLOOR = 0.505;  // src/uniform/solver.rs:31

// Work planes (FP64, ny x pitch each).
enum SgsPlane {
    S_UBX, S_UBY, S_TB, S_LXX, S_LXY, S_LYY, S_LTX, S_LTY,             // k_sgs_a
    S_SHXX, S_SHXY, S_SHYY, S_SMH, S_SBXX, S_SBXY, S_SBYY, S_SMB,    // k_sgs_b
    S_GTX, S_GTY, S_GBX, S_GBY, S_QSM, S_PHI, S_TMH, S_TMB,          // k_sgs_b
    S_NUMV, S_DENV, S_NUMK, S_DENK, S_NUMIX, S_KAPMIX,               // k_sgs_c
    S_CNU, S_CK,                                                     // k_sgs_d
    S_NPLANES
};

// One grid's inputs and outputs; a launch takes two (blockIdx.z).
template <class St>
struct SgsGrid {
    const St* pops;                    // REF populations
    const typename Fmt<St>::A* rho;    // fields (rho stored minus sp.rho_off)
    const typename Fmt<St>::A* ux;
    const typename Fmt<St>::A* uy;
    const typename Fmt<St>::A* tt;
    double* W;                          // S_NPLANES work planes
    typename Fmt<St>::A* nut;           // nu_t_pre out
    typename Fmt<St>::A* at;            // alpha_t_pre out
};
template <class St>
struct SgsGrids {
    SgsGrid<St> g[2];
};

struct SgsParams {
    int width = 2;           // box width in nodes: max(round(eta_test), 1)
    double dtest = 2.0;      // test filter width eta * dx (dx = 1)
    double alpha_exp = 0.5;  // smag_alpha
    double tau_s = 0.5;      // uniform: 0.5 + 3 max(nu_eff, 0.002/3), as in the collision;
                             // octree level: 0.5 + 3 nu of the level
    double nu_mol = 0.0, alpha_mol = 0.0, nu_sm_min = -0.1;
    double rho_off = 0.0;    // added to the stored density (1 when the format stores rho - 1)
};

struct Window {
    int x0, x1, y0, y1;
    double cnt;
};

// box_filter's window (src/uniform/solver.rs:1204-1227): `width` nodes
// starting (width - 1) / 2 before the node, clamped to the grid.
__device__ __forceinline__ Window box_window(const Geom& G, int ix, int iy, int width) {
    const int hl = (width - 1) / 2;
    Window w;
    w.y0 = iy - hl < 0 ? 0 : iy - hl;
    w.y1 = iy + width - hl < G.ny ? iy + width - hl : G.ny;
    w.x0 = ix - hl < 0 ? 0 : ix - hl;
    w.x1 = ix + width - hl < G.nx ? ix + width - hl : G.nx;
    w.cnt = double((w.y1 - w.y0) * (w.x1 - w.x0));
    return w;
}

// ddx / ddy (src/uniform/solver.rs:1229-1245): central, clamped at the walls.
template <class A>
__device__ __forceinline__ double ddx_f(const A* __restrict__ p, const Geom& G, int ix, int iy) {
    const int xm = ix == 0 ? 0 : ix - 1, xp = ix + 1 >= G.nx ? G.nx - 1 : ix + 1;
    return 0.5 * (double(p[iy * G.pitch + xp]) - double(p[iy * G.pitch + xm]));
}
template <class A>
__device__ __forceinline__ double ddy_f(const A* __restrict__ p, const Geom& G, int ix, int iy) {
    const int ym = iy == 0 ? 0 : iy - 1, yp = iy + 1 >= G.ny ? G.ny - 1 : iy + 1;
    return 0.5 * (double(p[yp * G.pitch + ix]) - double(p[ym * G.pitch + ix]));
}

// lilly_coefficient (src/uniform/solver.rs:1250-1261).
__host__ __device__ __forceinline__ double lilly_coefficient(double num, double den) {
    if (!isfinite(den) || !isfinite(num) || den <= 0.0) return 0.0;
    const double c = 0.5 * num / den;
    if (!isfinite(c)) return 0.0;
    return c < 0.0 ? 0.0 : (c > C_DYN_MAX ? C_DYN_MAX : c);
}

// Test-filter box of u_x, u_y, T at (x, y): box_filter's window and order.
template <class A>
__device__ __forceinline__ void box3(const A* __restrict__ ux, const A* __restrict__ uy, const A* __restrict__ tt,
                                     const Geom& G, int x, int y, int width, double& bu, double& bv, double& bt) {
    const Window w = box_window(G, x, y, width);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int yy = w.y0; yy < w.y1; ++yy)
        for (int xx = w.x0; xx < w.x1; ++xx) {
            const int k = yy * G.pitch + xx;
            s0 += double(ux[k]);
            s1 += double(uy[k]);
            s2 += double(tt[k]);
        }
    bu = s0 / w.cnt;
    bv = s1 / w.cnt;
    bt = s2 / w.cnt;
}

template <class St>
__global__ void __launch_bounds__(128) k_sgs_b(SgsGrids<St> S, Geom G, SgsParams sp) {
    using A = typename Fmt<St>::A;
    constexpr bool SH = Fmt<St>::SHIFT;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const SgsGrid<St> io = S.g[blockIdx.z];
    double* __restrict__ W = io.W;
    const A* ux = io.ux;
    const A* uy = io.uy;
    const A* tt = io.tt;
    const long long P = G.plane;
    const int k = iy * G.pitch + ix;
    // test-filter boxes at the node and at the neighbours of its central
    // differences (ddx / ddy clamp at the walls), and the Leonard boxes
    const int xm = ix == 0 ? 0 : ix - 1, xp = ix + 1 >= G.nx ? G.nx - 1 : ix + 1;
    const int ym = iy == 0 ? 0 : iy - 1, yp = iy + 1 >= G.ny ? G.ny - 1 : iy + 1;
    double ubx, uby, tb, ubx_xm, uby_xm, tb_xm, ubx_xp, uby_xp, tb_xp, ubx_ym, uby_ym, tb_ym, ubx_yp, uby_yp, tb_yp;
    box3<A>(ux, uy, tt, G, ix, iy, sp.width, ubx, uby, tb);
    box3<A>(ux, uy, tt, G, xm, iy, sp.width, ubx_xm, uby_xm, tb_xm);
    box3<A>(ux, uy, tt, G, xp, iy, sp.width, ubx_xp, uby_xp, tb_xp);
    box3<A>(ux, uy, tt, G, ix, ym, sp.width, ubx_ym, uby_ym, tb_ym);
    box3<A>(ux, uy, tt, G, ix, yp, sp.width, ubx_yp, uby_yp, tb_yp);
    {
        const Window w = box_window(G, ix, iy, sp.width);
        double l[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int yy = w.y0; yy < w.y1; ++yy)
            for (int xx = w.x0; xx < w.x1; ++xx) {
                const int kk = yy * G.pitch + xx;
                const double u = ux[kk], v = uy[kk], t = tt[kk];
                l[0] += u * u;
                l[1] += u * v;
                l[2] += v * v;
                l[3] += u * t;
                l[4] += v * t;
            }
        W[S_UBX * P + k] = ubx;
        W[S_UBY * P + k] = uby;
        W[S_TB * P + k] = tb;
#pragma unroll
        for (int p = 0; p < 5; ++p) W[(S_LXX + p) * P + k] = l[p] / w.cnt;
    }
    const double rho_k = double(io.rho[k]) + sp.rho_off, ux_k = ux[k], uy_k = uy[k], t_k = tt[k];
    double pi_xx = 0.0, pi_xy = 0.0, pi_yy = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const double cx = CX(i), cy = CY(i);
        const double fi = double(ldp(io.pops, G, i, iy, ix)) + (SH ? WD(i) : 0.0);
        const double fneq = fi - feq_full<double>(i, rho_k, ux_k, uy_k);
        pi_xx += fneq * cx * cx;
        pi_xy += fneq * cx * cy;
        pi_yy += fneq * cy * cy;
    }
    const double rho_m = rho_k > 1e-12 ? rho_k : 1e-12;
    const double denom = 2.0 * CS2 * sp.tau_s * rho_m;
    const double pi2 = pi_xx * pi_xx + 2.0 * pi_xy * pi_xy + pi_yy * pi_yy;
    const double shxx = -pi_xx / denom, shxy = -pi_xy / denom, shyy = -pi_yy / denom;
    W[S_SHXX * P + k] = shxx;
    W[S_SHXY * P + k] = shxy;
    W[S_SHYY * P + k] = shyy;
    W[S_SMH * P + k] = sqrt(pi2) / denom;
    // ddx / ddy of the boxed fields (src/uniform/solver.rs:1229-1245)
    const double sxx = 0.5 * (ubx_xp - ubx_xm);
    const double syy = 0.5 * (uby_yp - uby_ym);
    const double sxy = 0.5 * (0.5 * (uby_xp - uby_xm) + 0.5 * (ubx_yp - ubx_ym));
    W[S_SBXX * P + k] = sxx;
    W[S_SBXY * P + k] = sxy;
    W[S_SBYY * P + k] = syy;
    W[S_SMB * P + k] = sqrt(sxx * sxx + 2.0 * sxy * sxy + syy * syy);
    const double gtx = ddx_f(tt, G, ix, iy), gty = ddy_f(tt, G, ix, iy);
    const double gbx = 0.5 * (tb_xp - tb_xm), gby = 0.5 * (tb_yp - tb_ym);
    W[S_GTX * P + k] = gtx;
    W[S_GTY * P + k] = gty;
    W[S_GBX * P + k] = gbx;
    W[S_GBY * P + k] = gby;
    const double dux = ux_k - ubx, duy = uy_k - uby;
    const double du2 = dux * dux + duy * duy;
    W[S_QSM * P + k] = sqrt(0.5 * du2) / 2.0;
    const double dt_local = t_k - tb;
    W[S_PHI * P + k] = 0.5 * fabs(dt_local) * sqrt(0.5 * du2);
    const double th_x = gtx * shxx + gty * shxy;
    const double th_y = gtx * shxy + gty * shyy;
    W[S_TMH * P + k] = sqrt(2.0 * (th_x * th_x + th_y * th_y));
    const double tb_x = gbx * sxx + gby * sxy;
    const double tb_y = gbx * sxy + gby * syy;
    W[S_TMB * P + k] = sqrt(2.0 * (tb_x * tb_x + tb_y * tb_y));
}

template <class St>
__global__ void __launch_bounds__(128) k_sgs_c(SgsGrids<St> S, Geom G, SgsParams sp) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    double* __restrict__ W = S.g[blockIdx.z].W;
    const long long P = G.plane;
    const int k = iy * G.pitch + ix;
    const Window w = box_window(G, ix, iy, sp.width);
    double sq = 0.0, sph = 0.0;
    for (int yy = w.y0; yy < w.y1; ++yy)
        for (int xx = w.x0; xx < w.x1; ++xx) {
            const int kk = yy * G.pitch + xx;
            sq += W[S_QSM * P + kk];
            sph += W[S_PHI * P + kk];
        }
    const double qbar_h = sq / w.cnt, phibar_h = sph / w.cnt;
    const double ae = sp.alpha_exp, dx = 1.0, dtest = sp.dtest, delta_t = 1.0;
    const double nu_mix_t = pow(dtest * dtest * W[S_SMB * P + k], ae) * pow(dtest * qbar_h, 1.0 - ae);
    const double nu_mix_g = pow(dx * dx * W[S_SMH * P + k], ae) * pow(dx * W[S_QSM * P + k], 1.0 - ae);
    const double kap_mix_t =
        pow(dtest * dtest * dtest / delta_t * W[S_TMB * P + k], ae) * pow(dtest / delta_t * phibar_h, 1.0 - ae);
    const double kap_mix_g =
        pow(dx * dx * dx / delta_t * W[S_TMH * P + k], ae) * pow(dx / delta_t * W[S_PHI * P + k], 1.0 - ae);
    const double mxx = nu_mix_t * W[S_SBXX * P + k] - nu_mix_g * W[S_SHXX * P + k];
    const double mxy = nu_mix_t * W[S_SBXY * P + k] - nu_mix_g * W[S_SHXY * P + k];
    const double myy = nu_mix_t * W[S_SBYY * P + k] - nu_mix_g * W[S_SHYY * P + k];
    const double mx = kap_mix_t * W[S_GBX * P + k] - kap_mix_g * W[S_GTX * P + k];
    const double my = kap_mix_t * W[S_GBY * P + k] - kap_mix_g * W[S_GTY * P + k];
    const double ubx = W[S_UBX * P + k], uby = W[S_UBY * P + k], tb = W[S_TB * P + k];
    const double lxx = W[S_LXX * P + k] - ubx * ubx;
    const double lxy = W[S_LXY * P + k] - ubx * uby;
    const double lyy = W[S_LYY * P + k] - uby * uby;
    const double lkk3 = (lxx + lyy) / 3.0;
    const double ldxx = lxx - lkk3, ldyy = lyy - lkk3;
    const double ljx = W[S_LTX * P + k] - ubx * tb;
    const double ljy = W[S_LTY * P + k] - uby * tb;
    W[S_NUMV * P + k] = ldxx * mxx + 2.0 * lxy * mxy + ldyy * myy;
    W[S_DENV * P + k] = mxx * mxx + 2.0 * mxy * mxy + myy * myy;
    W[S_NUMK * P + k] = ljx * mx + ljy * my;
    W[S_DENK * P + k] = mx * mx + my * my;
    W[S_NUMIX * P + k] = nu_mix_g;
    W[S_KAPMIX * P + k] = kap_mix_g;
}

template <class St>
__global__ void __launch_bounds__(128) k_sgs_d(SgsGrids<St> S, Geom G, SgsParams sp) {
    using A = typename Fmt<St>::A;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    double* __restrict__ W = S.g[blockIdx.z].W;
    A* __restrict__ nut_pre = S.g[blockIdx.z].nut;
    A* __restrict__ at_pre = S.g[blockIdx.z].at;
    const long long P = G.plane;
    const int k = iy * G.pitch + ix;
    const Window w = box_window(G, ix, iy, sp.width);
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int yy = w.y0; yy < w.y1; ++yy)
        for (int xx = w.x0; xx < w.x1; ++xx) {
            const int kk = yy * G.pitch + xx;
#pragma unroll
            for (int p = 0; p < 4; ++p) s[p] += W[(S_NUMV + p) * P + kk];
        }
    const double cnu = lilly_coefficient(s[0] / w.cnt, s[1] / w.cnt);
    const double ck = lilly_coefficient(s[2] / w.cnt, s[3] / w.cnt);
    W[S_CNU * P + k] = cnu;
    W[S_CK * P + k] = ck;
    const double margin = (TAU_TRT_FLOOR - 0.5) / 3.0;
    const double nt = cnu * W[S_NUMIX * P + k];
    const double nu_t_min = fmax(sp.nu_sm_min * sp.nu_mol, margin - sp.nu_mol);
    nut_pre[k] = A(nt < nu_t_min ? nu_t_min : nt);
    const double at = ck * W[S_KAPMIX * P + k];
    const double alpha_t_min = fmax(sp.nu_sm_min * sp.alpha_mol, margin - sp.alpha_mol);
    at_pre[k] = A(at < alpha_t_min ? alpha_t_min : at);
}

// Mean and max of the Lilly coefficients (cs_dyn_mean / _max, kappa_dyn_mean
// / _max): one CTA, sums in a fixed order.
static __global__ void __launch_bounds__(256) k_sgs_stats(const double* __restrict__ W, Geom G,
                                                          double* __restrict__ out) {
    const long long P = G.plane;
    __shared__ double sh[4][256];
    double s0 = 0.0, m0 = 0.0, s1 = 0.0, m1 = 0.0;
    const int n = G.nx * G.ny;
    for (int j = threadIdx.x; j < n; j += 256) {
        const int k = (j / G.nx) * G.pitch + (j % G.nx);
        const double a = W[S_CNU * P + k], b = W[S_CK * P + k];
        s0 += a;
        m0 = fmax(m0, a);
        s1 += b;
        m1 = fmax(m1, b);
    }
    sh[0][threadIdx.x] = s0;
    sh[1][threadIdx.x] = m0;
    sh[2][threadIdx.x] = s1;
    sh[3][threadIdx.x] = m1;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
        for (int t = 0; t < 256; ++t) {
            a += sh[0][t];
            b = fmax(b, sh[1][t]);
            c += sh[2][t];
            d = fmax(d, sh[3][t]);
        }
        out[0] = a / double(n);
        out[1] = b;
        out[2] = c / double(n);
        out[3] = d;
    }
}

}  // namespace cav
