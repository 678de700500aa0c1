// diag.cuh -- deterministic FP64 reductions over a REF state: the
// diagnostics the reference computes on the host every progress_every steps
// (src/uniform/post.rs:68-199, 406-411; src/uniform/solver.rs:1012-1020;
// src/main.rs:168-276).  Warp shuffles, then a fixed-order block tree, then
// one block over the per-block partials: no floating-point atomics, so the
// result does not depend on scheduling.
#pragma once

#include "lattice.cuh"

namespace cav {

constexpr int DIAG_THREADS = 256;
constexpr int DIAG_NPART = 8;  // sum_rho, sum_f, max_u, max_uy, max_nut, nonfinite, sum_vol, spare

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide reduction of NV values (sum or max per slot) into out[0..NV).
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], const bool (&is_max)[NV], double* out) {
    __shared__ double sh[NV][DIAG_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double r = is_max[j] ? warp_max(v[j]) : warp_sum(v[j]);
        if (lane == 0) sh[j][wid] = r;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double r = lane < DIAG_THREADS / 32 ? sh[j][lane] : (is_max[j] ? 0.0 : 0.0);
            r = is_max[j] ? warp_max(r) : warp_sum(r);
            if (lane == 0) out[j] = r;
        }
    }
}

// Pass 1: per-block partials over the nodes.  max values are of absolute
// values (>= 0), so 0 is the neutral element.
template <class St>
__global__ void __launch_bounds__(DIAG_THREADS) k_diag_partials(const St* __restrict__ pop,
                                                                 const typename Fmt<St>::A* __restrict__ rho,
                                                                 const typename Fmt<St>::A* __restrict__ ux,
                                                                 const typename Fmt<St>::A* __restrict__ uy,
                                                                 const typename Fmt<St>::A* __restrict__ tt,
                                                                 const typename Fmt<St>::A* __restrict__ nut,
                                                                 double* __restrict__ partials, Geom G) {
    const long long n = (long long)G.nx * G.ny;
    double v[DIAG_NPART] = {0, 0, 0, 0, 0, 0, 0, 0};
    const bool is_max[DIAG_NPART] = {false, false, true, true, true, false, false, false};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int iy = int(idx / G.nx), ix = int(idx % G.nx);
        const long long k = (long long)iy * G.pitch + ix;
        const double r = rho[k], u = ux[k], w = uy[k], t = tt[k];
        double sf = 0.0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            double fv = double(ldp(pop, G, i, iy, ix));
            if (Fmt<St>::SHIFT) fv += WD(i);
            sf += fv;
        }
        v[0] += r;
        v[1] += sf;
        v[2] = fmax(v[2], fmax(fabs(u), fabs(w)));
        v[3] = fmax(v[3], fabs(w));
        v[4] = fmax(v[4], fabs(double(nut[k])));
        bool fin = isfinite(t) && isfinite(u) && isfinite(w) && isfinite(r) && r > 0.0;
        v[5] += fin ? 0.0 : 1.0;
        if (ix >= 1 && ix <= G.nx - 2 && iy >= 1 && iy <= G.ny - 2) v[6] += w * t;
    }
    block_reduce<DIAG_NPART>(v, is_max, partials + (long long)blockIdx.x * DIAG_NPART);
}

// Pass 2 (one block): partials in fixed order, plus the per-row Nusselt and
// y+ sums.  out[]: nu_hot, nu_cold, nu_link0, sum_rho, sum_f, max_u, max_uy,
// nut_max, y_plus, nu_volume, nonfinite.
template <class A>
__global__ void __launch_bounds__(DIAG_THREADS) k_diag_final(const double* __restrict__ partials, int nparts,
                                                              const A* __restrict__ ux, const A* __restrict__ uy,
                                                              const A* __restrict__ tt, const A* __restrict__ nut,
                                                              double nu_mol, double lz, double* __restrict__ out,
                                                              Geom G) {
    double v[DIAG_NPART + 4];
    bool is_max[DIAG_NPART + 4];
#pragma unroll
    for (int j = 0; j < DIAG_NPART + 4; ++j) {
        v[j] = 0.0;
        is_max[j] = (j == 2 || j == 3 || j == 4);
    }
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
#pragma unroll
        for (int j = 0; j < DIAG_NPART; ++j) {
            double p = partials[(long long)b * DIAG_NPART + j];
            v[j] = is_max[j] ? fmax(v[j], p) : v[j] + p;
        }
    }
    for (int iy = threadIdx.x; iy < G.ny; iy += blockDim.x) {
        const long long r = (long long)iy * G.pitch;
        v[DIAG_NPART + 0] += fabs(double(tt[r + 1]) - double(tt[r + 2]));
        v[DIAG_NPART + 1] += fabs(double(tt[r + G.nx - 2]) - double(tt[r + G.nx - 3]));
        v[DIAG_NPART + 2] += fabs(double(tt[r + 0]) - double(tt[r + 1]));
        if (iy >= 1 && iy <= G.ny - 2) {
            // y_plus_hot, post.rs:182-199: tau_w = (nu + nu_t(1)) |u_y(1) - u_y(0)|,
            // y+ = 0.5 sqrt(max(tau_w, 0)) / nu.
            double nu_eff = nu_mol + double(nut[r + 1]);
            double du = fabs(double(uy[r + 1]) - double(uy[r + 0]));
            double tau_w = nu_eff * du;
            v[DIAG_NPART + 3] += 0.5 * sqrt(fmax(tau_w, 0.0)) / nu_mol;
        }
    }
    __shared__ double res[DIAG_NPART + 4];
    block_reduce<DIAG_NPART + 4>(v, is_max, res);
    __syncthreads();
    if (threadIdx.x == 0) {
        const double ny = G.ny, dT = 1.0;
        out[0] = res[DIAG_NPART + 0] / ny * lz / dT;
        out[1] = res[DIAG_NPART + 1] / ny * lz / dT;
        out[2] = res[DIAG_NPART + 2] / ny * lz / dT;
        out[3] = res[0];
        out[4] = res[1];
        out[5] = res[2];
        out[6] = res[3];
        out[7] = res[4];
        out[8] = res[DIAG_NPART + 3] / double(G.ny - 2);
        out[9] = 1.0 + res[6] / (double(G.nx - 2) * double(G.ny - 2)) * lz / dT;
        out[10] = res[5];
    }
}

// TimeAverager::accumulate (src/uniform/post.rs:37-49) on the device; sums
// are FP64 and dense (k = iy*nx + ix).
template <class A>
__global__ void k_avg_accumulate(const A* __restrict__ ux, const A* __restrict__ uy, const A* __restrict__ tt,
                                 const A* __restrict__ nut, double* __restrict__ sums, Geom G) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const long long k = (long long)iy * G.pitch + ix;
    const long long d = (long long)iy * G.nx + ix, n = (long long)G.nx * G.ny;
    const double u = ux[k], w = uy[k];
    sums[d] += u;
    sums[n + d] += w;
    sums[2 * n + d] += double(tt[k]);
    sums[3 * n + d] += double(nut[k]);
    sums[4 * n + d] += u * u + w * w;
}

}  // namespace cav
