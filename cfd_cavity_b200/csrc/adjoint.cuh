// adjoint.cuh -- discrete adjoint of the cavity step: gradients of a
// time-averaged hot-wall Nusselt number with respect to the hot-wall
// temperature profile and the Smagorinsky constant.
//
// State X_s = post-collision populations + Guo force (the PC form) of step
// s-1; kernel s maps X_s -> X_{s+1} by pull (+ bounce-back, thermal BCs),
// macroscopic update and collision.  The adjoint of one step, for node x:
//   1. the adjoint of X_{s+1}(x) (the node's own outputs) is gathered from
//      the adjoints of the pulled inputs of the nodes that read them: the
//      transpose of the pull, again a gather because streaming is a
//      bijection (f) or reads every g source from at most three nodes
//      (the row-1 / row-(ny-2) values are copied to the adjacent wall rows);
//   2. the node's pulled inputs are recomputed from the stored X_s and
//      node_reverse() (node_ad.h) gives their adjoints, the adjoint of the
//      previous Guo force and dJ/dCs;
//   3. the hot-wall nodes' pulled g are geq(theta_w, 0, 0) = w_i theta_w:
//      their adjoints give dJ/dtheta_w.
// Objective J = mean over s in [ws, N] of nusselt_hot of the state after s
// steps (src/uniform/post.rs:68-78).  Accumulators are per node (Cs) and per
// row (theta), each written by one thread, so the gradient is deterministic.
#pragma once

#include "kernels.cuh"
#include "node_ad.h"

namespace cav {

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// P-buffer: adjoints of the pulled inputs of every node, 19 planes of type A
// in the population geometry: f 0..8, g 9..17, previous Guo force 18.
constexpr int APLANES = 19;

template <class A>
struct AdjObj {
    long long ws;  // first state of the averaging window
    A coef;        // lz / (ny * window length)
};

template <class A>
__device__ __forceinline__ ad::NodeScal<A> node_scal(const StepScalars<A>& c) {
    ad::NodeScal<A> s;
    s.beta = c.beta;
    s.nu = c.nu;
    s.alpha = c.alpha;
    s.c1 = A(1.5) * c.inv_tau_s;
    s.inv_pr_t = c.inv_pr_t;
    s.lambda = A(LAMBDA_TRT);
    s.q2 = c.geq_order == 1 ? A(0.0) : A(1.0);
    return s;
}

// dJ/dT at (ix, iy) of the state read by this kernel (columns 1 and 2 only).
template <class St>
__device__ __forceinline__ typename Fmt<St>::A nu_obj_adjoint(const St* __restrict__ X, const Geom& G, int ix,
                                                              int iy, typename Fmt<St>::A t_own,
                                                              const StepScalars<typename Fmt<St>::A>& c,
                                                              typename Fmt<St>::A coef) {
    using A = typename Fmt<St>::A;
    if (ix != 1 && ix != 2) return A(0.0);
    const A t_other = gather_t<St>(X, G, ix == 1 ? 2 : 1, iy, c);
    const A diff = ix == 1 ? t_own - t_other : t_other - t_own;  // T(1) - T(2)
    const A sgn = diff > A(0.0) ? A(1.0) : (diff < A(0.0) ? A(-1.0) : A(0.0));
    return ix == 1 ? coef * sgn : -coef * sgn;
}

// Adjoint of the final state's objective term (no collision follows).
template <class St>
__global__ void k_adj_final(const St* __restrict__ X, typename Fmt<St>::A* __restrict__ P, Geom G,
                            StepScalars<typename Fmt<St>::A> c, AdjObj<typename Fmt<St>::A> obj,
                            long long s) {
    using A = typename Fmt<St>::A;
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const int k = iy * G.pitch + ix;
    const int Pp = int(G.plane);
    A at = A(0.0);
    if (s >= obj.ws && (ix == 1 || ix == 2)) at = nu_obj_adjoint<St>(X, G, ix, iy, gather_t<St>(X, G, ix, iy, c), c, obj.coef);
#pragma unroll
    for (int q = 0; q < Q; ++q) P[q * Pp + k] = A(0.0);
#pragma unroll
    for (int q = 0; q < Q; ++q) P[(Q + q) * Pp + k] = at;
    P[18 * Pp + k] = A(0.0);
}

// One adjoint step s (X = stored X_s, Pin = P of step s+1, Pout = P of step s).
// Step scalars of step s from the per-step table (rows 0..S, row S = steady
// state); s = *step_dev + j in graph replays, s = j otherwise.
template <class A>
__device__ __forceinline__ StepScalars<A> table_scalars(const StepScalars<A>* __restrict__ table, int S,
                                                        const long long* step_dev, long long j, long long* s_out) {
    const long long s = (step_dev ? *step_dev : 0) + j;
    *s_out = s;
    StepScalars<A> c = table[s < S ? s : S];
    c.step = s;
    c.step_dev = nullptr;
    return c;
}

template <class St>
__global__ void __launch_bounds__(128) k_adj_step(const St* __restrict__ X, const typename Fmt<St>::A* __restrict__ Xfy,
                                                  const typename Fmt<St>::A* __restrict__ Pin,
                                                  typename Fmt<St>::A* __restrict__ Pout, double* __restrict__ acc_cs,
                                                  double* __restrict__ acc_theta, Geom G,
                                                  const StepScalars<typename Fmt<St>::A>* __restrict__ table, int S,
                                                  const long long* step_dev, long long j,
                                                  AdjObj<typename Fmt<St>::A> obj, const St* __restrict__ Xpre,
                                                  const typename Fmt<St>::A* __restrict__ Xfy_pre) {
    using A = typename Fmt<St>::A;
    pdl_wait();
    pdl_trigger();
    long long s;
    const StepScalars<A> c = table_scalars<A>(table, S, step_dev, j, &s);
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    const int W = G.pitch, Pp = int(G.plane);
    const int k = iy * W + ix;
    const int nx = G.nx, ny = G.ny;
    // The next kernel of the sweep reads the previous state of the segment
    // (recomputed earlier, usually evicted to HBM): bring this node's part
    // of it into L2 now, so that its loads are L2 hits.
    if (Xpre) {
#pragma unroll
        for (int q = 0; q < NPLANES; ++q) prefetch_l2(Xpre + (q * Pp + k));
        prefetch_l2(Xfy_pre + k);
    }
    // 1. adjoint of this node's outputs X_{s+1}(x), gathered from its readers.
    // Branch-free: every load reads a valid address and the unused ones are
    // discarded by selects, so all of a node's loads are in flight together.
    // Rows 1 / ny-2 were copied to the wall rows 0 / ny-1, so their readers'
    // adjoints add up; only rows within two of a wall read those (a row of a
    // block is one warp, so the branch is uniform).
    const bool near_wall = iy <= 2 || iy >= ny - 3;
    A af[Q], ag[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int rx = ix + CX(q), ry = iy + CY(q);
        const bool in = rx >= 0 && rx < nx && ry >= 0 && ry < ny;
        const int kr = in ? ry * W + rx : k;
        af[q] = Pin[(in ? q : OPP(q)) * Pp + kr];
        const bool gin = in && rx >= 1 && rx <= nx - 2 && ry >= 1 && ry <= ny - 2;
        ag[q] = gin ? Pin[(Q + q) * Pp + kr] : A(0.0);
    }
    if (near_wall) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int rx = ix + CX(q), ry = iy + CY(q);
            const bool gin = rx >= 1 && rx <= nx - 2 && ry >= 1 && ry <= ny - 2;
            if (gin && (ry == 1 || ry == ny - 2)) {
                const int kw = ry == 1 ? rx : (ny - 1) * W + rx;
                ag[q] = ag[q] + Pin[(Q + q) * Pp + kw];
            }
        }
    }
    const A afy = Pin[18 * Pp + k];
    // 2. recompute the node's pulled inputs from X_s.
    A f[Q], g[Q];
    pull_node<St>(X, G, ix, iy, c, f, g);
    A h[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) h[i] = Fmt<St>::SHIFT ? f[i] : f[i] - A(WD(i));
    const A fyp = Xfy[k];
    const bool wall = is_wall(G, ix, iy);
    A at = A(0.0);
    if (s >= obj.ws && (ix == 1 || ix == 2)) {
        A t = g[0];
#pragma unroll
        for (int j = 1; j < Q; ++j) t = t + g[j];
        at = nu_obj_adjoint<St>(X, G, ix, iy, t, c, obj.coef);
    }
    A ah[Q], agi[Q], afyp;
    const A bcs = ad::node_reverse<A>(h, g, fyp, wall, c.cs, node_scal<A>(c), af, ag, afy, at, ah, agi, &afyp);
    acc_cs[iy * nx + ix] += double(bcs);
    // 3. outputs: adjoints of the pulled inputs; hot-wall theta gradient.
    const bool wall_col = ix == 0 || ix == nx - 1;
#pragma unroll
    for (int q = 0; q < Q; ++q) Pout[q * Pp + k] = ah[q];
#pragma unroll
    for (int q = 0; q < Q; ++q) Pout[(Q + q) * Pp + k] = wall_col ? A(0.0) : agi[q];
    Pout[18 * Pp + k] = afyp;
    if (ix == 0) {
        // g_i = w_i theta (quadratic and linear geq agree at u = 0)
        double sw = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) sw += WD(q) * double(agi[q]);
        acc_theta[iy] += sw;
    }
}

// Forward step into a separate state (pops + Guo force): the recomputation
// of a checkpoint segment.  Same node body as k_fused.
template <class St>
__global__ void __launch_bounds__(256) k_fwd_slot(const St* __restrict__ src, St* __restrict__ dst,
                                                  const typename Fmt<St>::A* fy_in, typename Fmt<St>::A* fy_out,
                                                  Geom G, const StepScalars<typename Fmt<St>::A>* __restrict__ table,
                                                  int S, const long long* step_dev, long long j) {
    using A = typename Fmt<St>::A;
    pdl_wait();
    pdl_trigger();
    long long s;
    const StepScalars<A> c = table_scalars<A>(table, S, step_dev, j, &s);
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    if (ix >= G.nx || iy >= G.ny) return;
    fused_node_io<St, false, false, false>(src, dst, fy_in, fy_out, nullptr, nullptr, nullptr, G, ix, iy, c);
}

}  // namespace cav
