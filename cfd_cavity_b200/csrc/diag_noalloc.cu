// diag_noalloc.cu -- cav_diag_noalloc: the cavity diagnostics over
// caller-owned device arrays, with no device allocation at all.
//
// Who needs it.  cav_diag works on a cav_handle, whose reduction scratch the
// library cudaMalloc's when the handle is created.  Some callers cannot let
// a library allocate on their behalf: a host framework whose caching
// allocator has already reserved the device memory it is allowed to use, so
// that a foreign cudaMalloc fails or pushes it out of its budget; or a
// time-stepping loop that must not stall, where cudaMalloc / cudaFree may
// synchronise the whole device.  Such callers keep the state in their own
// device buffers and call this entry point instead.
//
// Scratch.  The per-row partial sums live in g_row_scratch below, a
// file-scope device array of CAV_NOALLOC_MAX_ROWS x 8 doubles (512 KiB) that
// every GPU loading this library holds until the process exits.  In host
// code the name g_row_scratch is only a host-side stand-in for the symbol,
// not a device address: every call, with the caller's device current, asks
// the runtime for the real address (cudaGetSymbolAddress, cheap once the
// module is loaded) and passes it to the kernels.  Nothing is cached, so a
// cudaDeviceReset or another context between calls cannot leave a stale
// address behind.  The first call on a device may load the library's device
// code there, so it should come before any stream capture on that device.
// Every row's partials are rewritten by each call before they are read, so
// nothing has to be cleared between calls; but the array keeps the last
// call's contents and is shared by all calls on a device, so two calls whose
// kernels overlap on the GPU (different streams, no ordering between them)
// race on it and must be serialised by the caller.
//
// Errors.  A CUDA error already pending when the call starts (left by the
// caller's own work) is reported as CAV_ERR_CUDA without launching anything
// and is not cleared: the caller still finds it with cudaGetLastError.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../include/cavity.h"
#include "diag.cuh"

namespace {

constexpr int NPART = 8;  // per row: sum rho, sum f, max u, max uy, max nu_t, non-finite, sum vol, spare

static __device__ __align__(256) double g_row_scratch[CAV_NOALLOC_MAX_ROWS * NPART];

// Pass 1: one block per row of a dense FP64 state, row-partials into scratch.
__global__ void __launch_bounds__(cav::DIAG_THREADS)
k_rows(const double* __restrict__ rho, const double* __restrict__ ux, const double* __restrict__ uy,
       const double* __restrict__ tt, const double* __restrict__ nut, const double* __restrict__ f, int nx,
       int ny, double* __restrict__ scratch) {
    const int iy = blockIdx.x;
    double v[NPART] = {0, 0, 0, 0, 0, 0, 0, 0};
    const bool is_max[NPART] = {false, false, true, true, true, false, false, false};
    for (int ix = threadIdx.x; ix < nx; ix += blockDim.x) {
        const long long k = (long long)iy * nx + ix;
        const double r = rho[k], u = ux[k], w = uy[k], t = tt[k];
        double sf = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) sf += f[k * 9 + i];
        v[0] += r;
        v[1] += sf;
        v[2] = fmax(v[2], fmax(fabs(u), fabs(w)));
        v[3] = fmax(v[3], fabs(w));
        v[4] = fmax(v[4], fabs(nut[k]));
        const bool fin = isfinite(t) && isfinite(u) && isfinite(w) && isfinite(r) && r > 0.0;
        v[5] += fin ? 0.0 : 1.0;
        if (ix >= 1 && ix <= nx - 2 && iy >= 1 && iy <= ny - 2) v[6] += w * t;
    }
    cav::block_reduce<NPART>(v, is_max, scratch + (long long)iy * NPART);
}

// Pass 2 (one block): rows in a fixed order plus the per-row Nusselt / y+
// terms (post.rs:68-199); out[] follows the field order of cav_diag_out.
__global__ void __launch_bounds__(cav::DIAG_THREADS)
k_final(const double* __restrict__ scratch, const double* __restrict__ uy, const double* __restrict__ tt,
        const double* __restrict__ nut, int nx, int ny, double nu_mol, double lz, double* __restrict__ out) {
    constexpr int NV = NPART + 4;
    double v[NV];
    bool is_max[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        v[j] = 0.0;
        is_max[j] = (j == 2 || j == 3 || j == 4);
    }
    for (int iy = threadIdx.x; iy < ny; iy += blockDim.x) {
#pragma unroll
        for (int j = 0; j < NPART; ++j) {
            const double p = scratch[(long long)iy * NPART + j];
            v[j] = is_max[j] ? fmax(v[j], p) : v[j] + p;
        }
        const long long r = (long long)iy * nx;
        v[NPART + 0] += fabs(tt[r + 1] - tt[r + 2]);
        v[NPART + 1] += fabs(tt[r + nx - 2] - tt[r + nx - 3]);
        v[NPART + 2] += fabs(tt[r + 0] - tt[r + 1]);
        if (iy >= 1 && iy <= ny - 2) {
            const double tau_w = (nu_mol + nut[r + 1]) * fabs(uy[r + 1] - uy[r + 0]);
            v[NPART + 3] += 0.5 * sqrt(fmax(tau_w, 0.0)) / nu_mol;
        }
    }
    __shared__ double res[NV];
    cav::block_reduce<NV>(v, is_max, res);
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = res[NPART + 0] / double(ny) * lz;
        out[1] = res[NPART + 1] / double(ny) * lz;
        out[2] = res[NPART + 2] / double(ny) * lz;
        out[3] = res[0];
        out[4] = res[1];
        out[5] = res[2];
        out[6] = res[3];
        out[7] = res[4];
        out[8] = res[NPART + 3] / double(ny - 2);
        out[9] = 1.0 + res[6] / (double(nx - 2) * double(ny - 2)) * lz;
        out[10] = res[5] == 0.0 ? 1.0 : 0.0;
    }
}

// Rejections are reported by status code and one line on stderr (this entry
// point has no handle to hold a message).
int err(int code, const char* msg) {
    fprintf(stderr, "cav_diag_noalloc: %s\n", msg);
    return code;
}

}  // namespace

extern "C" {

int cav_diag_noalloc(const double* rho, const double* ux, const double* uy, const double* t, const double* nu_t,
                     const double* f, int32_t nx, int32_t ny, double nu, double lz, double* out, void* stream) {
    if (!rho || !ux || !uy || !t || !nu_t || !f || !out) return err(CAV_ERR_ARG, "null device pointer");
    if (nx < 4 || ny < 4) return err(CAV_ERR_ARG, "nx and ny must be at least 4");
    if (ny > CAV_NOALLOC_MAX_ROWS) {
        char buf[160];
        snprintf(buf, sizeof buf, "ny = %d exceeds CAV_NOALLOC_MAX_ROWS = %d (rows of the static scratch)", ny,
                 CAV_NOALLOC_MAX_ROWS);
        return err(CAV_ERR_ARG, buf);
    }
    if (!(nu > 0.0)) return err(CAV_ERR_ARG, "nu must be positive");
    // an error the caller left pending is reported, not consumed
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) return err(CAV_ERR_CUDA, cudaGetErrorString(pending));
    // the device address of the static scratch on the current device
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_row_scratch);
    if (e != cudaSuccess || !p) {
        if (e != cudaSuccess) cudaGetLastError();  // this call's own failure
        return err(CAV_ERR_CUDA, e != cudaSuccess ? cudaGetErrorString(e) : "null scratch address");
    }
    double* scratch = static_cast<double*>(p);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_rows<<<ny, cav::DIAG_THREADS, 0, s>>>(rho, ux, uy, t, nu_t, f, nx, ny, scratch);
    e = cudaGetLastError();  // nothing was pending, so a failure here is this launch's
    if (e != cudaSuccess) return err(CAV_ERR_CUDA, cudaGetErrorString(e));
    k_final<<<1, cav::DIAG_THREADS, 0, s>>>(scratch, uy, t, nu_t, nx, ny, nu, lz, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return err(CAV_ERR_CUDA, cudaGetErrorString(e));
    return CAV_OK;
}

}  // extern "C"
