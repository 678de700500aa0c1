// The hardware stochastic rounding of binary16 and bfloat16 pairs
// (h16x2_enc_sr, bf16x2_enc_sr: cvt.rs) against the software h16_enc /
// bf16_store on 2^21 deterministic pseudo-random values (magnitudes
// 2^-20 .. 2^16, both signs): prints the binary16 differences in the normal
// and in the subnormal range, and the bfloat16 differences.  Built and run by
// tests/test_gpu_sr.py.
#include <cstdio>
#include "lattice.cuh"
using namespace cav;
constexpr int N = 1 << 20;
__global__ void k(unsigned* mism, unsigned* sub, unsigned* bmism) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint32_t s = mix32(uint32_t(i) * 2654435761u + 12345u);
    uint32_t s2 = mix32(s ^ 0x9e3779b9u);
    // magnitudes 2^-20 .. 2^15 (scaled lane values), both signs
    const float a = ldexpf(1.0f + float(s & 0xffffff) / 16777216.0f, int((s >> 24) % 36) - 20) * ((s2 & 1) ? -1.f : 1.f);
    const float b = ldexpf(1.0f + float(s2 >> 8) / 16777216.0f, int(s2 % 36) - 20) * ((s & 1) ? -1.f : 1.f);
    const uint32_t r = mix32(s ^ s2);
    const uint32_t d = h16x2_enc_sr(a, b, r);
    const unsigned short ha = h16_enc(a, true, r & 0xffff0000u), hb = h16_enc(b, true, r << 16);
    const bool sa = fabsf(a) < 6.103515625e-05f, sb = fabsf(b) < 6.103515625e-05f;  // binary16 subnormal range
    if ((d >> 16) != ha) atomicAdd(sa ? sub : mism, 1u);
    if ((d & 0xffffu) != hb) atomicAdd(sb ? sub : mism, 1u);
    const uint32_t db = bf16x2_enc_sr(a, b, r);
    if ((db >> 16) != bf16_store(a, true, r & 0xffff0000u)) atomicAdd(bmism, 1u);
    if ((db & 0xffffu) != bf16_store(b, true, r << 16)) atomicAdd(bmism, 1u);
}
int main() {
    unsigned *m, *s, *bm, hm = 0, hs = 0, hb = 0;
    cudaMalloc(&m, 4); cudaMalloc(&s, 4); cudaMalloc(&bm, 4);
    cudaMemset(m, 0, 4); cudaMemset(s, 0, 4); cudaMemset(bm, 0, 4);
    k<<<N / 256, 256>>>(m, s, bm);
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(&hm, m, 4, cudaMemcpyDeviceToHost); cudaMemcpy(&hs, s, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(&hb, bm, 4, cudaMemcpyDeviceToHost);
    printf("err %d  mismatches (normal range) %u  (subnormal range) %u  of %d  bf16 %u\n", int(e), hm, hs, 2 * N,
           hb);
    return e == cudaSuccess ? 0 : 1;
}
