// Integer-pipe peak measurement for the roofline denominators: a full-device grid of
// independent 32-bit POPC chains (the XU pipe the pair kernel's popcount mode saturates)
// and of LOP3 chains (the ALU pipe of its zero-test mode).  Eight independent chains per
// thread hide the pipe latency; the result is written so nothing is optimised away.
#include <cuda_runtime.h>
#include <cstdint>

namespace qsfb {
namespace dev {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) popc_peak_kernel(uint32_t seed, int iters, uint32_t* out) {
    uint32_t v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = seed ^ (threadIdx.x * 0x9e3779b9u + c * 0x85ebca6bu);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) v[c] = __popc(v[c]) ^ v[c];   // 1 POPC + 1 LOP per step
    }
    uint32_t acc = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc += v[c];
    if (acc == 0x12345678u) out[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(256) lop3_peak_kernel(uint32_t seed, int iters, uint32_t* out) {
    uint32_t a[kChains], b = seed * 0x27d4eb2fu, c = seed ^ 0x165667b1u;
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = seed ^ (threadIdx.x * 0x9e3779b9u + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = (a[k] ^ b) | (a[k] & c);   // one LOP3
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) acc += a[k];
    if (acc == 0x12345678u) out[blockIdx.x] = acc;
}

}  // namespace dev

// ops/s of the chosen pipe (which = 0: POPC, 1: LOP3), timed with CUDA events after one
// warm-up launch; `out` must hold gridDim u32 (never written in practice).
cudaError_t microbench_peak(int which, int num_sms, uint32_t* d_out, cudaStream_t st,
                            double* ops_per_s) {
    const int blocks = num_sms * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int rep = 0; rep < 2; ++rep) {
        cudaEventRecord(e0, st);
        if (which == 0) dev::popc_peak_kernel<<<blocks, threads, 0, st>>>(rep + 1, iters, d_out);
        else dev::lop3_peak_kernel<<<blocks, threads, 0, st>>>(rep + 1, iters, d_out);
        cudaEventRecord(e1, st);
    }
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return err;
    const double ops = (double)blocks * threads * iters * dev::kChains;
    *ops_per_s = ops / (ms * 1e-3);
    return cudaGetLastError();
}

}  // namespace qsfb
