// Random-information-set upper bound on the device: the GF(2) elimination half of the
// reference's random_is_seed (cpp/distfind/bz.cpp:70-116).  The host draws the column
// orders exactly as the reference does (std::mt19937 + std::shuffle per stream); here one
// warp takes one trial: the K x n code generator (K <= 128 rows, n <= 128 columns) sits in
// registers, row i on lane i%32 slot i/32, and is put in restricted row-echelon form over
// the trial's column order with the reference's pivot rule (first row at or below the rank
// with a 1 in the column, swapped into position `rank`, then cleared from every other
// row).  Per column: one ballot per 32-row slot in use, one pivot broadcast by shuffle, one
// masked XOR per slot in use.
// The lightest logical nonzero row of every trial is folded into the side's 32-bit key
// (weight:17 | trial:8 | row:7) with one atomicMin per warp.
#include <cuda_runtime.h>
#include <cstdint>

#include "seed_types.hpp"

namespace qsfb {
namespace dev {

template <int W>
__device__ __forceinline__ void get_slot(const unsigned long long (&r)[4][W], int s,
                                         unsigned long long (&out)[W]) {
#pragma unroll
    for (int w = 0; w < W; ++w)
        out[w] = s == 0 ? r[0][w] : s == 1 ? r[1][w] : s == 2 ? r[2][w] : r[3][w];
}

template <int W>
__device__ __forceinline__ void put_slot(unsigned long long (&r)[4][W], int s,
                                         const unsigned long long (&v)[W]) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (q == s) {
#pragma unroll
            for (int w = 0; w < W; ++w) r[q][w] = v[w];
        }
}

template <int W>
__global__ void __launch_bounds__(128) seed_trials_kernel(const SeedDesc* __restrict__ descs,
                                                          int ndesc, int total_trials) {
    const int lane = threadIdx.x & 31;
    const int gt = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (gt >= total_trials) return;
    int lo = 0, hi = ndesc - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (descs[mid].trial_base <= gt) lo = mid; else hi = mid - 1;
    }
    const SeedDesc& D = descs[lo];
    const int t = gt - D.trial_base;
    const int K = D.K, n = D.n;
    const int S = (K + 31) >> 5;   // row slots in use (warp-uniform): the rest stay zero

    unsigned long long r[4][W];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int row = 32 * s + lane;
#pragma unroll
        for (int w = 0; w < W; ++w) r[s][w] = row < K ? __ldg(D.gen + (size_t)row * W + w) : 0ull;
    }
    const uint8_t* perm = D.perm + (size_t)t * n;
    int rank = 0;
    for (int ci = 0; ci < n && rank < K; ++ci) {
        const int col = __ldg(perm + ci);
        const int wd = col >> 6;
        const unsigned long long bit = 1ull << (col & 63);
        unsigned b[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            b[s] = 0u;
            if (s < S) {
                unsigned long long v = 0;
#pragma unroll
                for (int w = 0; w < W; ++w) if (w == wd) v = r[s][w];
                b[s] = __ballot_sync(0xffffffffu, (v & bit) != 0ull);
            }
        }
        int sel = -1;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            unsigned m = b[s];
            const int first = 32 * s;
            if (rank >= first + 32) m = 0u;
            else if (rank > first) m &= ~((1u << (rank - first)) - 1u);
            if (sel < 0 && m) sel = first + __ffs(m) - 1;
        }
        if (sel < 0) continue;
        const int ps = sel >> 5, pl = sel & 31, rs = rank >> 5, rl = rank & 31;
        unsigned long long pv[W], ov[W], tmp[W];
        get_slot<W>(r, ps, tmp);
#pragma unroll
        for (int w = 0; w < W; ++w) pv[w] = __shfl_sync(0xffffffffu, tmp[w], pl);
        get_slot<W>(r, rs, tmp);
#pragma unroll
        for (int w = 0; w < W; ++w) ov[w] = __shfl_sync(0xffffffffu, tmp[w], rl);
        if (lane == pl) put_slot<W>(r, ps, ov);   // old row `rank` moves to `sel`
        if (lane == rl) put_slot<W>(r, rs, pv);   // pivot row moves to `rank`
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (s >= S) continue;
            const int row = 32 * s + lane;
            unsigned long long v = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) if (w == wd) v = r[s][w];
            if (row != rank && (v & bit)) {
#pragma unroll
                for (int w = 0; w < W; ++w) r[s][w] ^= pv[w];
            }
        }
        ++rank;
    }

    // lightest logical nonzero row of this trial
    unsigned key = 0xffffffffu;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int row = 32 * s + lane;
        if (row >= K) continue;
        int wt = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) wt += __popcll(r[s][w]);
        if (wt == 0 || wt >= D.init_best) continue;
        bool logical = D.count_all != 0;
        for (int c = 0; c < D.kcheck && !logical; ++c) {
            unsigned long long acc = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) acc ^= __ldg(D.check + (size_t)c * W + w) & r[s][w];
            logical = (__popcll(acc) & 1) != 0;
        }
        if (!logical) continue;
        const unsigned k = ((unsigned)wt << 15) | ((unsigned)t << 7) | (unsigned)row;
        key = k < key ? k : key;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned o = __shfl_xor_sync(0xffffffffu, key, off);
        key = o < key ? o : key;
    }
    if (lane == 0 && key != 0xffffffffu) atomicMin(D.key, key);
}

}  // namespace dev

cudaError_t launch_seed_trials(int W, const SeedDesc* d_descs, int ndesc, int total_trials,
                               cudaStream_t st) {
    if (total_trials <= 0) return cudaSuccess;
    const int warps_per_block = 4;
    const int blocks = (total_trials + warps_per_block - 1) / warps_per_block;
    if (W == 1) dev::seed_trials_kernel<1><<<blocks, 128, 0, st>>>(d_descs, ndesc, total_trials);
    else if (W == 2) dev::seed_trials_kernel<2><<<blocks, 128, 0, st>>>(d_descs, ndesc, total_trials);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace qsfb
