// Random-information-set upper bound on the device: the GF(2) elimination half of the
// reference's random_is_seed (cpp/distfind/bz.cpp:24-70, the trial loop at :36-51).  The
// host draws the column orders exactly as the reference does (std::mt19937 + std::shuffle
// per stream); here one warp takes one trial: the K x n code generator (K <= 128 rows,
// n <= 256 columns, W = ceil(n/64) words per row) sits in registers, row i on lane i%32 slot i/32, and is put in
// reduced row-echelon form over the trial's column order.  The reference's pivot rule takes
// the first row at or below the rank with a 1 in the column, swaps it into position `rank`
// and clears the column from every other row.  The rows that result do not depend on which
// candidate row is taken (the reduced row of each pivot column is unique), and row `rank`
// of the reference's matrix is the one reduced on the rank-th pivot column.  So no row
// moves here: the pivot is the first row not yet used as a pivot that has a 1 in the
// column, and each row remembers the rank at which it became a pivot, its position in the
// reference's matrix.  A row that is no pivot when the trial ends is zero in every column
// (the code generator's rows are independent, so normally none is left).  The number of slots
// in use, S = ceil(K/32), is a compile-time constant of the trial's body (one body per S,
// chosen per trial).  Per column: the column index from a register by shuffle, one ballot
// per slot, one pivot broadcast by shuffle, one masked XOR per slot.
// The lightest logical nonzero row of every trial is folded into the side's 32-bit key
// (weight:17 | trial:8 | row:7) with one atomicMin per warp.
#include <cuda_runtime.h>
#include <cstdint>

#include "seed_types.hpp"

namespace qsfb {
namespace dev {

// One column of the elimination, with the column's word WD fixed at compile time: the
// column is the same for the whole warp, so the caller branches on its word once instead
// of every row selecting it.  Returns false when no row is left to pivot on.
template <int W, int S, int WD>
__device__ __forceinline__ bool eliminate_column(unsigned long long (&r)[S][W],
                                                 unsigned long long bit, uint32_t& piv,
                                                 uint32_t& pos, int rank, int lane) {
    // the first row, in row order, that is no pivot row yet and has a 1 in the column (the
    // rows' bits in the column are read once, for this search and for the clearing below)
    bool hit[S];
    unsigned m[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        hit[s] = (r[s][WD] & bit) != 0ull;
        m[s] = __ballot_sync(0xffffffffu, hit[s] && ((piv >> s) & 1u) == 0u);
    }
    int sel = -1;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (m[s]) {   // the same on every lane
            sel = 32 * s + __ffs(m[s]) - 1;
            break;
        }
    if (sel < 0) return false;
    const int ps = sel >> 5, pl = sel & 31;   // the same on every lane
    unsigned long long pv[W];
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (s == ps) {
#pragma unroll
            for (int w = 0; w < W; ++w) pv[w] = __shfl_sync(0xffffffffu, r[s][w], pl);
        }
    if (lane == pl) {
        piv |= 1u << ps;
        pos |= (uint32_t)rank << (8 * ps);
    }
    // clear the column from every other row
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (hit[s] && !(s == ps && lane == pl)) {
#pragma unroll
            for (int w = 0; w < W; ++w) r[s][w] ^= pv[w];
        }
    return true;
}

// One trial with the K rows in S slots of 32 (K <= 32 S): S and W fixed at compile time,
// so every per-column step touches only the slots in use.
template <int W, int S>
__device__ __forceinline__ void run_trial(const SeedDesc& D, int t, int lane) {
    const int K = D.K, n = D.n;
    unsigned long long r[S][W];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int row = 32 * s + lane;
#pragma unroll
        for (int w = 0; w < W; ++w) r[s][w] = row < K ? __ldg(D.gen + (size_t)row * W + w) : 0ull;
    }
    // the trial's column order: bytes PB lane .. PB lane + PB - 1 on this lane (PB = 4 for
    // n <= 128, 8 for n <= 256)
    constexpr int PB = W <= 2 ? 4 : 8;
    const uint8_t* perm = D.perm + (size_t)t * n;
    uint32_t pw[PB / 4];
#pragma unroll
    for (int j = 0; j < PB / 4; ++j) pw[j] = 0u;
#pragma unroll
    for (int j = 0; j < PB; ++j) {
        const int c = PB * lane + j;
        if (c < n) pw[j >> 2] |= (uint32_t)__ldg(perm + c) << (8 * (j & 3));
    }
    int rank = 0;
    uint32_t piv = 0u;   // bit s: row 32 s + lane is a pivot row
    uint32_t pos = 0u;   // byte s: the rank at which it became one
    for (int ci = 0; ci < n && rank < K; ++ci) {
        const uint32_t src = PB == 4 ? pw[0] : pw[(ci >> 2) & (PB / 4 - 1)];   // uniform
        const int col =
            (int)((__shfl_sync(0xffffffffu, src, ci / PB) >> (8 * (ci & 3))) & 0xffu);
        const unsigned long long bit = 1ull << (col & 63);
        const int wd = W == 1 ? 0 : col >> 6;   // the column's word, uniform over the warp
        bool took;
        if (W == 1 || wd == 0)
            took = eliminate_column<W, S, 0>(r, bit, piv, pos, rank, lane);
        else if (W == 2 || wd == 1)
            took = eliminate_column<W, S, (W > 1 ? 1 : 0)>(r, bit, piv, pos, rank, lane);
        else if (W == 3 || wd == 2)
            took = eliminate_column<W, S, (W > 2 ? 2 : 0)>(r, bit, piv, pos, rank, lane);
        else
            took = eliminate_column<W, S, (W > 3 ? 3 : 0)>(r, bit, piv, pos, rank, lane);
        rank += took ? 1 : 0;
    }

    // lightest logical nonzero row of this trial
    unsigned key = 0xffffffffu;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        if (!((piv >> s) & 1u)) continue;   // not a pivot row: zero
        const int row = (int)((pos >> (8 * s)) & 0xffu);   // its row in the reference's matrix
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

template <int W>
__global__ void __launch_bounds__(64, 16) seed_trials_kernel(const SeedDesc* __restrict__ descs,
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
    switch ((D.K + 31) >> 5) {   // row slots in use, uniform over the warp
        case 0: return;
        case 1: run_trial<W, 1>(D, t, lane); break;
        case 2: run_trial<W, 2>(D, t, lane); break;
        case 3: run_trial<W, 3>(D, t, lane); break;
        default: run_trial<W, 4>(D, t, lane); break;
    }
}

}  // namespace dev

cudaError_t launch_seed_trials(int W, const SeedDesc* d_descs, int ndesc, int total_trials,
                               cudaStream_t st) {
    if (total_trials <= 0) return cudaSuccess;
    // Blocks of two warps (64 threads x at most 64 registers, the kernel's launch bound):
    // they fit in the 4,096 registers a running tensor-core sweep CTA (640 threads x 96)
    // leaves free on its SM, so a preparation that overlaps the rounds starts at once
    // instead of queueing behind the sweep's launch.
    const int warps_per_block = 2;
    const int blocks = (total_trials + warps_per_block - 1) / warps_per_block;
    if (W == 1) dev::seed_trials_kernel<1><<<blocks, 64, 0, st>>>(d_descs, ndesc, total_trials);
    else if (W == 2) dev::seed_trials_kernel<2><<<blocks, 64, 0, st>>>(d_descs, ndesc, total_trials);
    else if (W == 3) dev::seed_trials_kernel<3><<<blocks, 64, 0, st>>>(d_descs, ndesc, total_trials);
    else if (W == 4) dev::seed_trials_kernel<4><<<blocks, 64, 0, st>>>(d_descs, ndesc, total_trials);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace qsfb
