// Information sets on the device: the GF(2) eliminations that give every side its
// information-set generator matrices (reference cpp/distfind/css.cpp:177-203 greedy peel,
// :355-364 one restricted_rref per matroid-partition class; the elimination itself is
// cpp/qsf/gf2.cpp:42-58), fused with the two derived tables the pair sweeps read.
//
// One warp per side.  The K x n code generator (K <= 128, n <= 128) sits in registers, row
// i on lane i%32 slot i/32 (S = ceil(K/32) slots, a compile-time constant per side).  A
// column step is the reference's pivot rule: one ballot per slot finds the first row at or
// below the rank with a 1 in the column, two shuffles move that row to position `rank`, and
// one masked XOR per slot clears the column from every other row.
//   greedy (lists == nullptr): restricted RREF over the active columns in ascending order,
//     on the working matrix left by the previous set; the next active set drops this set's
//     pivots and the columns that are zero in every row; stop when nothing was dropped or
//     nothing is left.  Ranks come out non-increasing, so this is also the rank-sorted order.
//   explicit lists: each set is a restricted RREF of a fresh copy of the generator over its
//     column list, in list order (the matroid partition's classes, chosen on the host).
// After each set's elimination the warp writes
//   * the set's generator rows into a heap shared by all sides (one atomic bump per set),
//   * red[g][r]: row r restricted to the set's non-pivot columns (ascending), 32-bit words,
//   * syn[g][r]: bit c = parity(check_c & row r), the per-row detector syndrome,
// and its rank, heap offset and pivot mask into the side's meta block.
#include <cuda_runtime.h>
#include <cstdint>

#include "infoset_types.hpp"

namespace qsfb {
namespace dev {

template <int W, int S>
struct Rows {
    unsigned long long r[S][W];

    __device__ __forceinline__ void load(const unsigned long long* __restrict__ gen, int K, int lane) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int row = 32 * s + lane;
#pragma unroll
            for (int w = 0; w < W; ++w) r[s][w] = row < K ? __ldg(gen + (size_t)row * W + w) : 0ull;
        }
    }
    __device__ __forceinline__ unsigned long long word(int s, int wd) const {
        unsigned long long v = r[s][0];
#pragma unroll
        for (int w = 1; w < W; ++w) if (w == wd) v = r[s][w];
        return v;
    }
    __device__ __forceinline__ void get(int s, unsigned long long (&out)[W]) const {
#pragma unroll
        for (int w = 0; w < W; ++w) {
            out[w] = r[0][w];
#pragma unroll
            for (int q = 1; q < S; ++q) if (q == s) out[w] = r[q][w];
        }
    }
    __device__ __forceinline__ void put(int s, const unsigned long long (&v)[W]) {
#pragma unroll
        for (int q = 0; q < S; ++q)
            if (q == s) {
#pragma unroll
                for (int w = 0; w < W; ++w) r[q][w] = v[w];
            }
    }

    // One column of the restricted RREF: returns true when the column took a pivot.
    __device__ __forceinline__ bool step(int col, int rank, int lane) {
        const int wd = col >> 6;
        const unsigned long long bit = 1ull << (col & 63);
        int sel = -1;
#pragma unroll
        for (int s = S - 1; s >= 0; --s) {
            unsigned m = __ballot_sync(0xffffffffu, (word(s, wd) & bit) != 0ull);
            const int first = 32 * s;
            if (rank >= first + 32) m = 0u;
            else if (rank > first) m &= ~0u << (rank - first);
            if (m) sel = first + __ffs(m) - 1;
        }
        if (sel < 0) return false;
        const int ps = sel >> 5, pl = sel & 31, rs = rank >> 5, rl = rank & 31;
        unsigned long long pv[W], ov[W], tmp[W];
        get(ps, tmp);
#pragma unroll
        for (int w = 0; w < W; ++w) pv[w] = __shfl_sync(0xffffffffu, tmp[w], pl);
        get(rs, tmp);
#pragma unroll
        for (int w = 0; w < W; ++w) ov[w] = __shfl_sync(0xffffffffu, tmp[w], rl);
        if (lane == pl) put(ps, ov);   // the old row `rank` moves to `sel`
        if (lane == rl) put(rs, pv);   // the pivot row moves to `rank`
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int row = 32 * s + lane;
            if (row != rank && (word(s, wd) & bit)) {
#pragma unroll
                for (int w = 0; w < W; ++w) r[s][w] ^= pv[w];
            }
        }
        return true;
    }
};

// Outputs of set g: generator rows (heap), non-pivot rows, syndromes, meta.
template <int W, int S>
__device__ __forceinline__ void emit_set(const InfosetDesc& D, const Rows<W, S>& M, int g, int rank,
                                         const unsigned long long (&piv)[2], int lane,
                                         unsigned long long* __restrict__ heap,
                                         unsigned long long* __restrict__ heap_ctr) {
    const int K = D.K;
    unsigned long long off = 0;
    if (lane == 0) off = atomicAdd(heap_ctr, (unsigned long long)K * W);
    off = __shfl_sync(0xffffffffu, off, 0);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int row = 32 * s + lane;
        if (row < K) {
#pragma unroll
            for (int w = 0; w < W; ++w) heap[off + (size_t)row * W + w] = M.r[s][w];
        }
    }
    // non-pivot columns of [0, n), ascending, 32 per output word
    unsigned long long np0 = ~piv[0], np1 = W > 1 ? ~piv[1] : 0ull;
    if (D.n < 64) { np0 &= (1ull << D.n) - 1ull; np1 = 0ull; }
    else if (D.n < 128) np1 &= (1ull << (D.n - 64)) - 1ull;
    uint32_t* red = D.red + (size_t)g * K * D.W32;
    for (int ow = 0; ow < D.W32; ++ow) {
        uint32_t acc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] = 0u;
        for (int j = 0; j < 32; ++j) {
            int c;
            if (np0) { c = __ffsll((long long)np0) - 1; np0 &= np0 - 1ull; }
            else if (np1) { c = 64 + __ffsll((long long)np1) - 1; np1 &= np1 - 1ull; }
            else break;
#pragma unroll
            for (int s = 0; s < S; ++s)
                acc[s] |= (uint32_t)((M.word(s, c >> 6) >> (c & 63)) & 1ull) << j;
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int row = 32 * s + lane;
            if (row < K) red[(size_t)row * D.W32 + ow] = acc[s];
        }
    }
    // detector syndromes, 32 checks per output word; the 32 check rows of a word are loaded
    // by the 32 lanes (one each) and broadcast by shuffle, so no lane waits on a chain of
    // dependent global loads
    uint32_t* syn = D.syn + (size_t)g * K * D.SWP;
    for (int ow = 0; ow < D.SWP; ++ow) {
        uint32_t acc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] = 0u;
        const int cl = 32 * ow + lane;
        unsigned long long mine[W];
#pragma unroll
        for (int w = 0; w < W; ++w) mine[w] = cl < D.kcheck ? __ldg(D.check + (size_t)cl * W + w) : 0ull;
        const int nc = min(32, D.kcheck - 32 * ow);
        for (int j = 0; j < nc; ++j) {
            unsigned long long ck[W];
#pragma unroll
            for (int w = 0; w < W; ++w) ck[w] = __shfl_sync(0xffffffffu, mine[w], j);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                int p = 0;
#pragma unroll
                for (int w = 0; w < W; ++w) p += __popcll(ck[w] & M.r[s][w]);
                acc[s] |= (uint32_t)(p & 1) << j;
            }
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int row = 32 * s + lane;
            if (row < K) syn[(size_t)row * D.SWP + ow] = acc[s];
        }
    }
    if (lane == 0) {
        D.meta->rank[g] = rank;
        D.meta->g_off[g] = (int)off;
        D.meta->piv[g][0] = piv[0];
        D.meta->piv[g][1] = piv[1];
    }
}

template <int W, int S>
__device__ void side_sets(const InfosetDesc& D, int lane, unsigned long long* __restrict__ heap,
                          unsigned long long* __restrict__ heap_ctr) {
    const int K = D.K, n = D.n;
    Rows<W, S> M;
    M.load(D.gen, K, lane);
    int sets = 0;
    if (D.lists == nullptr) {
        unsigned long long act[2];
        act[0] = n >= 64 ? ~0ull : (1ull << n) - 1ull;
        act[1] = n >= 128 ? ~0ull : (n > 64 ? (1ull << (n - 64)) - 1ull : 0ull);
        for (;;) {
            unsigned long long piv[2] = {0ull, 0ull};
            int rank = 0;
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                unsigned long long m = act[w];
                while (m && rank < K) {
                    const int col = 64 * w + __ffsll((long long)m) - 1;
                    m &= m - 1ull;
                    if (M.step(col, rank, lane)) {
                        piv[w] |= 1ull << (col & 63);
                        ++rank;
                    }
                }
            }
            emit_set<W, S>(D, M, sets, rank, piv, lane, heap, heap_ctr);
            ++sets;
            // columns still holding a 1 in some row (the OR of the rows, over the warp)
            unsigned long long any[2] = {0ull, 0ull};
#pragma unroll
            for (int s = 0; s < S; ++s)
#pragma unroll
                for (int w = 0; w < W; ++w) any[w] |= M.r[s][w];
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)any[w]);
                const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(any[w] >> 32));
                any[w] = ((unsigned long long)hi << 32) | lo;
            }
            const unsigned long long nx0 = act[0] & ~piv[0] & any[0];
            const unsigned long long nx1 = act[1] & ~piv[1] & any[1];
            if ((nx0 == act[0] && nx1 == act[1]) || (nx0 == 0ull && nx1 == 0ull)) break;
            if (sets == kInfosetMaxSets) { sets = -1; break; }
            act[0] = nx0;
            act[1] = nx1;
        }
    } else {
        int off = 0;
        for (int g = 0; g < D.nlists; ++g) {
            if (g > 0) M.load(D.gen, K, lane);   // every class starts from the generator
            unsigned long long piv[2] = {0ull, 0ull};
            int rank = 0;
            const int len = D.list_len[g];
            for (int ci = 0; ci < len && rank < K; ++ci) {
                const int col = __ldg(D.lists + off + ci);
                if (M.step(col, rank, lane)) {
                    if (col < 64) piv[0] |= 1ull << col;
                    else piv[1] |= 1ull << (col - 64);
                    ++rank;
                }
            }
            off += len;
            emit_set<W, S>(D, M, g, rank, piv, lane, heap, heap_ctr);
        }
        sets = D.nlists;
    }
    if (lane == 0) D.meta->sets = sets;
}

template <int W>
__global__ void __launch_bounds__(32) infoset_kernel(const InfosetDesc* __restrict__ descs,
                                                      int ndesc,
                                                      unsigned long long* __restrict__ heap,
                                                      unsigned long long* __restrict__ heap_ctr) {
    const int lane = threadIdx.x & 31;
    const int side = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (side >= ndesc) return;
    const InfosetDesc& D = descs[side];
    switch ((D.K + 31) >> 5) {   // row slots in use, uniform over the warp
        case 0: if (lane == 0) D.meta->sets = 0; return;
        case 1: side_sets<W, 1>(D, lane, heap, heap_ctr); break;
        case 2: side_sets<W, 2>(D, lane, heap, heap_ctr); break;
        case 3: side_sets<W, 3>(D, lane, heap, heap_ctr); break;
        default: side_sets<W, 4>(D, lane, heap, heap_ctr); break;
    }
}

}  // namespace dev

cudaError_t launch_infosets(int W, const InfosetDesc* d_descs, int ndesc,
                            unsigned long long* d_heap, unsigned long long* d_heap_ctr,
                            cudaStream_t st) {
    if (ndesc <= 0) return cudaSuccess;
    // one warp per block: it fits in the registers a running tensor-core sweep CTA leaves
    // free on its SM, so it does not wait for the sweep's launch to end
    const int blocks = ndesc;
    if (W == 1) dev::infoset_kernel<1><<<blocks, 32, 0, st>>>(d_descs, ndesc, d_heap, d_heap_ctr);
    else if (W == 2) dev::infoset_kernel<2><<<blocks, 32, 0, st>>>(d_descs, ndesc, d_heap, d_heap_ctr);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace qsfb
