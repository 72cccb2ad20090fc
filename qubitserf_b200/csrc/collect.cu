// sm_100a kernels of the low-weight collector (the codeaut_bz_* boundary): list generation
// and the pair sweep that appends every subset XOR of weight 1..keep.
//
// Semantics kept from the reference (cpp/codeaut/bz.cpp:82-97 and the CollectSink of
// cpp/qsf/enum_core.hpp:90-103): for every subset size sw the XOR of every sw-subset of the
// generator's rows is a hit when its full Hamming weight lies in [1, keep]; duplicates are
// allowed here and removed by the host.  The traversal is this engine's own
// (collect_types.hpp): prefix/suffix lists of probe words and pivot counts, swept as
// rectangles of pairs with the prefix entries in registers and the suffix entries
// broadcast to the warp.
//
// The sweep is bound by the POPC (XU) pipe: per pair a few XORs/ORs and one or two POPCs
// give a lower bound on pivots + popc(probe) (probe_bound below); a three-input minimum
// folds eight of them per suffix entry and only a minimum under keep + 1 makes the lane
// append its candidate pairs.  collect_exact_kernel then unranks both subsets of every
// candidate, XORs their full rows and appends the codeword when its weight is in range.
#include <cuda_runtime.h>
#include <cstdint>

#include "collect_types.hpp"
#include "engine_types.hpp"
#include "enum_device.cuh"

namespace qsfb {
namespace dev {

constexpr int kCRX = kCollectTileX / 32;   // prefix entries per lane
constexpr int kCFar = 1 << 20;             // pivot count of an empty register slot
static_assert(kCRX == 8, "the minimum fold below takes eight register entries");

// ---------------------------------------------------------------- list generation
// One thread per run of kGenRun consecutive entries of a list: the first entry is unranked
// over the binomial table, the next follow by the colex successor (the rows that leave and
// enter change the XOR; usually one of each).
__global__ void __launch_bounds__(256) collect_gen_kernel(const CollectListDesc* __restrict__ lists,
                                                          int nlists, unsigned long long runs,
                                                          CollectShared S,
                                                          const unsigned long long* __restrict__ B) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long gr = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         gr < runs; gr += stride) {
        int lo = 0, hi = nlists - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (lists[mid].run_base <= gr) lo = mid; else hi = mid - 1;
        }
        const CollectListDesc& D = lists[lo];
        const unsigned long long e0 = (gr - D.run_base) * kGenRun;
        const int n = (int)(D.count - e0 < (unsigned long long)kGenRun ? D.count - e0 : kGenRun);
        const int s = D.size;
        int c[kCollectMaxSize], top[kCollectMaxSize];
        colex_unrank(B, e0, s, S.m, top);   // largest first
        for (int i = 0; i < s; ++i) c[i] = top[s - 1 - i];
        auto row_of = [&](int v) { return D.reflect ? S.m - 1 - v : v; };
        uint32_t acc[kCollectMaxProbe];
#pragma unroll
        for (int h = 0; h < kCollectMaxProbe; ++h) acc[h] = 0u;
        auto xor_row = [&](int r) {
            const uint32_t* p = S.probe_rows + (size_t)r * S.HP;
#pragma unroll
            for (int h = 0; h < kCollectMaxProbe; ++h)
                if (h < S.HP) acc[h] ^= __ldg(p + h);
        };
        int pc = 0;
        for (int i = 0; i < s; ++i) {
            const int r = row_of(c[i]);
            xor_row(r);
            pc += __ldg(S.piv + r);
        }
        for (int j = 0; j < n; ++j) {
            const unsigned long long e = e0 + j;
            uint32_t* o = D.probe + e * (unsigned long long)S.HP;
#pragma unroll
            for (int h = 0; h < kCollectMaxProbe; ++h)
                if (h < S.HP) o[h] = acc[h];
            D.pc[e] = (uint8_t)pc;
            if (j + 1 == n) break;
            // colex successor: lowest t with c[t] + 1 < c[t+1] (c[s] = m)
            int t = 0;
            while (t < s - 1 && c[t] + 1 == c[t + 1]) ++t;
            for (int i = 0; i <= t; ++i) {
                const int r_old = row_of(c[i]);
                xor_row(r_old);
                pc -= __ldg(S.piv + r_old);
                c[i] = i < t ? i : c[i] + 1;
                const int r_new = row_of(c[i]);
                xor_row(r_new);
                pc += __ldg(S.piv + r_new);
            }
        }
    }
}

// ---------------------------------------------------------------- pair sweep
// HP probe words of one staged suffix entry (16-byte aligned for HP >= 4, 8 for HP = 2).
template <int HP>
__device__ __forceinline__ void stage_probe(const uint32_t* p, uint32_t (&v)[HP]) {
    if constexpr (HP >= 4) {
#pragma unroll
        for (int h = 0; h < HP; h += 4) {
            const uint4 a = *reinterpret_cast<const uint4*>(p + h);
            v[h] = a.x; v[h + 1] = a.y; v[h + 2] = a.z; v[h + 3] = a.w;
        }
    } else if constexpr (HP == 2) {
        const uint2 a = *reinterpret_cast<const uint2*>(p);
        v[0] = a.x; v[1] = a.y;
    } else {
        v[0] = p[0];
    }
}

template <int HP>
__device__ __forceinline__ void load_probe(const uint32_t* __restrict__ p, uint32_t (&v)[HP]) {
    if constexpr (HP == 8) {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
        const uint4 b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else if constexpr (HP == 4) {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else if constexpr (HP == 2) {
        const uint2 a = __ldg(reinterpret_cast<const uint2*>(p));
        v[0] = a.x; v[1] = a.y;
    } else {
        v[0] = __ldg(p);
    }
}

// Lower bound on the probe weight of a pair (the popcount of the XORed probe words):
//   FILT 0: the exact sum, HP POPCs;
//   FILT 2 / 4: popc of the OR of the 2 / 4 XORed words, one POPC;
//   FILT 6: carry-save over four words, popc(a^b^c^d) + 2 popc(maj(a,b,c) | (a^b^c)&d),
//           exact except that a column set in all four counts 2 (two POPCs).
template <int HP, int FILT>
__device__ __forceinline__ int probe_bound(const uint32_t (&x)[HP], const uint32_t (&y)[HP]) {
    if constexpr (FILT == 0) {
        int s = 0;
#pragma unroll
        for (int h = 0; h < HP; ++h) s += __popc(x[h] ^ y[h]);
        return s;
    } else if constexpr (FILT == 2) {
        static_assert(HP >= 2, "FILT 2 reads two probe words");
        return __popc((x[0] ^ y[0]) | (x[1] ^ y[1]));
    } else if constexpr (FILT == 4) {
        static_assert(HP >= 4, "FILT 4 reads four probe words");
        return __popc((x[0] ^ y[0]) | (x[1] ^ y[1]) | (x[2] ^ y[2]) | (x[3] ^ y[3]));
    } else {
        static_assert(FILT == 6 && HP >= 4, "FILT 6 reads four probe words");
        const uint32_t a = x[0] ^ y[0], b = x[1] ^ y[1], c = x[2] ^ y[2], d = x[3] ^ y[3];
        const uint32_t s3 = a ^ b ^ c;
        const uint32_t carry = ((a & b) | (a & c) | (b & c)) | (s3 & d);
        return __popc(s3 ^ d) + 2 * __popc(carry);
    }
}

// Exact evaluation of the candidates (prefix entry, suffix entry, subset size): both subsets
// unranked, their full rows XORed, the codeword appended when its weight is in [1, keep].
// The candidate count is read on the device; the hit counter keeps counting past the
// output capacity so that the host learns the exact hit count.
__global__ void __launch_bounds__(256) collect_exact_kernel(const CollectLevelDesc* __restrict__ levels,
                                                            CollectShared S,
                                                            const unsigned long long* __restrict__ B) {
    const unsigned long long nc = S.ctr[1] < S.cand_cap ? S.ctr[1] : S.cand_cap;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < nc;
         i += stride) {
        const unsigned long long w0 = S.cand[2 * i], ey = S.cand[2 * i + 1];
        const int sw = (int)(w0 >> 56);
        const unsigned long long ex = w0 & ((1ull << 56) - 1);
        const CollectLevelDesc& L = levels[sw - 1];
        int c[kCollectMaxSize];
        unsigned long long acc[kCollectMaxWords];
#pragma unroll
        for (int w = 0; w < kCollectMaxWords; ++w) acc[w] = 0ull;
        auto xor_row = [&](int r) {
            const unsigned long long* p = S.rows + (size_t)r * S.S64;
#pragma unroll
            for (int w = 0; w < kCollectMaxWords; ++w)
                if (w < S.S64) acc[w] ^= __ldg(p + w);
        };
        colex_unrank(B, ex, L.a, S.m, c);
        for (int k = 0; k < L.a; ++k) xor_row(c[k]);
        colex_unrank(B, ey, L.b, S.m, c);
        for (int k = 0; k < L.b; ++k) xor_row(S.m - 1 - c[k]);
        int wt = 0;
#pragma unroll
        for (int w = 0; w < kCollectMaxWords; ++w)
            if (w < S.S64) wt += __popcll(acc[w]);
        if (wt < 1 || wt > S.keep) continue;
        const unsigned long long slot = atomicAdd(S.ctr, 1ull);
        if (slot >= S.cap) continue;
        unsigned long long* o = S.out + slot * (unsigned long long)S.S64;
#pragma unroll
        for (int w = 0; w < kCollectMaxWords; ++w)
            if (w < S.S64) o[w] = acc[w];
    }
}

// The probe words of four consecutive staged entries (16-byte aligned: k is a multiple of 4).
template <int HP>
__device__ __forceinline__ void stage_group(const uint32_t* p, uint32_t (&v)[4][HP]) {
    if constexpr (HP == 1) {
        const uint4 a = *reinterpret_cast<const uint4*>(p);
        v[0][0] = a.x; v[1][0] = a.y; v[2][0] = a.z; v[3][0] = a.w;
    } else {
#pragma unroll
        for (int g = 0; g < 4; ++g) stage_probe<HP>(p + g * HP, v[g]);
    }
}

// The lane's eight prefix entries against one suffix entry: a bound per pair, one minimum,
// and for the rare pairs under keep + 1 an appended candidate.
template <int HP, int FILT>
__device__ __forceinline__ void pair_step(const CollectShared& S, const CollectTerm& T,
                                          const uint32_t (&xv)[kCRX][HP], const int (&xpc)[kCRX],
                                          const uint32_t (&ya)[HP], int pa, int lim, int level,
                                          unsigned long long xoff, int lane,
                                          unsigned long long ey) {
    int v[kCRX];
#pragma unroll
    for (int i = 0; i < kCRX; ++i) v[i] = xpc[i] + probe_bound<HP, FILT>(xv[i], ya);
    int mn = __vimin3_s32(v[0], v[1], v[2]);
    mn = __vimin3_s32(mn, v[3], v[4]);
    mn = __vimin3_s32(mn, v[5], v[6]);
    mn = min(mn, v[7]);
    if (mn + pa <= lim) {
        // unrolled: a run-time index into v[] would move it to local memory for every step
#pragma unroll
        for (int i = 0; i < kCRX; ++i) {
            if (v[i] + pa > lim) continue;
            const unsigned long long slot = atomicAdd(S.ctr + 1, 1ull);
            if (slot >= S.cand_cap) continue;
            S.cand[2 * slot] = (T.x0 + xoff + (unsigned long long)(i * 32 + lane)) |
                               ((unsigned long long)(level + 1) << 56);
            S.cand[2 * slot + 1] = ey;
        }
    }
}

// One warp per job (a 256-entry prefix tile of one term against up to kCollectChunkY
// suffix entries, staged in the warp's slice of shared memory), jobs handed out by a
// per-level counter; four warps per block.  A pair whose bound is under
// keep + 1 is appended to the candidates (rare: the probe filter is sized for it).
template <int HP, int FILT>
__global__ void __launch_bounds__(128) collect_pairs_kernel(const CollectLevelDesc* __restrict__ levels,
                                                            int level, CollectShared S,
                                                            const unsigned long long* __restrict__ B) {
    const CollectLevelDesc& L = levels[level];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ __align__(16) uint32_t ys_all[4][kCollectChunkY * HP];
    __shared__ __align__(16) uint8_t yq_all[4][kCollectChunkY];
    uint32_t* ys = ys_all[warp];
    uint8_t* yq = yq_all[warp];
    for (;;) {
        unsigned long long job = 0;
        if (lane == 0) job = atomicAdd(S.job_ctr + level, 1ull);
        job = __shfl_sync(0xffffffffu, job, 0);
        if (job >= L.jobs) break;
        int lo = 0, hi = L.nterms - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (L.terms[mid].job_base <= job) lo = mid; else hi = mid - 1;
        }
        const CollectTerm& T = L.terms[lo];
        const unsigned long long j = job - T.job_base;
        const unsigned long long xt = j / T.ychunks, yc = j - xt * T.ychunks;
        const unsigned long long xoff = xt * kCollectTileX;
        uint32_t xv[kCRX][HP];
        int xpc[kCRX];
#pragma unroll
        for (int i = 0; i < kCRX; ++i) {
            const unsigned long long xo = xoff + (unsigned long long)(i * 32 + lane);
            if (xo < T.nx) {
                const unsigned long long e = T.x0 + xo;
                load_probe<HP>(L.xp + e * HP, xv[i]);
                xpc[i] = __ldg(L.xpc + e);
            } else {
#pragma unroll
                for (int h = 0; h < HP; ++h) xv[i][h] = 0u;
                xpc[i] = kCFar;
            }
        }
        const unsigned long long y0 = yc * kCollectChunkY;
        const unsigned long long y1 = T.ny < y0 + kCollectChunkY ? T.ny : y0 + kCollectChunkY;
        const int cnt = (int)(y1 - y0);
        const int lim = S.keep;
        // the job's suffix entries go to this warp's shared-memory stage (coalesced), and the
        // pair loop reads them back as broadcasts
        __syncwarp();   // every lane is done with the previous job's stage
        for (int e = lane; e < cnt; e += 32) {
            uint32_t v[HP];
            load_probe<HP>(L.yp + (y0 + (unsigned long long)e) * HP, v);
#pragma unroll
            for (int h = 0; h < HP; ++h) ys[e * HP + h] = v[h];
            yq[e] = __ldg(L.ypc + y0 + e);
        }
        __syncwarp();
        // four staged entries per step: their probe words in 16-byte loads and their pivot
        // counts in one 32-bit word; the ragged end of the chunk goes one entry at a time
        int k = 0;
        for (; k + 4 <= cnt; k += 4) {
            uint32_t yv[4][HP];
            stage_group<HP>(ys + k * HP, yv);
            const uint32_t pcs = *reinterpret_cast<const uint32_t*>(yq + k);
#pragma unroll
            for (int g = 0; g < 4; ++g)
                pair_step<HP, FILT>(S, T, xv, xpc, yv[g], (int)((pcs >> (8 * g)) & 0xffu), lim,
                                    level, xoff, lane, y0 + (unsigned long long)(k + g));
        }
        for (; k < cnt; ++k) {
            uint32_t ya[HP];
            stage_probe<HP>(ys + k * HP, ya);
            pair_step<HP, FILT>(S, T, xv, xpc, ya, (int)yq[k], lim, level, xoff, lane,
                                y0 + (unsigned long long)k);
        }
    }
}

}  // namespace dev

cudaError_t launch_collect_gen(const CollectListDesc* d_lists, int nlists, unsigned long long runs,
                               const CollectShared& S, const unsigned long long* d_binom,
                               int num_sms, cudaStream_t st) {
    if (runs == 0) return cudaSuccess;
    const unsigned long long want = (runs + 255) / 256;
    const unsigned long long cap = (unsigned long long)num_sms * 8;
    const unsigned int grid = (unsigned int)(want < cap ? want : cap);
    dev::collect_gen_kernel<<<grid, 256, 0, st>>>(d_lists, nlists, runs, S, d_binom);
    return cudaGetLastError();
}

cudaError_t launch_collect_exact(const CollectLevelDesc* d_levels, const CollectShared& S,
                                 const unsigned long long* d_binom, int num_sms, cudaStream_t st) {
    dev::collect_exact_kernel<<<num_sms * 4, 256, 0, st>>>(d_levels, S, d_binom);
    return cudaGetLastError();
}

cudaError_t launch_collect_pairs(const CollectLevelDesc* d_levels, int level,
                                 unsigned long long jobs, const CollectShared& S,
                                 const unsigned long long* d_binom, int num_sms,
                                 cudaStream_t st) {
    if (jobs == 0) return cudaSuccess;
    // as many blocks as fit on the device at once (jobs are handed out dynamically)
    const unsigned long long want = (jobs + 3) / 4;   // four warps per block
#define QSFB_COLLECT_CASE(H, F)                                                              \
    if (S.HP == H && S.filt == F) {                                                          \
        static int per_sm = 0;                                                               \
        if (per_sm == 0 && cudaOccupancyMaxActiveBlocksPerMultiprocessor(                    \
                               &per_sm, dev::collect_pairs_kernel<H, F>, 128, 0) != cudaSuccess) \
            return cudaGetLastError();                                                       \
        const unsigned long long cap = (unsigned long long)num_sms * (per_sm > 0 ? per_sm : 1); \
        const unsigned int grid = (unsigned int)(want < cap ? want : cap);                   \
        dev::collect_pairs_kernel<H, F><<<grid, 128, 0, st>>>(d_levels, level, S, d_binom);  \
        return cudaGetLastError();                                                           \
    }
    QSFB_COLLECT_CASE(1, 0)
    QSFB_COLLECT_CASE(2, 0)
    QSFB_COLLECT_CASE(2, 2)
    QSFB_COLLECT_CASE(4, 0)
    QSFB_COLLECT_CASE(4, 4)
    QSFB_COLLECT_CASE(4, 6)
    QSFB_COLLECT_CASE(8, 0)
#undef QSFB_COLLECT_CASE
    return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace qsfb
