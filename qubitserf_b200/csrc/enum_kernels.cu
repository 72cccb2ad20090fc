// sm_100a kernels of the BZ enumeration: list generation and the XOR-popcount pair sweep.
//
// Semantics kept from the reference (cpp/qsf/enum_core.hpp:74-88, 109-194): for every
// active information set g and every w-subset S of its K rows, c = XOR of the rows; c is
// a candidate if it is a logical (no detector, or odd overlap with some detector row) and
// its full Hamming weight does not exceed the current bound; the level returns the
// smallest candidate.  The traversal is this engine's own (engine_types.hpp): subsets are
// split into a colex-ordered prefix list and a reflected-colex suffix list, so a level is
// a set of rectangles of independent (prefix, suffix) pairs that a warp sweeps with the
// prefix entries in registers and the suffix entries broadcast from L1.
//
// The hot loop is bound by the POPC (XU) pipe: per pair a few LOP3s fold the XORed probe
// words into one (or two) words whose popcount bounds the probe weight from below, one
// POPC each and one fused add/min; the pivot columns never enter it (they contribute the
// pivot-row count).  A chunk whose minimum stays at or above the bound is rejected there;
// the rare chunks under it are rescanned exactly, their survivors re-evaluated over all
// words, tested against the detector syndromes and folded into the side's packed witness
// key with one 64-bit atomicMin.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "engine_types.hpp"
#include "enum_device.cuh"

namespace qsfb {
namespace dev {

constexpr int RX = 8;           // register-side entries per lane
constexpr int kChunk = 32;      // loop entries between survivor checks

// ---------------------------------------------------------------- list generation
// One thread per run of kGenRun consecutive entries of a list: the first entry is unranked
// (binary searches over the binomial table), the next ones follow by the colex successor
// (raise the lowest element that can move, reset the ones below it), so the XOR of the
// rows changes by the few rows that leave and enter -- usually one of each.  Lists over at
// most 128 rows keep the subset as a bit mask in registers (gen_run_mask); longer ones
// keep its elements in an array.
__device__ __forceinline__ void xor_row(const GenDesc& D, int row, uint32_t (&acc)[4]) {
    const uint32_t* r = D.red + (size_t)row * D.W32;
#pragma unroll
    for (int h = 0; h < 4; ++h)
        if (h < D.HP && h < D.W32) acc[h] ^= __ldg(r + h);
}

// Write entry e of list D: its probe words, pivot count and (where a tensor plan reads it)
// its +-1 row.
__device__ __forceinline__ void put_entry(const GenDesc& D, unsigned long long e,
                                          const uint32_t (&acc)[4], int pc) {
    uint32_t* o = D.out + e * (unsigned long long)D.HP;
    if (D.HP == 4) {
        *reinterpret_cast<uint4*>(o) = make_uint4(acc[0], acc[1], acc[2], acc[3]);
    } else if (D.HP == 2) {
        *reinterpret_cast<uint2*>(o) = make_uint2(acc[0], acc[1]);
    } else {
        o[0] = acc[0];
    }
    if (D.pc) D.pc[e] = (uint8_t)pc;
    if (D.pm && e >= D.pm_lo && e < D.pm_hi)   // +-1 form of the rows a tensor plan reads
        write_pm_row(D.pm, e, acc[0], acc[1], D.n_enc);
}

// Lists over K <= 128 rows: the subset is a 128-bit mask in registers.  Entry e0 is
// unranked straight into the mask; the colex successor of a k-subset is the next larger
// integer with the same popcount (add the lowest set bit, then move the bits that the carry
// cleared back to the bottom), and the XOR of the rows changes by the bits that flip.
__device__ __forceinline__ void gen_run_mask(const GenDesc& D, const unsigned long long* B,
                                             unsigned long long e0, int n) {
    typedef unsigned __int128 u128;
    const int s = D.size, K = D.K;
    u128 x = 0;
    {
        unsigned long long r = e0;
        int hi = K;
        for (int i = s; i >= 1; --i) {   // colex unrank, largest element first
            const int lo = colex_top(B, r, i, hi);
            x |= (u128)1 << lo;
            r -= binom(B, lo, i);
            hi = lo;
        }
    }
    // element v stands for row v (colex) or row K - 1 - v (reflected); pivot rows are < rank
    u128 piv = 0;
    if (D.rank > 0) {
        const u128 low = D.rank >= 128 ? ~(u128)0 : (((u128)1 << D.rank) - 1);
        piv = D.reflect ? (low << (K - D.rank)) : low;
    }
    auto flip = [&](u128 d, uint32_t (&acc)[4]) {
        for (int half = 0; half < 2; ++half) {
            unsigned long long w = (unsigned long long)(d >> (64 * half));
            while (w) {
                const int b = 64 * half + __ffsll((long long)w) - 1;
                w &= w - 1;
                xor_row(D, D.reflect ? K - 1 - b : b, acc);
            }
        }
    };
    auto popc128 = [](u128 v) {
        return __popcll((unsigned long long)v) + __popcll((unsigned long long)(v >> 64));
    };
    uint32_t acc[4] = {0u, 0u, 0u, 0u};
    flip(x, acc);
    for (int j = 0; j < n; ++j) {
        put_entry(D, e0 + j, acc, popc128(x & piv));
        if (j + 1 == n) break;
        const unsigned long long lo64 = (unsigned long long)x;
        const int p = lo64 ? __ffsll((long long)lo64) - 1
                           : 64 + __ffsll((long long)(unsigned long long)(x >> 64)) - 1;
        const u128 v = x + ((u128)1 << p);
        const u128 moved = (v ^ x);
        const u128 next = v | (p + 2 < 128 ? (moved >> (p + 2)) : (u128)0);
        flip(x ^ next, acc);
        x = next;
    }
}

// Lists built from the list one size smaller of the same set and orientation.  In colex
// order the s-subsets whose largest element is c come as one block, after the C(c, s)
// subsets of [0, c), and in the order of their other s-1 elements, which are exactly the
// first C(c, s-1) entries of the smaller list.  So entry C(c, s) + j is entry j of the
// smaller list with row c added: its probe words the smaller entry's XOR row c, its pivot
// count the smaller entry's plus one when row c is a pivot row.  Only the run's first
// entry is located (its largest element, by colex_top); the rest stream through the
// smaller list.
__device__ __forceinline__ void gen_run_rec(const GenDesc& D, const unsigned long long* B,
                                            unsigned long long e0, int n) {
    const int s = D.size, K = D.K;
    int c = colex_top(B, e0, s, K);
    unsigned long long j = e0 - binom(B, c, s);
    unsigned long long blk = binom(B, c, s - 1);   // entries whose largest element is c
    for (int k = 0; k < n; ++k) {
        while (j >= blk) {   // into the next block (blk >= 1: c >= s - 1)
            j -= blk;
            ++c;
            blk = binom(B, c, s - 1);
        }
        const int row = D.reflect ? K - 1 - c : c;
        uint32_t acc[4] = {0u, 0u, 0u, 0u};
        const uint32_t* in = D.src + j * (unsigned long long)D.HP;
        if (D.HP == 4) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(in));
            acc[0] = q.x; acc[1] = q.y; acc[2] = q.z; acc[3] = q.w;
        } else if (D.HP == 2) {
            const uint2 q = __ldg(reinterpret_cast<const uint2*>(in));
            acc[0] = q.x; acc[1] = q.y;
        } else {
            acc[0] = __ldg(in);
        }
        xor_row(D, row, acc);
        const int pc = D.src_pc ? (int)__ldg(D.src_pc + j) + (row < D.rank ? 1 : 0) : 0;
        put_entry(D, e0 + k, acc, pc);
        ++j;
    }
}

__global__ void __launch_bounds__(256) gen_lists_kernel(const GenDesc* __restrict__ descs,
                                                        int ndesc, unsigned long long total,
                                                        const unsigned long long* __restrict__ B) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long gr = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         gr < total; gr += stride) {
        int lo = 0, hi = ndesc - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (descs[mid].entry_base <= gr) lo = mid; else hi = mid - 1;
        }
        const GenDesc& D = descs[lo];
        const unsigned long long e0 = (gr - D.entry_base) * kGenRun;
        const int n = (int)(D.count - e0 < (unsigned long long)kGenRun ? D.count - e0 : kGenRun);
        if (D.src) {
            gen_run_rec(D, B, e0, n);
            continue;
        }
        if (D.K <= 128) {
            gen_run_mask(D, B, e0, n);
            continue;
        }
        const int s = D.size;
        // colex combination, ascending: c[0] < c[1] < ... < c[s-1]
        int c[kMaxW], top[kMaxW];
        colex_unrank(B, e0, s, D.K, top);          // largest first
        for (int i = 0; i < s; ++i) c[i] = top[s - 1 - i];
        auto row_of = [&](int v) { return D.reflect ? D.K - 1 - v : v; };
        uint32_t acc[4] = {0u, 0u, 0u, 0u};
        int pc = 0;
        for (int i = 0; i < s; ++i) {
            const int r = row_of(c[i]);
            xor_row(D, r, acc);
            pc += r < D.rank;
        }
        for (int j = 0; j < n; ++j) {
            put_entry(D, e0 + j, acc, pc);
            if (j + 1 == n) break;
            // colex successor: lowest t with c[t] + 1 < c[t+1] (c[s] = K)
            int t = 0;
            while (t < s - 1 && c[t] + 1 == c[t + 1]) ++t;
            for (int i = 0; i <= t; ++i) {
                const int r_old = row_of(c[i]);
                xor_row(D, r_old, acc);
                pc -= r_old < D.rank;
                c[i] = i < t ? i : c[i] + 1;
                const int r_new = row_of(c[i]);
                xor_row(D, r_new, acc);
                pc += r_new < D.rank;
            }
        }
    }
}

// ---------------------------------------------------------------- pair sweep
// Probe filters.  A filter maps the XORed probe words of a pair to a lower bound on their
// popcount sum, at fewer POPCs (the XU pipe, the sweep's bottleneck) than the exact sum:
//   FILT 1..4: popc(a | b | ...) over the first FILT words (one POPC);
//   FILT 6:    carry-save over four words, popc(a^b^c^d) + 2 popc(maj(a,b,c) | (a^b^c)&d),
//              exact except that a column set in all four words counts 2 (two POPCs).
// Every pair whose exact sum is under the bound is under it on the filter as well, so the
// filter only decides which chunks get the exact rescan.
__host__ __device__ constexpr int filter_words(int filt) { return filt == 6 ? 4 : filt; }

template <int H, int HP>
__device__ __forceinline__ void load_entry(const uint32_t* __restrict__ p, uint32_t (&v)[H]) {
    if constexpr (HP == 4) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(p));
        const uint32_t t[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int h = 0; h < H; ++h) v[h] = t[h];
    } else if constexpr (HP == 2) {
        const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
        v[0] = q.x;
        if constexpr (H > 1) v[1] = q.y;
    } else {
        v[0] = __ldg(p);
    }
}

// Filter value of one pair (no pivot rows).
template <int FILT>
__device__ __forceinline__ int filter_value(const uint32_t (&x)[filter_words(FILT)],
                                            const uint32_t (&y)[filter_words(FILT)]) {
    if constexpr (FILT == 6) {
        const uint32_t a = x[0] ^ y[0], b = x[1] ^ y[1], c = x[2] ^ y[2], d = x[3] ^ y[3];
        const uint32_t s = a ^ b ^ c;
        const uint32_t mj = (a & b) | (c & (a | b));
        return __popc(s ^ d) + 2 * __popc(mj | (s & d));
    } else {
        uint32_t v = x[0] ^ y[0];
#pragma unroll
        for (int h = 1; h < FILT; ++h) v |= x[h] ^ y[h];
        return __popc(v);
    }
}

// OR of the XORed probe words (zero exactly when every probe word of the pair's XOR is).
template <int H>
__device__ __forceinline__ uint32_t xor_or(const uint32_t (&x)[H], const uint32_t (&y)[H]) {
    uint32_t v = x[0] ^ y[0];
#pragma unroll
    for (int h = 1; h < H; ++h) v |= x[h] ^ y[h];
    return v;
}

// m = min(m, filter + extra), the add folded into the DPX add-min.
template <int FILT>
__device__ __forceinline__ int fold_min(const uint32_t (&x)[filter_words(FILT)],
                                        const uint32_t (&y)[filter_words(FILT)], int extra, int m) {
    if constexpr (FILT == 6) {
        const uint32_t a = x[0] ^ y[0], b = x[1] ^ y[1], c = x[2] ^ y[2], d = x[3] ^ y[3];
        const uint32_t s = a ^ b ^ c;
        const uint32_t mj = (a & b) | (c & (a | b));
        return __viaddmin_s32(__popc(s ^ d) + extra, 2 * __popc(mj | (s & d)), m);
    } else {
        uint32_t v = x[0] ^ y[0];
#pragma unroll
        for (int h = 1; h < FILT; ++h) v |= x[h] ^ y[h];
        return __viaddmin_s32(__popc(v), extra, m);
    }
}

// Zero test: running unsigned minimum of the OR of the XORed probe words (no POPC); a
// pair can only be a candidate when every probe word of its XOR is zero.
template <int H>
__device__ __forceinline__ uint32_t fold_zero(const uint32_t (&x)[H], const uint32_t (&y)[H],
                                              uint32_t m) {
    uint32_t v = x[0] ^ y[0];
#pragma unroll
    for (int h = 1; h < H; ++h) v |= x[h] ^ y[h];
    return v < m ? v : m;
}

// MODE 0: rank-deficient set (per-entry pivot counts); 1: full-rank set, popcount bound;
// 2: full-rank set whose bound leaves no room for any non-pivot bit (zero test).
// FILT is the probe filter (filter_words(FILT) probe words of the HP stored per entry).
template <int FILT, int HP, int MODE>
__global__ void __launch_bounds__(128) pairs_kernel(const LevelDesc* __restrict__ descs,
                                                    int ndesc, unsigned long long total_jobs,
                                                    unsigned long long* __restrict__ job_counter,
                                                    const unsigned long long* __restrict__ B) {
    constexpr bool FULL = MODE != 0;
    constexpr bool ZERO = MODE == 2;
    constexpr int H = filter_words(FILT);
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long job = 0;
        if (lane == 0) job = atomicAdd(job_counter, 1ull);
        job = __shfl_sync(0xffffffffu, job, 0);
        if (job >= total_jobs) break;

        int lo = 0, hi = ndesc - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (descs[mid].job_base <= job) lo = mid; else hi = mid - 1;
        }
        const LevelDesc& D = descs[lo];
        const unsigned long long local = job - D.job_base;
        // term t: largest t with term_jobs[t] <= local
        int tl = 0, th = D.nterms - 1;
        while (tl < th) {
            const int mid = (tl + th + 1) >> 1;
            if (__ldg(D.term_jobs + mid) <= local) tl = mid; else th = mid - 1;
        }
        const unsigned long long idx = local - __ldg(D.term_jobs + tl);
        const int p = D.p_lo + tl;
        const unsigned long long nx = binom(B, p, D.a - 1);
        const unsigned long long ny = binom(B, D.K - 1 - p, D.b);
        const unsigned long long xoff = binom(B, p, D.a);
        const int regX = nx >= ny;
        const unsigned long long reg_n = regX ? nx : ny;
        const unsigned long long loop_n = regX ? ny : nx;
        const unsigned long long njl = (loop_n + D.loop_tile - 1) / D.loop_tile;
        const unsigned long long ri = idx / njl, li = idx - ri * njl;
        const unsigned long long reg0 = ri * kRegTile;
        const unsigned long long reg_cnt =
            (reg_n - reg0) < (unsigned long long)kRegTile ? (reg_n - reg0) : kRegTile;
        const unsigned long long loop0 = li * D.loop_tile;
        const int loop_cnt = (int)((loop_n - loop0) < (unsigned long long)D.loop_tile
                                       ? (loop_n - loop0) : (unsigned long long)D.loop_tile);
        const uint32_t* regbase = regX ? D.la + xoff * HP : D.rb;
        const uint8_t* regpc = regX ? (D.pca ? D.pca + xoff : nullptr) : D.pcb;
        const uint32_t* loopbase = regX ? D.rb : D.la + xoff * HP;
        const uint8_t* looppc = regX ? D.pcb : (D.pca ? D.pca + xoff : nullptr);

        // strict bound: the key's weight field holds (best weight + 1)
        int T = (int)(*((volatile unsigned long long*)D.key) >> kKeyWtShift);

        uint32_t x[RX][H];
        int thr[RX], m[RX], pcr[RX];
#pragma unroll
        for (int i = 0; i < RX; ++i) {
            const unsigned long long e = reg0 + lane + 32 * i;
            const bool ok = (unsigned long long)(lane + 32 * i) < reg_cnt;
            if (ok) {
                load_entry<H, HP>(regbase + e * HP, x[i]);
                pcr[i] = FULL ? (regX ? D.a : D.b) : (int)regpc[e];
            } else {
#pragma unroll
                for (int h = 0; h < H; ++h) x[i][h] = 0u;
                pcr[i] = 1 << 20;
            }
            thr[i] = T - pcr[i] - (FULL ? (regX ? D.b : D.a) : 0);
            m[i] = ZERO ? -1 : 0x7fffffff;
        }

        // Sweep the loop entries in chunks of kChunk; after each chunk the (rare) lanes
        // whose running minimum reached the bound rescan just that chunk.
        const uint32_t* lp = loopbase + loop0 * HP;
        const uint8_t* lpc = FULL ? nullptr : looppc + loop0;
        for (int c0 = 0; c0 < loop_cnt; c0 += kChunk) {
            const int cn = (loop_cnt - c0) < kChunk ? (loop_cnt - c0) : kChunk;
            int j = c0;
            const int cend = c0 + cn;
            if (FULL) {
                for (; j + 4 <= cend; j += 4) {
                    uint32_t y0[H], y1[H], y2[H], y3[H];
                    load_entry<H, HP>(lp + (j + 0) * HP, y0);
                    load_entry<H, HP>(lp + (j + 1) * HP, y1);
                    load_entry<H, HP>(lp + (j + 2) * HP, y2);
                    load_entry<H, HP>(lp + (j + 3) * HP, y3);
#pragma unroll
                    for (int i = 0; i < RX; ++i) {
                        // two pairs per three-input DPX minimum
                        if constexpr (ZERO) {
                            uint32_t mm = (uint32_t)m[i];
                            mm = __vimin3_u32(xor_or<H>(x[i], y0), xor_or<H>(x[i], y1), mm);
                            mm = __vimin3_u32(xor_or<H>(x[i], y2), xor_or<H>(x[i], y3), mm);
                            m[i] = (int)mm;
                        } else {
                            int mm = m[i];
                            mm = __vimin3_s32(filter_value<FILT>(x[i], y0),
                                              filter_value<FILT>(x[i], y1), mm);
                            mm = __vimin3_s32(filter_value<FILT>(x[i], y2),
                                              filter_value<FILT>(x[i], y3), mm);
                            m[i] = mm;
                        }
                    }
                }
                for (; j < cend; ++j) {
                    uint32_t y0[H];
                    load_entry<H, HP>(lp + j * HP, y0);
#pragma unroll
                    for (int i = 0; i < RX; ++i) {
                        if constexpr (ZERO) m[i] = (int)fold_zero<H>(x[i], y0, (uint32_t)m[i]);
                        else m[i] = fold_min<FILT>(x[i], y0, 0, m[i]);
                    }
                }
            } else {
                for (; j < cend; ++j) {
                    uint32_t y0[H];
                    load_entry<H, HP>(lp + j * HP, y0);
                    const int pcy = (int)__ldg(lpc + j);
#pragma unroll
                    for (int i = 0; i < RX; ++i) m[i] = fold_min<FILT>(x[i], y0, pcy, m[i]);
                }
            }
            // entries whose chunk minimum reached the bound, as a bit mask: walking it keeps
            // m[], thr[] and pcr[] indexed by constants only (a run-time index would move
            // them to local memory, and m[] is updated for every loop entry)
            uint32_t flagged = 0u;
#pragma unroll
            for (int i = 0; i < RX; ++i)
                flagged |= (ZERO ? (m[i] == 0 && thr[i] > 0) : m[i] < thr[i]) ? (1u << i) : 0u;
            if (flagged) {
                while (flagged) {
                    const int i = __ffs(flagged) - 1;
                    flagged &= flagged - 1u;
                    const unsigned long long e = reg0 + lane + 32 * i;
                    const int pc = FULL ? (regX ? D.a : D.b) : (int)regpc[e];
                    T = survivor_scan(D, B, regX, xoff, e, pc, loop0 + (unsigned long long)c0,
                                      cn, T);
                }
#pragma unroll
                for (int i = 0; i < RX; ++i)
                    thr[i] = T - pcr[i] - (FULL ? (regX ? D.b : D.a) : 0);
            }
#pragma unroll
            for (int i = 0; i < RX; ++i) m[i] = ZERO ? -1 : 0x7fffffff;
        }
        if (lane == 0) atomicAdd(D.count, reg_cnt * (unsigned long long)loop_cnt);
    }
}

// Zero the kPmPadRows rows after each new +-1 list (whole-tile operand copies read past a
// list's last entry): one block per pad area per pass, 256 threads x 16 bytes per store.
__global__ void __launch_bounds__(256) zero_pads_kernel(int8_t* const* __restrict__ pads,
                                                        int npads) {
    constexpr int kVecs = kPmPadRows * kPmRowBytes / 16;   // 16-byte stores per pad area
    for (int p = blockIdx.x; p < npads; p += gridDim.x) {
        uint4* o = reinterpret_cast<uint4*>(pads[p]);
        for (int i = threadIdx.x; i < kVecs; i += blockDim.x) o[i] = make_uint4(0u, 0u, 0u, 0u);
    }
}

}  // namespace dev

// ---------------------------------------------------------------- host launchers
cudaError_t launch_zero_pads(int8_t* const* d_pads, int npads, int num_sms, cudaStream_t st) {
    if (npads <= 0) return cudaSuccess;
    const int blocks = std::min(npads, num_sms * 8);
    dev::zero_pads_kernel<<<blocks, 256, 0, st>>>(d_pads, npads);
    return cudaGetLastError();
}

cudaError_t launch_gen_lists(const GenDesc* d_descs, int ndesc, unsigned long long total,
                             const unsigned long long* d_binom, int num_sms, cudaStream_t st) {
    if (total == 0) return cudaSuccess;   // total: runs of kGenRun entries
    unsigned long long blocks = (total + 255) / 256;
    const unsigned long long cap = (unsigned long long)num_sms * 16;
    if (blocks > cap) blocks = cap;
    dev::gen_lists_kernel<<<(unsigned)blocks, 256, 0, st>>>(d_descs, ndesc, total, d_binom);
    return cudaGetLastError();
}

template <int FILT, int HP, int MODE>
static cudaError_t launch_pairs_t(const LevelDesc* d, int nd, unsigned long long jobs,
                                  unsigned long long* ctr, const unsigned long long* B,
                                  int num_sms, cudaStream_t st) {
    static int blocks_per_sm = 0;
    if (blocks_per_sm == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm,
                                                      dev::pairs_kernel<FILT, HP, MODE>, 128, 0);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    unsigned long long blocks = (unsigned long long)num_sms * blocks_per_sm;
    const unsigned long long need = (jobs + 3) / 4;   // 4 warps per block
    if (need < blocks) blocks = need;
    if (blocks < 1) blocks = 1;
    dev::pairs_kernel<FILT, HP, MODE><<<(unsigned)blocks, 128, 0, st>>>(d, nd, jobs, ctr, B);
    return cudaGetLastError();
}

#define QSFB_PAIRS_CASE(F, HP, M) \
    case ((F) * 8 + (HP)) * 4 + (M): \
        return launch_pairs_t<F, HP, M>(d, nd, jobs, ctr, B, num_sms, st);

cudaError_t launch_pairs(int filt, int HP, int mode, const LevelDesc* d, int nd,
                         unsigned long long jobs, unsigned long long* ctr,
                         const unsigned long long* B, int num_sms, cudaStream_t st) {
    if (jobs == 0) return cudaSuccess;
    switch ((filt * 8 + HP) * 4 + mode) {
        QSFB_PAIRS_CASE(1, 1, 0) QSFB_PAIRS_CASE(1, 1, 1) QSFB_PAIRS_CASE(1, 1, 2)
        QSFB_PAIRS_CASE(2, 2, 0) QSFB_PAIRS_CASE(2, 2, 1) QSFB_PAIRS_CASE(2, 2, 2)
        QSFB_PAIRS_CASE(2, 4, 0) QSFB_PAIRS_CASE(2, 4, 1) QSFB_PAIRS_CASE(2, 4, 2)
        QSFB_PAIRS_CASE(3, 4, 0) QSFB_PAIRS_CASE(3, 4, 1)
        QSFB_PAIRS_CASE(4, 4, 0) QSFB_PAIRS_CASE(4, 4, 1)
        QSFB_PAIRS_CASE(6, 4, 0) QSFB_PAIRS_CASE(6, 4, 1)
        default: return cudaErrorInvalidValue;
    }
}
#undef QSFB_PAIRS_CASE

}  // namespace qsfb
