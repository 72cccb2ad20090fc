// Device helpers shared by the pair-sweep kernels (CUDA-core and tensor-core): subset
// unranking over the binomial table, the reference's lexicographic rank, and the exact
// survivor evaluation that both sweeps fall back to for the rare pairs their filters pass.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "engine_types.hpp"

namespace qsfb {
namespace dev {

constexpr int kLd = kBinomMaxK + 1;
constexpr int kMaxWords = 32;   // n <= 1024 bits after pivot removal; detector <= 1024 rows
constexpr int kMaxW = 64;

__device__ __forceinline__ unsigned long long binom(const unsigned long long* __restrict__ B,
                                                    int n, int k) {
    if (k < 0 || n < 0 || k > n) return 0ull;
    return __ldg(B + (size_t)n * kLd + k);
}

// Colex unrank: the r-th s-subset of [0, hi) in colex order, written largest first into
// c[0..s-1] (c[0] > c[1] > ...).  r = sum_i C(c_i, s - i).
__device__ __forceinline__ void colex_unrank(const unsigned long long* __restrict__ B,
                                             unsigned long long r, int s, int hi, int* c) {
    for (int i = s; i >= 1; --i) {
        // largest x in [i-1, hi-1] with C(x, i) <= r
        int lo = i - 1, top = hi - 1;
        while (lo < top) {
            const int mid = (lo + top + 1) >> 1;
            if (binom(B, mid, i) <= r) lo = mid; else top = mid - 1;
        }
        c[s - i] = lo;
        r -= binom(B, lo, i);
        hi = lo;
    }
}

// Rows of entry e of a list: colex (reflect=0) rows ascending after reversal, or reflected
// colex (reflect=1) rows K-1-c.  Writes rows ascending into rows[0..s-1].
__device__ __forceinline__ void list_rows(const unsigned long long* __restrict__ B,
                                          unsigned long long e, int s, int K, int reflect,
                                          int* rows) {
    int c[kMaxW];
    colex_unrank(B, e, s, K, c);
    for (int i = 0; i < s; ++i) rows[i] = reflect ? (K - 1 - c[i]) : c[s - 1 - i];
}

// ---------------------------------------------------------------- survivors
// Lexicographic rank of sorted positions (the reference's unrank order,
// cpp/qsf/combinatorics.hpp:52-61): C(K,w) - 1 - sum_i C(K-1-s_i, w-i).
static __device__ unsigned long long lex_rank(const unsigned long long* __restrict__ B,
                                       const int* s, int w, int K) {
    unsigned long long acc = 0;
    for (int i = 0; i < w; ++i) acc += binom(B, K - 1 - s[i], w - i);
    return binom(B, K, w) - 1ull - acc;
}

// Full evaluation of register entry `ereg` against the loop entries [l0, l0+ln).  Each pair
// is first re-screened on all stored probe words (a lower bound on its weight) and only
// then rebuilt from its rows.  Returns the (possibly lowered) strict bound T.
static __device__ __noinline__ int survivor_scan(const LevelDesc& D, const unsigned long long* __restrict__ B,
                                          int regX, unsigned long long xoff,
                                          unsigned long long ereg, int pc_reg,
                                          unsigned long long l0, int ln, int T) {
    const int sreg = regX ? D.a : D.b;
    const int sloop = regX ? D.b : D.a;
    const uint32_t* regbase = regX ? D.la + xoff * (unsigned long long)D.HP : D.rb;
    const uint32_t* lbase = regX ? D.rb : D.la + xoff * (unsigned long long)D.HP;
    const uint8_t* lpc = regX ? D.pcb : (D.pca ? D.pca + xoff : nullptr);
    uint32_t xr[4];
    for (int h = 0; h < D.HP; ++h) xr[h] = __ldg(regbase + ereg * D.HP + h);

    int rreg[kMaxW], rloop[kMaxW];
    if (regX) list_rows(B, xoff + ereg, D.a, D.K, 0, rreg);
    else list_rows(B, ereg, D.b, D.K, 1, rreg);
    uint32_t fr[kMaxWords], sr[kMaxWords];
    for (int h = 0; h < D.W32; ++h) fr[h] = 0u;
    for (int h = 0; h < D.SW; ++h) sr[h] = 0u;
    for (int i = 0; i < sreg; ++i) {
        const uint32_t* r = D.red + (size_t)rreg[i] * D.W32;
        for (int h = 0; h < D.W32; ++h) fr[h] ^= __ldg(r + h);
        const uint32_t* s = D.syn + (size_t)rreg[i] * D.SW;
        for (int h = 0; h < D.SW; ++h) sr[h] ^= __ldg(s + h);
    }
    for (int j = 0; j < ln; ++j) {
        const unsigned long long el = l0 + (unsigned long long)j;
        const int pcl = lpc ? (int)__ldg(lpc + el) : sloop;
        int lb = pc_reg + pcl;
        for (int h = 0; h < D.HP; ++h) lb += __popc(xr[h] ^ __ldg(lbase + el * D.HP + h));
        if (lb >= T) continue;
        if (regX) list_rows(B, el, D.b, D.K, 1, rloop);
        else list_rows(B, xoff + el, D.a, D.K, 0, rloop);
        int wt = pc_reg + pcl;
        uint32_t fl[kMaxWords];
        for (int h = 0; h < D.W32; ++h) fl[h] = 0u;
        for (int i = 0; i < sloop; ++i) {
            const uint32_t* r = D.red + (size_t)rloop[i] * D.W32;
            for (int h = 0; h < D.W32; ++h) fl[h] ^= __ldg(r + h);
        }
        for (int h = 0; h < D.W32; ++h) wt += __popc(fr[h] ^ fl[h]);
        if (wt >= T) continue;
        bool logical = D.count_all != 0;
        if (!logical) {
            uint32_t acc = 0u;
            for (int h = 0; h < D.SW; ++h) {
                uint32_t s = sr[h];
                for (int i = 0; i < sloop; ++i) s ^= __ldg(D.syn + (size_t)rloop[i] * D.SW + h);
                acc |= s;
            }
            logical = acc != 0u;
        }
        if (!logical) continue;
        // sorted positions: prefix rows (all <= p) then suffix rows (all > p)
        int pos[kMaxW];
        const int* pre = regX ? rreg : rloop;
        const int* suf = regX ? rloop : rreg;
        for (int i = 0; i < D.a; ++i) pos[i] = pre[i];
        for (int i = 0; i < D.b; ++i) pos[D.a + i] = suf[i];
        const unsigned long long rk = lex_rank(B, pos, D.w, D.K) >> D.rank_shift;
        const unsigned long long key = ((unsigned long long)(wt + 1) << kKeyWtShift) |
                                       ((unsigned long long)D.g << kKeyGShift) |
                                       (rk & kKeyRankMask);
        const unsigned long long old = atomicMin(D.key, key);
        const unsigned long long cur = old < key ? old : key;
        const int nb = (int)(cur >> kKeyWtShift);
        if (nb < T) T = nb;
    }
    return T;
}

// 4 bits -> the low bit of 4 bytes: the multiplier puts copies of the nibble 7 bits apart
// (bits 0-3, 7-10, 14-17, 21-24, no overlap, so no carries), and bit i of the nibble lands
// on bit 8i of copy i.
__device__ __forceinline__ uint32_t spread4(uint32_t nib) {
    return (nib * 0x00204081u) & 0x01010101u;
}

// 16 probe bits -> 16 int8 columns of a +-1 row: set -> +1, clear -> -1, dead (beyond the
// live columns, `live` bit clear) -> 0.  Per byte 0xFF - 0xFE * bit is 0x01 or 0xFF (no
// borrows between bytes); the live mask is applied only on the row's last chunks.
__device__ __forceinline__ uint4 pm_chunk(uint32_t bits, uint32_t live) {
    uint32_t q[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) q[n] = 0xFFFFFFFFu - 0xFEu * spread4((bits >> (4 * n)) & 0xFu);
    if (live != 0xFFFFu) {
#pragma unroll
        for (int n = 0; n < 4; ++n) q[n] &= spread4((live >> (4 * n)) & 0xFu) * 0xFFu;
    }
    return make_uint4(q[0], q[1], q[2], q[3]);
}

// One +-1 row (kPmRowBytes = 64 columns from the first two probe words), written as four
// 16-byte chunks at their 64-byte-swizzle positions (chunk c of row e at c ^ ((e >> 1) & 3)).
__device__ __forceinline__ void write_pm_row(int8_t* out, unsigned long long e, uint32_t w0,
                                             uint32_t w1, int n_live) {
    uint4* row = reinterpret_cast<uint4*>(out + e * kPmRowBytes);
    const int sw = (int)((e >> 1) & 3);
#pragma unroll
    for (int j = 0; j < 4; ++j) {              // columns [16j, 16j + 16)
        const uint32_t bits = ((j < 2 ? w0 : w1) >> (16 * (j & 1))) & 0xFFFFu;
        const int l = n_live - 16 * j;
        const uint32_t live = l >= 16 ? 0xFFFFu : (l > 0 ? (1u << l) - 1u : 0u);
        row[j ^ sw] = pm_chunk(bits, live);
    }
}

}  // namespace dev
}  // namespace qsfb
