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

// log2(i!) and 1/i for the estimate in colex_top
static __constant__ float kLog2Fact[kBinomMaxK + 1] = {
    0.0f, 0.0f, 1.0f, 2.5849625f, 4.5849625f, 6.9068906f,
    9.4918531f, 12.299208f, 15.299208f, 18.469133f, 21.7910611f, 25.2504927f,
    28.8354552f, 32.535895f, 36.3432499f, 40.2501405f, 44.2501405f, 48.3376033f,
    52.5075283f, 56.7554558f, 61.0773839f, 65.4697013f, 69.929133f, 74.4526949f,
    79.0376574f, 83.6815136f, 88.3819533f, 93.1368408f, 97.9441958f, 102.802177f,
    107.709067f, 112.663264f, 117.663264f, 122.707658f, 127.795121f, 132.924404f,
    138.094329f, 143.303782f, 148.55171f, 153.837112f, 159.15904f, 164.516592f,
    169.908909f, 175.335174f, 180.794606f, 186.286459f, 191.810021f, 197.36461f,
    202.949572f, 208.564282f, 214.208138f, 219.880563f, 225.581003f, 231.308924f,
    237.063811f, 242.845171f, 248.652526f, 254.485416f, 260.343397f, 266.22604f,
    272.13293f, 278.063668f, 284.017864f, 289.995144f, 295.995144f};
static __constant__ float kInvK[kBinomMaxK + 1] = {
    0.0f, 1.0f, 0.5f, 0.333333333f, 0.25f, 0.2f,
    0.166666667f, 0.142857143f, 0.125f, 0.111111111f, 0.1f, 0.0909090909f,
    0.0833333333f, 0.0769230769f, 0.0714285714f, 0.0666666667f, 0.0625f, 0.0588235294f,
    0.0555555556f, 0.0526315789f, 0.05f, 0.0476190476f, 0.0454545455f, 0.0434782609f,
    0.0416666667f, 0.04f, 0.0384615385f, 0.037037037f, 0.0357142857f, 0.0344827586f,
    0.0333333333f, 0.0322580645f, 0.03125f, 0.0303030303f, 0.0294117647f, 0.0285714286f,
    0.0277777778f, 0.027027027f, 0.0263157895f, 0.0256410256f, 0.025f, 0.0243902439f,
    0.0238095238f, 0.023255814f, 0.0227272727f, 0.0222222222f, 0.0217391304f, 0.0212765957f,
    0.0208333333f, 0.0204081633f, 0.02f, 0.0196078431f, 0.0192307692f, 0.0188679245f,
    0.0185185185f, 0.0181818182f, 0.0178571429f, 0.0175438596f, 0.0172413793f, 0.0169491525f,
    0.0166666667f, 0.0163934426f, 0.0161290323f, 0.0158730159f, 0.015625f};

// The largest x in [i-1, hi-1] with C(x, i) <= r (C(i-1, i) = 0, so one exists).  A binary
// search costs ~log2(hi) dependent table reads; here C(x, i) ~ (x - (i-1)/2)^i / i! gives
// the estimate x ~ (r i!)^(1/i) + (i-1)/2, and the exact answer is within a step or two of
// it, found by walking up while C(x+1, i) <= r and down while C(x, i) > r (C is increasing
// in x on [i-1, hi-1]; saturated entries compare as larger than any r).
__device__ __forceinline__ int colex_top(const unsigned long long* __restrict__ B,
                                         unsigned long long r, int i, int hi) {
    int x;
    if (i == 1) {
        x = r < (unsigned long long)(hi - 1) ? (int)r : hi - 1;   // C(x, 1) = x
        return x;
    }
    const float g = exp2f((log2f((float)r + 1.0f) + kLog2Fact[i]) * kInvK[i]) + 0.5f * (float)(i - 1);
    x = g >= (float)(hi - 1) ? hi - 1 : (int)g;
    x = x < i - 1 ? i - 1 : x;
    while (x + 1 <= hi - 1 && binom(B, x + 1, i) <= r) ++x;
    while (x > i - 1 && binom(B, x, i) > r) --x;
    return x;
}

// Colex unrank: the r-th s-subset of [0, hi) in colex order, written largest first into
// c[0..s-1] (c[0] > c[1] > ...).  r = sum_i C(c_i, s - i).
__device__ __forceinline__ void colex_unrank(const unsigned long long* __restrict__ B,
                                             unsigned long long r, int s, int hi, int* c) {
    for (int i = s; i >= 1; --i) {
        const int x = colex_top(B, r, i, hi);   // largest x in [i-1, hi-1] with C(x, i) <= r
        c[s - i] = x;
        r -= binom(B, x, i);
        hi = x;
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
