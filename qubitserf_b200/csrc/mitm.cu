// sm_100a kernels of the meet-in-the-middle distance (method "mitm"): the parts of one
// coordinate half and their syndromes, the hash table of the left parts and the probe of
// the right parts (mitm_types.hpp).
//
// Semantics kept from the reference (cpp/distfind/mitm.cpp:95-316): a part of weight w is a
// w-subset of the half's coordinates (symplectic: of its qubits, with one of Z, X, Y on
// each); its syndrome is the XOR of the parity check's columns over the part, its logical
// fingerprint the XOR of the detector's columns; a level hits when a left and a right part
// share a syndrome and (count_all or) differ in fingerprint.  The reference hashes the left
// parts on the host (std::unordered_map) and probes with threads; here both sides are
// generated on the device, one part per thread, and the table is exact: a 64-bit tag claims
// a slot, the full syndrome is compared before any match counts, and two syndromes that
// share a tag are reported so that the host rebuilds with another seed.
//
// Every loop over the table is bounded by its size; no kernel waits on another thread.
#include <cuda_runtime.h>
#include <cstdint>

#include "engine_types.hpp"
#include "enum_device.cuh"
#include "mitm_types.hpp"

namespace qsfb {
namespace dev {

// Syndrome and fingerprint of part `id` of weight w over coordinates [first, first + count).
// Bits: id is the colex rank of the coordinate subset.  Symplectic: id = rank * 3^w + p,
// the base-3 digits of p choosing Z (0), X (1) or Y (2) on each qubit of the subset.
__device__ __forceinline__ void part_words(const MitmShared& S, const unsigned long long* B,
                                           unsigned long long id, int first, int count, int w,
                                           unsigned long long pw3,
                                           uint32_t (&syn)[kMitmMaxSynWords],
                                           uint32_t (&lg)[kMitmMaxLogWords]) {
#pragma unroll
    for (int k = 0; k < kMitmMaxSynWords; ++k) syn[k] = 0u;
#pragma unroll
    for (int k = 0; k < kMitmMaxLogWords; ++k) lg[k] = 0u;
    unsigned long long rank = id, pauli = 0;
    if (S.sym) { rank = id / pw3; pauli = id - rank * pw3; }
    int c[kMitmMaxWeight];
    colex_unrank(B, rank, w, count, c);
    auto add_col = [&](int col) {
        const uint32_t* sp = S.syn_cols + (size_t)col * S.SW;
#pragma unroll
        for (int k = 0; k < kMitmMaxSynWords; ++k)
            if (k < S.SW) syn[k] ^= __ldg(sp + k);
        const uint32_t* lp = S.log_cols + (size_t)col * S.LW;
#pragma unroll
        for (int k = 0; k < kMitmMaxLogWords; ++k)
            if (k < S.LW) lg[k] ^= __ldg(lp + k);
    };
    for (int i = 0; i < w; ++i) {
        const int coord = first + c[i];
        if (!S.sym) {
            add_col(coord);
        } else {
            const int digit = (int)(pauli % 3ull);
            pauli /= 3ull;
            if (digit != 1) add_col(coord);              // Z or Y: the z column
            if (digit != 0) add_col(S.qubits + coord);   // X or Y: the x column
        }
    }
}

__device__ __forceinline__ unsigned long long syn_hash(const uint32_t (&syn)[kMitmMaxSynWords],
                                                       int SW, unsigned long long seed) {
    unsigned long long h = seed ^ 0x243f6a8885a308d3ull;
#pragma unroll
    for (int k = 0; k < kMitmMaxSynWords; ++k) {
        if (k < SW) {
            h ^= syn[k];
            h *= 0x9e3779b97f4a7c15ull;
            h ^= h >> 29;
        }
    }
    h ^= h >> 32;
    h *= 0xd6e8feb86659fd93ull;
    h ^= h >> 32;
    return h;
}

constexpr int kMitmRun = 8;   // consecutive parts per thread

// Walk parts [id0, id0 + cnt) of weight w over coordinates [first, first + count), calling
// f(syn, lg) for each.  Bit parts of a half of at most 64 coordinates keep the subset as a
// 64-bit mask: the first is unranked into it, the next follow by the colex successor (the
// next integer of the same popcount) and only the columns of the bits that flip are XORed
// in.  Other parts (symplectic, or wider halves) are unranked one by one.
template <class F>
__device__ __forceinline__ void for_run(const MitmShared& S, const unsigned long long* B,
                                        unsigned long long id0, int cnt, int first, int count,
                                        int w, unsigned long long pw3, F&& f) {
    uint32_t syn[kMitmMaxSynWords], lg[kMitmMaxLogWords];
    if (S.sym || count > 64) {
        for (int j = 0; j < cnt; ++j) {
            part_words(S, B, id0 + j, first, count, w, pw3, syn, lg);
            f(syn, lg);
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < kMitmMaxSynWords; ++k) syn[k] = 0u;
#pragma unroll
    for (int k = 0; k < kMitmMaxLogWords; ++k) lg[k] = 0u;
    unsigned long long x = 0ull;
    {
        unsigned long long r = id0;
        int hi = count;
        for (int i = w; i >= 1; --i) {   // colex unrank, largest element first
            int lo = i - 1, top = hi - 1;
            while (lo < top) {
                const int mid = (lo + top + 1) >> 1;
                if (binom(B, mid, i) <= r) lo = mid; else top = mid - 1;
            }
            x |= 1ull << lo;
            r -= binom(B, lo, i);
            hi = lo;
        }
    }
    auto flip = [&](unsigned long long d) {
        while (d) {
            const int b = __ffsll((long long)d) - 1;
            d &= d - 1;
            const uint32_t* sp = S.syn_cols + (size_t)(first + b) * S.SW;
#pragma unroll
            for (int k = 0; k < kMitmMaxSynWords; ++k)
                if (k < S.SW) syn[k] ^= __ldg(sp + k);
            const uint32_t* lp = S.log_cols + (size_t)(first + b) * S.LW;
#pragma unroll
            for (int k = 0; k < kMitmMaxLogWords; ++k)
                if (k < S.LW) lg[k] ^= __ldg(lp + k);
        }
    };
    flip(x);
    for (int j = 0; j < cnt; ++j) {
        f(syn, lg);
        if (j + 1 == cnt) break;
        const int p = __ffsll((long long)x) - 1;
        const unsigned long long v = x + (1ull << p);
        const unsigned long long next = v | (p + 2 < 64 ? ((v ^ x) >> (p + 2)) : 0ull);
        flip(x ^ next);
        x = next;
    }
}

// Pass 1: every left part claims the slot of its tag (first empty slot on its probe
// sequence, or the slot its tag already owns) and the claimer writes syndrome + fingerprint.
__global__ void __launch_bounds__(256) mitm_claim_kernel(MitmShared S, MitmTable T, int first,
                                                         int count, int w, unsigned long long n,
                                                         unsigned long long pw3,
                                                         const unsigned long long* __restrict__ B) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long runs = (n + kMitmRun - 1) / kMitmRun;
    const int KW = S.SW + S.LW;
    for (unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         r < runs; r += stride) {
        const unsigned long long id0 = r * kMitmRun;
        const int cnt = (int)(n - id0 < (unsigned long long)kMitmRun ? n - id0 : kMitmRun);
        for_run(S, B, id0, cnt, first, count, w, pw3,
                [&](const uint32_t (&syn)[kMitmMaxSynWords], const uint32_t (&lg)[kMitmMaxLogWords]) {
            const unsigned long long h = syn_hash(syn, S.SW, T.seed);
            const unsigned long long tg = (h & T.tag_mask) | 1ull;
            unsigned long long slot = h & T.mask;
            bool placed = false;
            for (unsigned long long it = 0; it <= T.mask; ++it) {
                const unsigned long long old = atomicCAS(T.tag + slot, 0ull, tg);
                if (old == 0ull) {
                    uint32_t* k = T.key + slot * (unsigned long long)KW;
#pragma unroll
                    for (int q = 0; q < kMitmMaxSynWords; ++q)
                        if (q < S.SW) k[q] = syn[q];
#pragma unroll
                    for (int q = 0; q < kMitmMaxLogWords; ++q)
                        if (q < S.LW) k[S.SW + q] = lg[q];
                    placed = true;
                    break;
                }
                if (old == tg) { placed = true; break; }
                slot = (slot + 1) & T.mask;
            }
            if (!placed) atomicOr(S.status + kMitmOverrun, 1);
        });
    }
}

// Pass 2 (after pass 1 has finished): every left part finds its tag's slot, checks that the
// stored syndrome is its own (else two syndromes share the tag) and marks the bucket when its
// fingerprint differs from the stored one.
__global__ void __launch_bounds__(256) mitm_verify_kernel(MitmShared S, MitmTable T, int first,
                                                          int count, int w, unsigned long long n,
                                                          unsigned long long pw3,
                                                          const unsigned long long* __restrict__ B) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long runs = (n + kMitmRun - 1) / kMitmRun;
    const int KW = S.SW + S.LW;
    for (unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         r < runs; r += stride) {
        const unsigned long long id0 = r * kMitmRun;
        const int cnt = (int)(n - id0 < (unsigned long long)kMitmRun ? n - id0 : kMitmRun);
        for_run(S, B, id0, cnt, first, count, w, pw3,
                [&](const uint32_t (&syn)[kMitmMaxSynWords], const uint32_t (&lg)[kMitmMaxLogWords]) {
            const unsigned long long h = syn_hash(syn, S.SW, T.seed);
            const unsigned long long tg = (h & T.tag_mask) | 1ull;
            unsigned long long slot = h & T.mask;
            bool seen = false;
            for (unsigned long long it = 0; it <= T.mask; ++it) {
                const unsigned long long t = T.tag[slot];
                if (t == tg) { seen = true; break; }
                if (t == 0ull) break;
                slot = (slot + 1) & T.mask;
            }
            if (!seen) { atomicOr(S.status + kMitmOverrun, 1); return; }
            const uint32_t* k = T.key + slot * (unsigned long long)KW;
            bool same = true;
#pragma unroll
            for (int q = 0; q < kMitmMaxSynWords; ++q)
                if (q < S.SW) same = same && (k[q] == syn[q]);
            if (!same) { atomicOr(S.status + kMitmCollision, 1); return; }
            bool diff = false;
#pragma unroll
            for (int q = 0; q < kMitmMaxLogWords; ++q)
                if (q < S.LW) diff = diff || (k[S.SW + q] != lg[q]);
            if (diff && (T.flags[slot] & 1u) == 0u) atomicOr(T.flags + slot, 1u);
        });
    }
}

// Probe: every right part looks up its syndrome; a match is a hit when the problem counts
// every codeword, the bucket holds two fingerprints, or the stored one differs from its own.
__global__ void __launch_bounds__(256) mitm_probe_kernel(MitmShared S, MitmTable T, int first,
                                                         int count, int w, unsigned long long n,
                                                         unsigned long long pw3, int count_all,
                                                         const unsigned long long* __restrict__ B) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long runs = (n + kMitmRun - 1) / kMitmRun;
    const int KW = S.SW + S.LW;
    volatile int* found = S.status + kMitmFound;
    for (unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         r < runs; r += stride) {
        if (*found) return;   // the level already hit
        const unsigned long long id0 = r * kMitmRun;
        const int cnt = (int)(n - id0 < (unsigned long long)kMitmRun ? n - id0 : kMitmRun);
        for_run(S, B, id0, cnt, first, count, w, pw3,
                [&](const uint32_t (&syn)[kMitmMaxSynWords], const uint32_t (&lg)[kMitmMaxLogWords]) {
            const unsigned long long h = syn_hash(syn, S.SW, T.seed);
            const unsigned long long tg = (h & T.tag_mask) | 1ull;
            unsigned long long slot = h & T.mask;
            for (unsigned long long it = 0; it <= T.mask; ++it) {
                const unsigned long long t = T.tag[slot];
                if (t == 0ull) return;
                if (t == tg) {
                    // the only slot this syndrome can own: a left part with the same syndrome
                    // but another slot would have joined this one and been reported
                    const uint32_t* k = T.key + slot * (unsigned long long)KW;
                    bool same = true;
#pragma unroll
                    for (int q = 0; q < kMitmMaxSynWords; ++q)
                        if (q < S.SW) same = same && (k[q] == syn[q]);
                    if (!same) return;
                    bool hit = count_all != 0 || (T.flags[slot] & 1u) != 0u;
#pragma unroll
                    for (int q = 0; q < kMitmMaxLogWords; ++q)
                        if (q < S.LW) hit = hit || (k[S.SW + q] != lg[q]);
                    if (hit) atomicExch(S.status + kMitmFound, 1);
                    return;
                }
                slot = (slot + 1) & T.mask;
            }
            atomicOr(S.status + kMitmOverrun, 1);
        });
    }
}

}  // namespace dev

namespace {
unsigned int grid_for(unsigned long long n, int num_sms) {
    const unsigned long long runs = (n + dev::kMitmRun - 1) / dev::kMitmRun;
    const unsigned long long want = (runs + 255) / 256;
    const unsigned long long cap = (unsigned long long)num_sms * 16;
    return (unsigned int)(want < cap ? (want > 0 ? want : 1) : cap);
}
}  // namespace

cudaError_t launch_mitm_build(const MitmShared& S, const MitmTable& T, int first, int count,
                              int w, unsigned long long n, unsigned long long pw3,
                              const unsigned long long* d_binom, int num_sms, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const unsigned int g = grid_for(n, num_sms);
    dev::mitm_claim_kernel<<<g, 256, 0, st>>>(S, T, first, count, w, n, pw3, d_binom);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dev::mitm_verify_kernel<<<g, 256, 0, st>>>(S, T, first, count, w, n, pw3, d_binom);
    return cudaGetLastError();
}

cudaError_t launch_mitm_probe(const MitmShared& S, const MitmTable& T, int first, int count,
                              int w, unsigned long long n, unsigned long long pw3, int count_all,
                              const unsigned long long* d_binom, int num_sms, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    dev::mitm_probe_kernel<<<grid_for(n, num_sms), 256, 0, st>>>(S, T, first, count, w, n, pw3,
                                                                 count_all, d_binom);
    return cudaGetLastError();
}

}  // namespace qsfb
