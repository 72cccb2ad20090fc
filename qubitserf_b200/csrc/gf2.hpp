// Host-side bit-packed GF(2) linear algebra for the B200 BZ engine.
//
// Row format (shared with the reference's cpp/qsf/bits.hpp:1-3 so matrices cross the
// C ABI unchanged): a row is `stride = ceil(cols/64)` little-endian uint64 words, bit j
// in word j>>6 at offset j&63.
//
// The elimination routines make the SAME pivot choices as the reference
// (cpp/qsf/gf2.cpp:25-58): pivot = first row at or below the current rank holding a 1 in
// the next listed column, swapped into position `rank`, then XORed into every other row
// with a 1 there.  Those choices fix the information-set generator matrices, so keeping
// them identical is what makes the per-(information set, weight) enumeration and the
// returned witness reproducible against the reference.
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>

namespace qsfb {

using u64 = std::uint64_t;
using u32 = std::uint32_t;
using u8 = std::uint8_t;

inline int words_for(int bits) { return (bits + 63) >> 6; }
inline int popc64(u64 x) { return __builtin_popcountll(x); }

inline int vec_weight(const u64* v, int stride) {
    int w = 0;
    for (int i = 0; i < stride; ++i) w += popc64(v[i]);
    return w;
}
inline void vec_or(u64* d, const u64* s, int stride) {
    for (int i = 0; i < stride; ++i) d[i] |= s[i];
}
inline void vec_xor(u64* d, const u64* s, int stride) {
    for (int i = 0; i < stride; ++i) d[i] ^= s[i];
}
inline int vec_dot(const u64* a, const u64* b, int stride) {
    u64 acc = 0;
    for (int i = 0; i < stride; ++i) acc ^= a[i] & b[i];
    return popc64(acc) & 1;
}
inline bool vec_zero(const u64* v, int stride) {
    for (int i = 0; i < stride; ++i)
        if (v[i]) return false;
    return true;
}

// Dense row-major bit-packed matrix over GF(2).
struct Mat {
    int rows = 0, cols = 0, stride = 0;
    std::vector<u64> w;

    Mat() = default;
    Mat(int r, int c) : rows(r), cols(c), stride(words_for(c)), w((size_t)r * words_for(c), 0) {}

    u64* row(int i) { return w.data() + (size_t)i * stride; }
    const u64* row(int i) const { return w.data() + (size_t)i * stride; }
    int get(int i, int j) const { return (int)((row(i)[j >> 6] >> (j & 63)) & 1u); }
    void set(int i, int j, int v) {
        u64 m = 1ull << (j & 63);
        if (v) row(i)[j >> 6] |= m; else row(i)[j >> 6] &= ~m;
    }
    int row_weight(int i) const { return vec_weight(row(i), stride); }
    void swap_rows(int a, int b);
    void append_row(const u64* src);
};

Mat from_dense(const u8* data, int rows, int cols);

// RREF over all columns in order; returns the rank, optional pivot list.
int rref(Mat& m, std::vector<int>* pivots = nullptr);
// RREF restricted to the listed columns (in that order) with full-width row operations;
// returns the pivot columns.  Pivot i ends in row i.
std::vector<int> restricted_rref(Mat& m, const std::vector<int>& cols);
int drop_zero_rows(Mat& m);
// Canonical basis of {x : m x^T = 0}: one row per free column (ascending), with the
// pivot coordinates read from the RREF column.
Mat nullspace(const Mat& m);
bool in_span(const Mat& rref_m, const std::vector<int>& pivots, const u64* vec);
Mat transpose(const Mat& m);

}  // namespace qsfb
