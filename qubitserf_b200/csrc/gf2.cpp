// Host GF(2) elimination.  Pivot rules follow cpp/qsf/gf2.cpp:25-58 of the reference
// (first row >= rank with a 1 in the column, swap to `rank`, clear the column in every
// other row); the row operations are word-parallel over the packed rows.
#include "gf2.hpp"

#include <algorithm>
#include <utility>

namespace qsfb {

void Mat::swap_rows(int a, int b) {
    if (a == b) return;
    u64* ra = row(a);
    u64* rb = row(b);
    for (int i = 0; i < stride; ++i) std::swap(ra[i], rb[i]);
}

void Mat::append_row(const u64* src) {
    w.insert(w.end(), src, src + stride);
    rows += 1;
}

Mat from_dense(const u8* data, int rows, int cols) {
    Mat m(rows, cols);
    for (int i = 0; i < rows; ++i) {
        u64* r = m.row(i);
        const u8* s = data + (size_t)i * cols;
        for (int w = 0; w * 64 < cols; ++w) {
            const int hi = std::min(64, cols - w * 64);
            u64 word = 0;
            for (int j = 0; j < hi; ++j) word |= (u64)(s[w * 64 + j] & 1u) << j;
            r[w] = word;
        }
    }
    return m;
}

// One elimination step on column `col`: returns true if a pivot was placed at `rank`.
// The clearing pass is branchless (every row XORs the pivot row under a mask made from its
// bit in the column): which rows hold the bit is data, so a branch on it mispredicts about
// half the time.  S = words per row (0: any).
template <int S>
static inline bool eliminate_column_s(Mat& m, int rank, int col) {
    const int st = S > 0 ? S : m.stride;
    const int wd = col >> 6, sh = col & 63;
    u64* base = m.w.data();
    int sel = -1;
    for (int r = rank; r < m.rows; ++r)
        if ((base[(size_t)r * st + wd] >> sh) & 1u) { sel = r; break; }
    if (sel < 0) return false;
    m.swap_rows(rank, sel);
    u64* prow = base + (size_t)rank * st;
    if (S > 0) {
        u64 p[S > 0 ? S : 1];
        for (int k = 0; k < S; ++k) p[k] = prow[k];
        for (int r = 0; r < m.rows; ++r) {
            u64* row = base + (size_t)r * S;
            const u64 mask = (r == rank) ? 0ull : (0ull - ((row[wd] >> sh) & 1u));
            for (int k = 0; k < S; ++k) row[k] ^= p[k] & mask;
        }
    } else {
        for (int r = 0; r < m.rows; ++r) {
            if (r == rank) continue;
            u64* row = base + (size_t)r * st;
            const u64 mask = 0ull - ((row[wd] >> sh) & 1u);
            for (int k = 0; k < st; ++k) row[k] ^= prow[k] & mask;
        }
    }
    return true;
}

static inline bool eliminate_column(Mat& m, int rank, int col) {
    switch (m.stride) {
        case 1: return eliminate_column_s<1>(m, rank, col);
        case 2: return eliminate_column_s<2>(m, rank, col);
        case 3: return eliminate_column_s<3>(m, rank, col);
        case 4: return eliminate_column_s<4>(m, rank, col);
        default: return eliminate_column_s<0>(m, rank, col);
    }
}

// cpp/qsf/gf2.cpp:25-40
int rref(Mat& m, std::vector<int>* pivots) {
    if (pivots) pivots->clear();
    int rank = 0;
    for (int col = 0; col < m.cols && rank < m.rows; ++col) {
        if (!eliminate_column(m, rank, col)) continue;
        if (pivots) pivots->push_back(col);
        ++rank;
    }
    return rank;
}

// cpp/qsf/gf2.cpp:42-58
std::vector<int> restricted_rref(Mat& m, const std::vector<int>& cols) {
    std::vector<int> piv;
    int rank = 0;
    for (size_t ci = 0; ci < cols.size() && rank < m.rows; ++ci) {
        if (!eliminate_column(m, rank, cols[ci])) continue;
        piv.push_back(cols[ci]);
        ++rank;
    }
    return piv;
}

int drop_zero_rows(Mat& m) {
    int out = 0;
    for (int r = 0; r < m.rows; ++r) {
        if (vec_zero(m.row(r), m.stride)) continue;
        if (out != r) std::copy(m.row(r), m.row(r) + m.stride, m.row(out));
        ++out;
    }
    m.w.resize((size_t)out * m.stride);
    m.rows = out;
    return out;
}

// cpp/qsf/gf2.cpp:72-94 (canonical free-column basis)
Mat nullspace(const Mat& in) {
    Mat m = in;
    std::vector<int> piv;
    rref(m, &piv);
    const int rank = (int)piv.size();
    std::vector<char> is_piv(m.cols, 0);
    for (int p : piv) is_piv[p] = 1;
    // row of free column f: e_f plus e_{piv[r]} for every pivot row r with a 1 in column f,
    // filled row by row from the free-column bits of each pivot row
    Mat ns(m.cols - rank, m.cols);
    std::vector<int> out_of(m.cols, -1);
    std::vector<u64> freemask(m.stride, 0ull);
    int out = 0;
    for (int f = 0; f < m.cols; ++f) {
        if (is_piv[f]) continue;
        out_of[f] = out;
        ns.set(out, f, 1);
        freemask[f >> 6] |= 1ull << (f & 63);
        ++out;
    }
    for (int r = 0; r < rank; ++r) {
        const u64* row = m.row(r);
        const int p = piv[r];
        for (int w = 0; w < m.stride; ++w)
            for (u64 x = row[w] & freemask[w]; x; x &= x - 1) {
                const int f = w * 64 + __builtin_ctzll(x);
                ns.row(out_of[f])[p >> 6] |= 1ull << (p & 63);
            }
    }
    return ns;
}

bool in_span(const Mat& rm, const std::vector<int>& piv, const u64* vec) {
    std::vector<u64> t(vec, vec + rm.stride);
    for (size_t r = 0; r < piv.size(); ++r) {
        const int c = piv[r];
        if ((t[c >> 6] >> (c & 63)) & 1u) vec_xor(t.data(), rm.row((int)r), rm.stride);
    }
    return vec_zero(t.data(), rm.stride);
}

Mat transpose(const Mat& m) {
    Mat t(m.cols, m.rows);
    for (int i = 0; i < m.rows; ++i)
        for (int j = 0; j < m.cols; ++j)
            if (m.get(i, j)) t.set(j, i, 1);
    return t;
}

}  // namespace qsfb
