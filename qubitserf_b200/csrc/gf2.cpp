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
        for (int j = 0; j < cols; ++j)
            if (s[j] & 1) r[j >> 6] |= 1ull << (j & 63);
    }
    return m;
}

// One elimination step on column `col`: returns true if a pivot was placed at `rank`.
static inline bool eliminate_column(Mat& m, int rank, int col) {
    const int wd = col >> 6;
    const u64 bit = 1ull << (col & 63);
    int sel = -1;
    for (int r = rank; r < m.rows; ++r)
        if (m.row(r)[wd] & bit) { sel = r; break; }
    if (sel < 0) return false;
    m.swap_rows(rank, sel);
    const u64* p = m.row(rank);
    for (int r = 0; r < m.rows; ++r)
        if (r != rank && (m.row(r)[wd] & bit)) vec_xor(m.row(r), p, m.stride);
    return true;
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
    Mat ns(m.cols - rank, m.cols);
    int out = 0;
    for (int f = 0; f < m.cols; ++f) {
        if (is_piv[f]) continue;
        ns.set(out, f, 1);
        for (int r = 0; r < rank; ++r)
            if (m.get(r, f)) ns.set(out, piv[r], 1);
        ++out;
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
