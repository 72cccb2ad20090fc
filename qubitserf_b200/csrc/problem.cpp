// Problem reductions (host).  Each function states the reference lines whose semantics it
// keeps; the linear algebra is this engine's own (gf2.cpp).
#include "problem.hpp"

#include <algorithm>

namespace qsfb {

namespace {

int lowest_set(const u64* v, int stride) {
    for (int i = 0; i < stride; ++i)
        if (v[i]) return i * 64 + __builtin_ctzll(v[i]);
    return -1;
}

// Incrementally built triangular basis keyed by each row's lowest set column
// (the reducing basis of cpp/distfind/css.cpp:17-45).
struct Reducer {
    Mat rows;
    std::vector<int> piv;
    explicit Reducer(int cols) : rows(0, cols) {}
    // Branchless: whether a basis row applies is data, so a branch on it mispredicts.
    bool reduce(u64* v) const {
        const int st = rows.stride;
        const u64* base = rows.w.data();
        for (int i = 0; i < rows.rows; ++i) {
            const int p = piv[i];
            const u64 mask = 0ull - ((v[p >> 6] >> (p & 63)) & 1u);
            const u64* r = base + (size_t)i * st;
            for (int k = 0; k < st; ++k) v[k] ^= r[k] & mask;
        }
        return !vec_zero(v, st);
    }
    void add(const u64* reduced) {
        rows.append_row(reduced);
        piv.push_back(lowest_set(reduced, rows.stride));
    }
};

bool all_rows_even(const Mat& m) {
    for (int i = 0; i < m.rows; ++i)
        if (m.row_weight(i) & 1) return false;
    return true;
}

// Row of minimum weight (first on ties) -> (weight, row index); (0,-1) when empty.
std::pair<int, int> min_weight_row(const Mat& m) {
    int best = 1 << 30, arg = -1;
    for (int i = 0; i < m.rows; ++i) {
        const int w = m.row_weight(i);
        if (w < best) { best = w; arg = i; }
    }
    return arg < 0 ? std::make_pair(0, -1) : std::make_pair(best, arg);
}

Mat dot_matrix(const Mat& A, const Mat& B) {
    Mat E(A.rows, B.rows);
    for (int i = 0; i < A.rows; ++i)
        for (int j = 0; j < B.rows; ++j)
            if (vec_dot(A.row(i), B.row(j), A.stride)) E.set(i, j, 1);
    return E;
}

Mat rows_combine(const Mat& C, const Mat& B) {
    Mat out(C.rows, B.cols);
    for (int i = 0; i < C.rows; ++i)
        for (int j = 0; j < B.rows; ++j)
            if (C.get(i, j)) vec_xor(out.row(i), B.row(j), B.stride);
    return out;
}

// cpp/distfind/css.cpp:78-87
Problem build(const Mat& Hself, const Mat& Hother) {
    Problem p;
    p.n = Hself.cols;
    p.code_gen = nullspace(Hself);
    p.check = quotient_basis(Hself, Hother);
    Mat logicals = quotient_basis(Hother, Hself);
    p.even = all_rows_even(p.code_gen);
    auto mw = min_weight_row(logicals);
    p.seed_upper = mw.first;
    if (mw.second >= 0)
        p.seed_word.assign(logicals.row(mw.second), logicals.row(mw.second) + logicals.stride);
    return p;
}

std::vector<u64> pack_bytes(const u8* vec, int n) {
    std::vector<u64> v(words_for(n), 0);
    for (int j = 0; j < n; ++j)
        if (vec[j] & 1) v[j >> 6] |= 1ull << (j & 63);
    return v;
}

}  // namespace

namespace {
// Rows of ko = nullspace(other) independent of rowspan(self) (cpp/distfind/css.cpp:94-105).
Mat quotient_of(const Mat& self, const Mat& ko) {
    Reducer basis(self.cols);
    std::vector<u64> t(std::max(1, self.stride));
    for (int i = 0; i < self.rows; ++i) {
        std::copy(self.row(i), self.row(i) + self.stride, t.begin());
        if (basis.reduce(t.data())) basis.add(t.data());
    }
    Mat out(0, self.cols);
    for (int i = 0; i < ko.rows; ++i) {
        std::copy(ko.row(i), ko.row(i) + ko.stride, t.begin());
        if (!basis.reduce(t.data())) continue;
        basis.add(t.data());
        out.append_row(ko.row(i));
    }
    return out;
}

Problem from_parts(int n, Mat code_gen, Mat check, const Mat& logicals) {
    Problem p;
    p.n = n;
    p.code_gen = std::move(code_gen);
    p.check = std::move(check);
    p.even = all_rows_even(p.code_gen);
    auto mw = min_weight_row(logicals);
    p.seed_upper = mw.first;
    if (mw.second >= 0)
        p.seed_word.assign(logicals.row(mw.second), logicals.row(mw.second) + logicals.stride);
    return p;
}
}  // namespace

std::pair<Problem, Problem> css_problem_pair(const Mat& Hx, const Mat& Hz) {
    Mat nx = nullspace(Hx), nz = nullspace(Hz);
    Mat qxz = quotient_of(Hx, nz);   // quotient_basis(Hx, Hz): Z detector, X logicals
    Mat qzx = quotient_of(Hz, nx);   // quotient_basis(Hz, Hx): X detector, Z logicals
    Problem pz = from_parts(Hx.cols, nx, qxz, qzx);
    Problem px = from_parts(Hz.cols, nz, qzx, qxz);
    return {std::move(pz), std::move(px)};
}

Mat quotient_basis(const Mat& self, const Mat& other) {
    Mat ko = nullspace(other);
    Reducer basis(self.cols);
    for (int i = 0; i < self.rows; ++i) {
        std::vector<u64> t(self.row(i), self.row(i) + self.stride);
        if (basis.reduce(t.data())) basis.add(t.data());
    }
    Mat out(0, self.cols);
    for (int i = 0; i < ko.rows; ++i) {
        std::vector<u64> t(ko.row(i), ko.row(i) + ko.stride);
        if (!basis.reduce(t.data())) continue;
        basis.add(t.data());
        out.append_row(ko.row(i));
    }
    return out;
}

Problem css_problem(const Mat& Hx, const Mat& Hz, char which) {
    return which == 'X' ? build(Hz, Hx) : build(Hx, Hz);
}

Problem classical_problem(const Mat& H) {
    Problem p;
    p.n = H.cols;
    p.code_gen = nullspace(H);
    p.check = Mat(0, H.cols);
    p.count_all = true;
    p.even = all_rows_even(p.code_gen);
    auto mw = min_weight_row(p.code_gen);
    p.seed_upper = mw.first;
    if (mw.second >= 0)
        p.seed_word.assign(p.code_gen.row(mw.second),
                           p.code_gen.row(mw.second) + p.code_gen.stride);
    return p;
}

std::pair<Mat, Mat> css_center(const Mat& Gx, const Mat& Gz) {
    Mat E = dot_matrix(Gx, Gz);
    Mat Sx = rows_combine(nullspace(transpose(E)), Gx);
    rref(Sx);
    drop_zero_rows(Sx);
    Mat Sz = rows_combine(nullspace(E), Gz);
    rref(Sz);
    drop_zero_rows(Sz);
    return {Sx, Sz};
}

Problem subsystem_problem(const Mat& Gx, const Mat& Gz, char which) {
    auto c = css_center(Gx, Gz);
    return which == 'X' ? build(c.second, Gx) : build(c.first, Gz);
}

bool in_rowspace(const Mat& G, const u8* vec) {
    Mat R = G;
    std::vector<int> piv;
    rref(R, &piv);
    std::vector<u64> v = pack_bytes(vec, G.cols);
    return in_span(R, piv, v.data());
}

Problem coset_problem(const Mat& G, const u8* vec) {
    Problem p;
    const int n = G.cols;
    p.n = n;
    Mat M(G.rows + 1, n);
    for (int i = 0; i < G.rows; ++i) vec_xor(M.row(i), G.row(i), G.stride);
    std::vector<u64> v = pack_bytes(vec, n);
    vec_xor(M.row(G.rows), v.data(), M.stride);
    rref(M);
    drop_zero_rows(M);
    p.code_gen = M;
    Mat N = nullspace(G);
    Mat check(0, n);
    for (int i = 0; i < N.rows; ++i)
        if (vec_dot(N.row(i), v.data(), N.stride)) { check.append_row(N.row(i)); break; }
    p.check = check;
    p.even = all_rows_even(p.code_gen);
    p.seed_upper = vec_weight(v.data(), (int)v.size());
    p.seed_word = v;
    return p;
}

Mat symplectic_swap(const Mat& m) {
    const int q = m.cols / 2;
    Mat out(m.rows, m.cols);
    for (int i = 0; i < m.rows; ++i)
        for (int j = 0; j < q; ++j) {
            if (m.get(i, j)) out.set(i, q + j, 1);
            if (m.get(i, q + j)) out.set(i, j, 1);
        }
    return out;
}

int symplectic_row_weight(const u64* row, int q) {
    int w = 0;
    for (int j = 0; j < q; ++j) {
        const int z = (int)((row[j >> 6] >> (j & 63)) & 1u);
        const int xj = q + j;
        const int x = (int)((row[xj >> 6] >> (xj & 63)) & 1u);
        w += (z | x);
    }
    return w;
}

bool is_css_symplectic(const Mat& S) {
    const int q = S.cols / 2;
    for (int i = 0; i < S.rows; ++i) {
        bool hz = false, hx = false;
        for (int j = 0; j < q; ++j) {
            hz |= S.get(i, j) != 0;
            hx |= S.get(i, q + j) != 0;
        }
        if (hz && hx) return false;
    }
    return true;
}

std::pair<Mat, Mat> split_css(const Mat& S) {
    const int q = S.cols / 2;
    Mat Hx(0, q), Hz(0, q);
    Mat zr(1, q), xr(1, q);
    for (int i = 0; i < S.rows; ++i) {
        std::fill(zr.w.begin(), zr.w.end(), 0);
        std::fill(xr.w.begin(), xr.w.end(), 0);
        bool hz = false, hx = false;
        for (int j = 0; j < q; ++j) {
            if (S.get(i, j)) { zr.set(0, j, 1); hz = true; }
            if (S.get(i, q + j)) { xr.set(0, j, 1); hx = true; }
        }
        if (hx) Hx.append_row(xr.row(0));
        else if (hz) Hz.append_row(zr.row(0));
    }
    return {Hx, Hz};
}

Mat symplectic_center(const Mat& G) {
    Mat gram = dot_matrix(G, symplectic_swap(G));
    Mat C = rows_combine(nullspace(gram), G);
    rref(C);
    drop_zero_rows(C);
    return C;
}

// cpp/distfind/stab.cpp:98-132
Problem symplectic_problem(const Mat& Snorm, const Mat& Gtriv) {
    Problem p;
    p.symplectic = true;
    p.n = Snorm.cols;
    p.qubits = Snorm.cols / 2;
    p.code_gen = nullspace(symplectic_swap(Snorm));
    Mat L = quotient_basis(Snorm, symplectic_swap(Gtriv));
    p.check = symplectic_swap(L);
    p.even = false;
    p.count_all = false;
    int best = 0, arg = -1;
    std::vector<u8> bytes(p.n);
    for (int i = 0; i < p.code_gen.rows; ++i) {
        for (int j = 0; j < p.n; ++j) bytes[j] = (u8)p.code_gen.get(i, j);
        if (in_rowspace(Gtriv, bytes.data())) continue;
        const int w = symplectic_row_weight(p.code_gen.row(i), p.qubits);
        if (best == 0 || w < best) { best = w; arg = i; }
    }
    p.seed_upper = best;
    if (arg >= 0)
        p.seed_word.assign(p.code_gen.row(arg), p.code_gen.row(arg) + p.code_gen.stride);
    return p;
}

Problem symplectic_coset_problem(const Mat& G, const u8* op) {
    Problem p = coset_problem(G, op);
    p.symplectic = true;
    p.qubits = G.cols / 2;
    std::vector<u64> v = pack_bytes(op, G.cols);
    p.seed_upper = symplectic_row_weight(v.data(), p.qubits);
    p.seed_word = v;
    return p;
}

namespace {
std::vector<u64> phi_row(const u64* r, int q) {
    std::vector<u64> o(words_for(3 * q), 0);
    for (int j = 0; j < q; ++j) {
        const int a = (int)((r[j >> 6] >> (j & 63)) & 1u);
        const int xj = q + j;
        const int b = (int)((r[xj >> 6] >> (xj & 63)) & 1u);
        if (a) o[j >> 6] |= 1ull << (j & 63);
        if (b) o[xj >> 6] |= 1ull << (xj & 63);
        if (a ^ b) {
            const int t = 2 * q + j;
            o[t >> 6] |= 1ull << (t & 63);
        }
    }
    return o;
}
}  // namespace

Problem isometry_extend(const Problem& sp) {
    const int q = sp.qubits;
    Problem e;
    e.symplectic = false;
    e.qubits = 0;
    e.n = 3 * q;
    e.even = true;
    e.count_all = sp.count_all;
    e.seed_upper = sp.seed_upper > 0 ? 2 * sp.seed_upper : 0;
    if (!sp.seed_word.empty()) e.seed_word = phi_row(sp.seed_word.data(), q);
    e.code_gen = Mat(sp.code_gen.rows, e.n);
    for (int i = 0; i < sp.code_gen.rows; ++i) {
        std::vector<u64> r = phi_row(sp.code_gen.row(i), q);
        std::copy(r.begin(), r.end(), e.code_gen.row(i));
    }
    e.check = Mat(sp.check.rows, e.n);
    for (int i = 0; i < sp.check.rows; ++i)
        for (int j = 0; j < sp.n; ++j)
            if (sp.check.get(i, j)) e.check.set(i, j, 1);
    return e;
}

bool verify_witness(const Problem& p, const u64* c, int weight) {
    const int stride = words_for(p.n);
    if (vec_weight(c, stride) != weight) return false;
    Mat R = p.code_gen;
    std::vector<int> piv;
    rref(R, &piv);
    if (!in_span(R, piv, c)) return false;
    if (p.count_all) return !vec_zero(c, stride);
    for (int i = 0; i < p.check.rows; ++i)
        if (vec_dot(p.check.row(i), c, stride)) return true;
    return false;
}

}  // namespace qsfb
