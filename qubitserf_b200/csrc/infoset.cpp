// Information-set construction.  The column partition decides the ranks, hence the BZ
// lower bound at every level; the partition algorithm therefore keeps the reference's
// steps and tie-breaking (cpp/distfind/css.cpp:258-447): greedy peel, then an augmenting
// DFS matroid partition with the same class order, element order and size sort.
#include "infoset.hpp"

#include <algorithm>
#include <functional>

namespace qsfb {

namespace {

// cpp/distfind/css.cpp:258-284
std::vector<InfoSet> greedy_sets(const Mat& code_gen) {
    std::vector<InfoSet> seq;
    const int n = code_gen.cols;
    std::vector<int> active(n);
    for (int i = 0; i < n; ++i) active[i] = i;
    Mat work = code_gen;
    while (!active.empty()) {
        std::vector<int> piv = restricted_rref(work, active);
        seq.push_back({work, (int)piv.size(), piv});
        std::vector<char> is_piv(n, 0), nonzero(n, 0);
        for (int c : piv) is_piv[c] = 1;
        for (int r = 0; r < work.rows; ++r)
            for (int c : active)
                if (work.get(r, c)) nonzero[c] = 1;
        std::vector<int> next;
        next.reserve(active.size());
        for (int c : active)
            if (!is_piv[c] && nonzero[c]) next.push_back(c);
        if (next.size() == active.size()) break;
        active.swap(next);
    }
    return seq;
}

// Express column z over the independent class `cls`: (in_span, circuit) where circuit is
// the ascending list of class columns whose XOR is z (cpp/distfind/css.cpp:316-351).
// Origins are kept as bitsets over the columns, so the reference's sorted-list symmetric
// difference becomes an XOR and the circuit is read out in ascending order.
struct Expr {
    bool in_span;
    std::vector<int> circuit;
};

struct Expresser {
    int kw = 0, nw = 0;
    std::vector<u64> bv, bo;      // basis vectors (kw words) and origins (nw words)
    std::vector<int> bpiv;
    std::vector<u64> v, o;
    Expresser(int kw_, int n) : kw(kw_), nw(words_for(n)) {}

    Expr operator()(const std::vector<int>& cls, const std::vector<u64>& col, int z,
                    bool want_circuit) {
        const size_t cap = cls.size() + 1;
        if (bpiv.size() < cap) {
            bv.resize(cap * kw);
            bo.resize(cap * nw);
            bpiv.resize(cap);
        }
        v.assign(kw, 0);
        o.assign(nw, 0);
        int nb = 0;
        auto reduce = [&]() {
            for (int b = 0; b < nb; ++b) {
                const int p = bpiv[b];
                if ((v[p >> 6] >> (p & 63)) & 1u) {
                    for (int w = 0; w < kw; ++w) v[w] ^= bv[(size_t)b * kw + w];
                    for (int w = 0; w < nw; ++w) o[w] ^= bo[(size_t)b * nw + w];
                }
            }
        };
        for (int idx : cls) {
            for (int w = 0; w < kw; ++w) v[w] = col[(size_t)idx * kw + w];
            std::fill(o.begin(), o.end(), 0);
            o[idx >> 6] |= 1ull << (idx & 63);
            reduce();
            int lb = -1;
            for (int w = 0; w < kw; ++w)
                if (v[w]) { lb = w * 64 + __builtin_ctzll(v[w]); break; }
            if (lb >= 0) {
                for (int w = 0; w < kw; ++w) bv[(size_t)nb * kw + w] = v[w];
                for (int w = 0; w < nw; ++w) bo[(size_t)nb * nw + w] = o[w];
                bpiv[nb] = lb;
                ++nb;
            }
        }
        for (int w = 0; w < kw; ++w) v[w] = col[(size_t)z * kw + w];
        std::fill(o.begin(), o.end(), 0);
        reduce();
        bool zero = true;
        for (int w = 0; w < kw; ++w)
            if (v[w]) { zero = false; break; }
        Expr e{zero, {}};
        if (zero && want_circuit)
            for (int w = 0; w < nw; ++w)
                for (u64 x = o[w]; x; x &= x - 1) e.circuit.push_back(w * 64 + __builtin_ctzll(x));
        return e;
    }
};

// cpp/distfind/css.cpp:355-409
bool matroid_partition(const Mat& code_gen, std::vector<std::vector<int>>& out) {
    const int n = code_gen.cols, K = code_gen.rows, kw = words_for(K);
    std::vector<u64> col((size_t)n * kw, 0);
    std::vector<int> nonzero, zeros;
    for (int j = 0; j < n; ++j) {
        u64* c = &col[(size_t)j * kw];
        bool nz = false;
        for (int i = 0; i < K; ++i)
            if (code_gen.get(i, j)) { c[i >> 6] |= 1ull << (i & 63); nz = true; }
        (nz ? nonzero : zeros).push_back(j);
    }
    std::vector<std::vector<int>> cls;
    std::vector<char> visited(n, 0);
    Expresser express(kw, n);
    std::function<bool(int, int)> place = [&](int z, int forbidden) -> bool {
        for (int c = 0; c < (int)cls.size(); ++c) {
            if (c == forbidden) continue;
            if (!express(cls[c], col, z, false).in_span) { cls[c].push_back(z); return true; }
        }
        for (int c = 0; c < (int)cls.size(); ++c) {
            if (c == forbidden) continue;
            Expr e = express(cls[c], col, z, true);
            if (!e.in_span) continue;
            for (int y : e.circuit) {
                if (visited[y]) continue;
                visited[y] = 1;
                std::vector<int>& v = cls[c];
                v.erase(std::find(v.begin(), v.end(), y));
                v.push_back(z);
                if (place(y, c)) return true;
                v.erase(std::find(v.begin(), v.end(), z));
                v.push_back(y);
            }
        }
        return false;
    };
    for (int z : nonzero) {
        std::fill(visited.begin(), visited.end(), 0);
        if (!place(z, -1)) cls.push_back({z});
    }
    if (cls.empty()) cls.push_back({});
    for (int j : zeros) cls[0].push_back(j);
    std::vector<char> seen(n, 0);
    int total = 0;
    for (auto& c : cls)
        for (int j : c) {
            if (seen[j]) return false;
            seen[j] = 1;
            ++total;
        }
    if (total != n) return false;
    out.swap(cls);
    return true;
}

int count_full(const std::vector<InfoSet>& s, int K) {
    int f = 0;
    for (const auto& g : s) f += (g.rank == K);
    return f;
}

std::vector<InfoSet> gamma_sequence(const Mat& code_gen) {
    const int K = code_gen.rows, n = code_gen.cols;
    std::vector<InfoSet> greedy = greedy_sets(code_gen);
    if (K == 0) return greedy;
    int nnz = 0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < K; ++i)
            if (code_gen.get(i, j)) { ++nnz; break; }
    const int max_full = nnz / K;
    const int greedy_full = count_full(greedy, K);
    if (greedy_full >= max_full || n > 200) return greedy;
    std::vector<std::vector<int>> part;
    if (!matroid_partition(code_gen, part)) return greedy;
    std::sort(part.begin(), part.end(),
              [](const std::vector<int>& a, const std::vector<int>& b) {
                  return a.size() > b.size();
              });
    std::vector<InfoSet> seq;
    for (auto& cols : part) {
        if (cols.empty()) continue;
        Mat work = code_gen;
        std::vector<int> piv = restricted_rref(work, cols);
        seq.push_back({work, (int)piv.size(), piv});
    }
    if (seq.empty() || count_full(seq, K) <= greedy_full) return greedy;
    return seq;
}

}  // namespace

std::vector<InfoSet> information_sets(const Mat& code_gen) {
    std::vector<InfoSet> seq = gamma_sequence(code_gen);
    std::stable_sort(seq.begin(), seq.end(),
                     [](const InfoSet& a, const InfoSet& b) { return a.rank > b.rank; });
    return seq;
}

}  // namespace qsfb
