// Information-set construction.  The column partition decides the ranks, hence the BZ
// lower bound at every level; the partition algorithm therefore keeps the reference's
// steps and tie-breaking (cpp/distfind/css.cpp:177-366): greedy peel, then an augmenting
// DFS matroid partition with the same class order, element order and size sort.
#include "infoset.hpp"

#include <algorithm>
#include <functional>

namespace qsfb {

namespace {

// cpp/distfind/css.cpp:177-203
std::vector<InfoSet> greedy_sets(const Mat& code_gen) {
    std::vector<InfoSet> seq;
    const int n = code_gen.cols;
    std::vector<int> active(n);
    for (int i = 0; i < n; ++i) active[i] = i;
    Mat work = code_gen;
    while (!active.empty()) {
        std::vector<int> piv = restricted_rref(work, active);
        seq.push_back({work, (int)piv.size(), piv});
        std::vector<char> is_piv(n, 0);
        for (int c : piv) is_piv[c] = 1;
        // columns holding a 1 in some row: the OR of the rows
        std::vector<u64> any(work.stride, 0ull);
        for (int r = 0; r < work.rows; ++r) vec_or(any.data(), work.row(r), work.stride);
        std::vector<int> next;
        next.reserve(active.size());
        for (int c : active)
            if (!is_piv[c] && ((any[c >> 6] >> (c & 63)) & 1u)) next.push_back(c);
        if (next.size() == active.size()) break;
        active.swap(next);
    }
    return seq;
}

// Express column z over the independent class `cls`: (in_span, circuit) where circuit is
// the ascending list of class columns whose XOR is z (cpp/distfind/css.cpp:232-266).
// Origins are kept as bitsets over the columns, so the reference's sorted-list symmetric
// difference becomes an XOR and the circuit is read out in ascending order.  A class is
// independent, so both answers are unique whatever order its columns are inserted in:
// each class keeps its reduced basis between queries (extended when a column is appended,
// rebuilt after the augmenting path swaps columns) instead of rebuilding it per query.
struct Expr {
    bool in_span;
    std::vector<int> circuit;
};

struct ClassBasis {
    std::vector<u64> bv, bo;      // basis vectors (kw words) and origins (nw words)
    std::vector<int> bpiv;        // pivot (lowest set bit) of each basis vector
    int nb = 0;
    bool valid = false;
};

struct Expresser {
    int kw = 0, nw = 0;
    const std::vector<u64>* col = nullptr;
    std::vector<u64> v, o;
    Expresser(int kw_, int n, const std::vector<u64>* c) : kw(kw_), nw(words_for(n)), col(c) {}

    // v, o reduced against the basis: every pivot bit cleared, in insertion order
    void reduce(const ClassBasis& B) {
        for (int b = 0; b < B.nb; ++b) {
            const int p = B.bpiv[b];
            if ((v[p >> 6] >> (p & 63)) & 1u) {
                for (int w = 0; w < kw; ++w) v[w] ^= B.bv[(size_t)b * kw + w];
                for (int w = 0; w < nw; ++w) o[w] ^= B.bo[(size_t)b * nw + w];
            }
        }
    }
    void load(int z) {
        v.assign(col->begin() + (size_t)z * kw, col->begin() + (size_t)(z + 1) * kw);
        o.assign(nw, 0);
    }
    // append the reduced (v, o) as a basis vector when nonzero
    void push(ClassBasis& B) {
        int lb = -1;
        for (int w = 0; w < kw; ++w)
            if (v[w]) { lb = w * 64 + __builtin_ctzll(v[w]); break; }
        if (lb < 0) return;
        B.bv.insert(B.bv.end(), v.begin(), v.end());
        B.bo.insert(B.bo.end(), o.begin(), o.end());
        B.bpiv.push_back(lb);
        ++B.nb;
    }
    void build(ClassBasis& B, const std::vector<int>& cls) {
        B.bv.clear(); B.bo.clear(); B.bpiv.clear(); B.nb = 0;
        for (int idx : cls) {
            load(idx);
            o[idx >> 6] |= 1ull << (idx & 63);
            reduce(B);
            push(B);
        }
        B.valid = true;
    }
    Expr query(ClassBasis& B, const std::vector<int>& cls, int z, bool want_circuit) {
        if (!B.valid) build(B, cls);
        load(z);
        reduce(B);
        bool zero = true;
        for (int w = 0; w < kw; ++w)
            if (v[w]) { zero = false; break; }
        Expr e{zero, {}};
        if (zero && want_circuit)
            for (int w = 0; w < nw; ++w)
                for (u64 x = o[w]; x; x &= x - 1) e.circuit.push_back(w * 64 + __builtin_ctzll(x));
        return e;
    }
    // z was just queried against B (not in its span) and appended to the class
    void append_queried(ClassBasis& B, int z) {
        o[z >> 6] ^= 1ull << (z & 63);
        push(B);
    }
};

// cpp/distfind/css.cpp:274-328
bool matroid_partition(const Mat& code_gen, std::vector<std::vector<int>>& out) {
    const int n = code_gen.cols, K = code_gen.rows, kw = words_for(K);
    // columns as bit vectors over the rows (transpose by the set bits of each row)
    std::vector<u64> col((size_t)n * kw, 0);
    for (int i = 0; i < K; ++i) {
        const u64* r = code_gen.row(i);
        for (int w = 0; w < code_gen.stride; ++w)
            for (u64 x = r[w]; x; x &= x - 1) {
                const int j = w * 64 + __builtin_ctzll(x);
                col[(size_t)j * kw + (i >> 6)] |= 1ull << (i & 63);
            }
    }
    std::vector<int> nonzero, zeros;
    for (int j = 0; j < n; ++j) {
        const u64* c = &col[(size_t)j * kw];
        bool nz = false;
        for (int w = 0; w < kw; ++w) nz = nz || c[w] != 0;
        (nz ? nonzero : zeros).push_back(j);
    }
    std::vector<std::vector<int>> cls;
    std::vector<ClassBasis> basis;
    std::vector<char> visited(n, 0);
    Expresser express(kw, n, &col);
    std::function<bool(int, int)> place = [&](int z, int forbidden) -> bool {
        for (int c = 0; c < (int)cls.size(); ++c) {
            if (c == forbidden) continue;
            if (!express.query(basis[c], cls[c], z, false).in_span) {
                cls[c].push_back(z);
                express.append_queried(basis[c], z);
                return true;
            }
        }
        for (int c = 0; c < (int)cls.size(); ++c) {
            if (c == forbidden) continue;
            Expr e = express.query(basis[c], cls[c], z, true);
            if (!e.in_span) continue;
            for (int y : e.circuit) {
                if (visited[y]) continue;
                visited[y] = 1;
                std::vector<int>& v = cls[c];
                v.erase(std::find(v.begin(), v.end(), y));
                v.push_back(z);
                basis[c].valid = false;
                if (place(y, c)) return true;
                v.erase(std::find(v.begin(), v.end(), z));
                v.push_back(y);
                basis[c].valid = false;
            }
        }
        return false;
    };
    for (int z : nonzero) {
        std::fill(visited.begin(), visited.end(), 0);
        if (!place(z, -1)) {
            cls.push_back({z});
            basis.emplace_back();
        }
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

}  // namespace

int full_sets(const std::vector<InfoSet>& s, int K) { return count_full(s, K); }

bool matroid_sets(const Mat& code_gen, int greedy_full, std::vector<std::vector<int>>* lists,
                  std::vector<int>* ranks) {
    const int K = code_gen.rows, n = code_gen.cols;
    if (K == 0) return false;
    std::vector<u64> any(code_gen.stride, 0ull);   // columns holding a 1 in some row
    for (int i = 0; i < K; ++i) vec_or(any.data(), code_gen.row(i), code_gen.stride);
    int nnz = 0;
    for (int w = 0; w < code_gen.stride; ++w) nnz += popc64(any[w]);
    const int max_full = nnz / K;
    if (greedy_full >= max_full || n > 200) return false;
    std::vector<std::vector<int>> part;
    if (!matroid_partition(code_gen, part)) return false;
    std::sort(part.begin(), part.end(),
              [](const std::vector<int>& a, const std::vector<int>& b) {
                  return a.size() > b.size();
              });
    // The nonzero columns of a class are independent, so its restricted RREF has one pivot
    // per nonzero column: the ranks are known before any elimination.
    std::vector<std::vector<int>> seq;
    std::vector<int> rk;
    int full = 0;
    for (auto& cols : part) {
        if (cols.empty()) continue;
        int r = 0;
        for (int c : cols) r += (int)((any[c >> 6] >> (c & 63)) & 1u);
        full += (r == K);
        seq.push_back(cols);
        rk.push_back(r);
    }
    if (seq.empty() || full <= greedy_full) return false;
    std::vector<int> order(seq.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rk[a] > rk[b]; });
    lists->clear();
    ranks->clear();
    for (int i : order) {
        lists->push_back(std::move(seq[i]));
        ranks->push_back(rk[i]);
    }
    return true;
}

std::vector<InfoSet> information_sets(const Mat& code_gen) {
    // cpp/distfind/css.cpp:336-366: greedy peel, replaced by the matroid partition when it
    // packs more full-rank sets; then the rank-descending stable sort of bz.cpp:95-97
    std::vector<InfoSet> seq = greedy_sets(code_gen);
    std::vector<std::vector<int>> lists;
    std::vector<int> ranks;
    if (matroid_sets(code_gen, count_full(seq, code_gen.rows), &lists, &ranks)) {
        seq.clear();
        for (const auto& cols : lists) {
            Mat work = code_gen;
            std::vector<int> piv = restricted_rref(work, cols);
            seq.push_back({work, (int)piv.size(), piv});
        }
    }
    std::stable_sort(seq.begin(), seq.end(),
                     [](const InfoSet& a, const InfoSet& b) { return a.rank > b.rank; });
    return seq;
}

}  // namespace qsfb
