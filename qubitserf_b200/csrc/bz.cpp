// BZ schedule on the device engine.  Bounds, termination, verbose lines and the Z/X
// interleave keep the reference's semantics line for line (cpp/distfind/bz.cpp:118-403,
// cpp/distfind/progress.hpp:12-33) so that distance, lower_bound, proven and levels agree
// with the reference run on the same host; the enumeration itself runs on the GPU.
#include "bz.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <random>
#include <thread>

namespace qsfb {

namespace {

using clk = std::chrono::steady_clock;

double since(clk::time_point t) {
    return std::chrono::duration<double>(clk::now() - t).count();
}

void fprint_elapsed(double secs) {
    if (secs < 1.0) std::fprintf(stderr, "Elapsed:[%dms]\n", (int)(secs * 1000.0 + 0.5));
    else std::fprintf(stderr, "Elapsed:[%.3fs]\n", secs);
}
void verbose_bound(int lb, double secs, const char* tag) {
    if (*tag) std::fprintf(stderr, "%s-distance bound: >%d\n", tag, lb);
    else std::fprintf(stderr, "Distance bound: >%d\n", lb);
    fprint_elapsed(secs);
}
void verbose_final(int d, double secs, const char* tag) {
    if (*tag) std::fprintf(stderr, "%s-distance: =%d\n", tag, d);
    else std::fprintf(stderr, "Distance: =%d\n", d);
    fprint_elapsed(secs);
}

bool env_flag(const char* name) { return std::getenv(name) != nullptr; }

}  // namespace

// ------------------------------------------------------------------ seed
int random_is_seed(const Problem& p, int init_best, int trials, unsigned seed, int /*threads*/,
                   std::vector<u64>* word) {
    const int n = p.n;
    const int K = p.code_gen.rows;
    const int stride = p.code_gen.stride;
    if (K == 0) return init_best;
    int nth = (int)std::thread::hardware_concurrency();
    if (nth < 1) nth = 1;
    if (nth > trials) nth = trials;

    struct Out { int best; std::vector<u64> w; };
    auto run = [&](int lo, int hi, unsigned tseed) -> Out {
        std::mt19937 rng(tseed);
        std::vector<int> cols(n);
        Out o{init_best, {}};
        for (int it = lo; it < hi; ++it) {
            std::iota(cols.begin(), cols.end(), 0);
            std::shuffle(cols.begin(), cols.end(), rng);
            Mat M = p.code_gen;
            restricted_rref(M, cols);
            for (int r = 0; r < M.rows; ++r) {
                const int w = M.row_weight(r);
                if (w == 0 || w >= o.best) continue;
                bool logical = p.count_all;
                for (int c = 0; c < p.check.rows && !logical; ++c)
                    if (vec_dot(p.check.row(c), M.row(r), stride)) logical = true;
                if (logical) {
                    o.best = w;
                    o.w.assign(M.row(r), M.row(r) + stride);
                }
            }
        }
        return o;
    };
    std::vector<Out> res;
    if (nth == 1) {
        res.push_back(run(0, trials, seed));
    } else {
        res.resize(nth);
        std::vector<std::thread> pool;
        for (int t = 0; t < nth; ++t) {
            const int lo = (int)((long)trials * t / nth);
            const int hi = (int)((long)trials * (t + 1) / nth);
            pool.emplace_back([&, t, lo, hi]() {
                res[t] = run(lo, hi, seed + 0x9e3779b9u * (unsigned)(t + 1));
            });
        }
        for (auto& th : pool) th.join();
    }
    int best = init_best;
    for (const Out& o : res)
        if (o.best < best) {
            best = o.best;
            if (word) *word = o.w;
        }
    return best;
}

// ------------------------------------------------------------------ side
int BzSide::setup(Device* d, Session* s, const Problem& p, const BzOptions& opt, const char* t) {
    tag = t;
    prob = &p;
    K = p.code_gen.rows;
    even = p.even;
    has_logicals = !(K == 0 || (!p.count_all && p.check.rows == 0));
    if (!has_logicals) { resolved = true; return kOk; }
    sets = information_sets(p.code_gen);
    ng = (int)sets.size();
    ranks.resize(ng);
    for (int g = 0; g < ng; ++g) ranks[g] = sets[g].rank;
    inner = p.seed_upper > 0 ? p.seed_upper : kWeightNone;
    if (p.seed_upper > 0) best_word = p.seed_word;
    std::vector<u64> w;
    const int seeded = random_is_seed(p, inner, opt.seed_trials, 0x9e3779b9u, opt.threads, &w);
    if (seeded < inner) { inner = seeded; best_word = w; }
    maxw = K;
    return dev.init(d, s, p, sets);
}

int BzSide::active_at(int w) const {
    int a = 0;
    while (a < ng && (w + 1) - (K - ranks[a]) > 0) ++a;
    return a;
}

int BzSide::outer_at(int w) const {
    int o = 0;
    for (int g = 0; g < ng; ++g) o += std::max(0, (w + 1) - (K - ranks[g]));
    if (even) o += (o & 1);
    return o;
}

void BzSide::absorb(int w, const LevelOut& o) {
    if (o.found && o.wt < inner) {
        inner = o.wt;
        best_from_level = true;
        best_w = w;
        best_g = o.g;
        best_rank = o.rank;
        best_shift = o.rank_shift;
    }
    ++level;
    outer = outer_at(w);
}

bool BzSide::witness(std::vector<u64>& out) const {
    if (!best_from_level) {
        out = best_word;
        return !out.empty();
    }
    if (best_shift != 0 || best_g < 0 || best_g >= ng) return false;
    // Unrank the lexicographic rank (cpp/qsf/combinatorics.hpp:52-61 order).
    std::vector<std::vector<unsigned long long>> C(K + 1, std::vector<unsigned long long>(best_w + 1, 0));
    for (int n = 0; n <= K; ++n) {
        C[n][0] = 1;
        for (int k = 1; k <= std::min(n, best_w); ++k)
            C[n][k] = C[n - 1][k - 1] + (k <= n - 1 ? C[n - 1][k] : 0);
    }
    auto bn = [&](int n, int k) -> unsigned long long {
        if (k < 0 || n < 0 || k > n) return 0;
        return C[n][k];
    };
    unsigned long long r = best_rank;
    const Mat& G = sets[best_g].g;
    out.assign(G.stride, 0);
    int x = 0;
    for (int i = 0; i < best_w; ++i) {
        for (;;) {
            const unsigned long long cnt = bn(K - 1 - x, best_w - 1 - i);
            if (r < cnt) break;
            r -= cnt;
            ++x;
        }
        if (x >= K) return false;
        vec_xor(out.data(), G.row(x), G.stride);
        ++x;
    }
    return true;
}

// ------------------------------------------------------------------ drivers
namespace {

int run_one(Session* s, BzSide& S, int w, LevelOut& o, BzResult& r, int side_idx) {
    std::vector<LevelReq> q(1);
    q[0].side = &S.dev;
    q[0].w = w;
    q[0].active = S.active_at(w);
    q[0].bound = S.inner;
    std::vector<LevelOut> outs;
    if (q[0].active == 0) {
        o = LevelOut();
    } else {
        const int rc = run_levels(s, q, outs, &r.stats);
        if (rc != kOk) return rc;
        o = outs[0];
    }
    r.trace.push_back({side_idx, w, q[0].active, o.counts});
    return kOk;
}

void finish_witness(const BzSide& S, const Problem& p, BzResult& r, int side_idx) {
    std::vector<u64> c;
    r.witness_side = side_idx;
    if (r.distance >= 0 && S.witness(c)) {
        r.witness = c;
        r.witness_ok = verify_witness(p, c.data(), r.distance);
    }
}

}  // namespace

int bz_distance(Device* dev, const Problem& p, const BzOptions& opt, BzResult& r) {
    const auto t0 = clk::now();
    r = BzResult();
    const int K = p.code_gen.rows;
    if (K == 0 || (!p.count_all && p.check.rows == 0)) {
        r.distance = -1;
        r.seconds = since(t0);
        return kOk;
    }
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    BzSide S;
    int rc = S.setup(dev, lease.s, p, opt, "");
    if (rc != kOk) return rc;
    const bool no_stop = opt.no_early_stop || env_flag("DISTFIND_NO_EARLY_STOP");
    for (int w = 1; w <= S.maxw; ++w) {
        const auto te0 = clk::now();
        LevelOut o;
        rc = run_one(lease.s, S, w, o, r, 0);
        if (rc != kOk) return rc;
        S.absorb(w, o);
        if (S.inner <= S.outer && !no_stop) {
            S.proven = true;
            if (opt.verbose) verbose_final(S.inner, since(t0), "");
            break;
        }
        if (opt.verbose) verbose_bound(std::max(0, S.outer - 1), since(te0), "");
    }
    r.distance = S.inner >= kWeightNone ? -1 : S.inner;
    r.levels = S.level;
    r.lower_bound = S.outer;
    r.proven = S.proven;
    finish_witness(S, p, r, 0);
    r.seconds = since(t0);
    return kOk;
}

int bz_min_interleaved(Device* dev, const Problem& pz, const Problem& px, const BzOptions& opt,
                       BzResult& r) {
    const auto t0 = clk::now();
    r = BzResult();
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    BzSide Z, X;
    int rc = Z.setup(dev, lease.s, pz, opt, "Z");
    if (rc != kOk) return rc;
    rc = X.setup(dev, lease.s, px, opt, "X");
    if (rc != kOk) return rc;
    BzSide* sides[2] = {&Z, &X};
    int best = kWeightNone;
    if (Z.has_logicals) best = std::min(best, Z.inner);
    if (X.has_logicals) best = std::min(best, X.inner);
    const int maxw = std::max(Z.has_logicals ? Z.maxw : 0, X.has_logicals ? X.maxw : 0);
    for (int w = 1; w <= maxw; ++w) {
        for (int si = 0; si < 2; ++si) {
            BzSide* S = sides[si];
            if (S->resolved) continue;
            if (w > S->maxw) continue;
            if (S->outer >= best) { S->resolved = true; continue; }
            const auto te0 = clk::now();
            LevelOut o;
            rc = run_one(lease.s, *S, w, o, r, si);
            if (rc != kOk) return rc;
            S->absorb(w, o);
            best = std::min(best, S->inner);
            if (S->inner <= S->outer) {
                S->proven = true;
                S->resolved = true;
                if (opt.verbose) verbose_final(S->inner, since(t0), S->tag);
            } else {
                if (opt.verbose) verbose_bound(std::max(0, S->outer - 1), since(te0), S->tag);
                if (S->outer >= best) S->resolved = true;
            }
        }
        if (Z.resolved && X.resolved) break;
    }
    auto v = [](const BzSide& S) { return S.has_logicals ? S.inner : kWeightNone; };
    const int dist = std::min(v(Z), v(X));
    r.distance = dist >= kWeightNone ? -1 : dist;
    const int lb = std::min(Z.has_logicals ? Z.outer : kWeightNone, X.has_logicals ? X.outer : kWeightNone);
    r.lower_bound = lb >= kWeightNone ? 0 : lb;
    r.levels = std::max(Z.level, X.level);
    r.proven = Z.resolved && X.resolved && dist < kWeightNone;
    if (r.distance >= 0) {
        if (v(Z) <= v(X)) finish_witness(Z, pz, r, 0);
        else finish_witness(X, px, r, 1);
    }
    r.seconds = since(t0);
    return kOk;
}

int symplectic_bz_distance(Device* dev, const Problem& sp, const BzOptions& opt, BzResult& r) {
    Problem e = isometry_extend(sp);
    if (opt.verbose)
        std::fprintf(stderr,
                     "distfind: non-CSS BZ via the (a|b)->(a|b|a^b) isometry; the bounds below "
                     "are Hamming weights of the length-%d code (= 2 x symplectic weight), so the "
                     "symplectic distance is half the reported value.\n", e.n);
    const int rc = bz_distance(dev, e, opt, r);
    if (rc != kOk) return rc;
    if (r.distance > 0) r.distance /= 2;
    if (r.lower_bound > 0) r.lower_bound /= 2;
    return kOk;
}

}  // namespace qsfb
