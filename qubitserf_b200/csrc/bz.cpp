// BZ schedule on the device engine.  Bounds, termination, verbose lines and the Z/X
// interleave keep the reference's semantics (cpp/distfind/bz.cpp:72-370,
// cpp/distfind/progress.hpp:12-33) so that distance, lower_bound, proven and levels agree
// with the reference run on the same host; the enumeration itself runs on the GPU.
#include "bz.hpp"

#include <algorithm>
#include <tuple>
#include <mutex>
#include <memory>
#include <map>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <random>
#include <thread>
#include <cstring>
#include <condition_variable>

#include <nvtx3/nvToolsExt.h>

#include "infoset_types.hpp"
#include "seed_types.hpp"

namespace qsfb {

double now_seconds() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

namespace {

void fprint_elapsed(double secs) {
    if (secs < 1.0) std::fprintf(stderr, "Elapsed:[%dms]\n", (int)(secs * 1000.0 + 0.5));
    else std::fprintf(stderr, "Elapsed:[%.3fs]\n", secs);
}
void verbose_bound(int lb, double secs, const char* tag) {
    if (*tag) std::fprintf(stderr, "%s-distance bound: >%d\n", tag, lb);
    else std::fprintf(stderr, "Distance bound: >%d\n", lb);
    fprint_elapsed(secs);
}
// DISTFIND_PROFILE: one line per enumerated level of a single-side run, in the reference's
// format (cpp/distfind/bz.cpp:132, 147-155), with the backend named "cuda".
bool profile_on() {
    static const bool on = std::getenv("DISTFIND_PROFILE") != nullptr;
    return on;
}

void verbose_final(int d, double secs, const char* tag) {
    if (*tag) std::fprintf(stderr, "%s-distance: =%d\n", tag, d);
    else std::fprintf(stderr, "Distance: =%d\n", d);
    fprint_elapsed(secs);
}

}  // namespace

// ------------------------------------------------------------------ seed
int random_is_seed(const Problem& p, int init_best, int trials, unsigned seed, bool parallel,
                   std::vector<u64>* word) {
    const int n = p.n;
    const int K = p.code_gen.rows;
    const int stride = p.code_gen.stride;
    if (K == 0 || trials <= 0) return init_best;
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
    std::vector<Out> res(nth);
    auto chunk = [&](int t) {
        const int lo = (int)((long)trials * t / nth);
        const int hi = (int)((long)trials * (t + 1) / nth);
        // one stream: the reference's single-thread case uses `seed` itself
        const unsigned ts = nth == 1 ? seed : seed + 0x9e3779b9u * (unsigned)(t + 1);
        res[t] = run(lo, hi, ts);
    };
    if (!parallel || nth == 1) {
        for (int t = 0; t < nth; ++t) chunk(t);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nth; ++t) pool.emplace_back(chunk, t);
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

namespace {
// The column orders depend only on (n, trials, seed) and the process's thread count, so
// every code of the same length shares them: computed once per key.
std::vector<int> seed_orders_uncached(int n, int trials, unsigned seed, int only);
std::mutex g_orders_mu;
std::map<std::tuple<int, int, unsigned>, std::shared_ptr<const std::vector<int>>> g_orders;
}  // namespace

std::vector<int> seed_orders(int n, int trials, unsigned seed, int only) {
    const auto key = std::make_tuple(n, trials, seed);
    std::shared_ptr<const std::vector<int>> all;
    {
        std::lock_guard<std::mutex> lk(g_orders_mu);
        auto it = g_orders.find(key);
        if (it != g_orders.end()) all = it->second;
    }
    if (!all) {
        auto v = std::make_shared<const std::vector<int>>(seed_orders_uncached(n, trials, seed, -1));
        std::lock_guard<std::mutex> lk(g_orders_mu);
        all = g_orders.emplace(key, v).first->second;
    }
    if (only < 0) return *all;
    if (only >= trials || (size_t)(only + 1) * n > all->size()) return {};
    return std::vector<int>(all->begin() + (size_t)only * n, all->begin() + (size_t)(only + 1) * n);
}

namespace {
std::mutex g_bytes_mu;
std::map<std::tuple<int, int, unsigned>, std::shared_ptr<const std::vector<uint8_t>>> g_bytes;
}  // namespace

std::shared_ptr<const std::vector<uint8_t>> seed_order_bytes(int n, int trials, unsigned seed) {
    const auto key = std::make_tuple(n, trials, seed);
    {
        std::lock_guard<std::mutex> lk(g_bytes_mu);
        auto it = g_bytes.find(key);
        if (it != g_bytes.end()) return it->second;
    }
    const std::vector<int> ord = seed_orders(n, trials, seed);
    auto v = std::make_shared<const std::vector<uint8_t>>(ord.begin(), ord.end());
    std::lock_guard<std::mutex> lk(g_bytes_mu);
    return g_bytes.emplace(key, v).first->second;
}

namespace {
std::vector<int> seed_orders_uncached(int n, int trials, unsigned seed, int only) {
    int nth = (int)std::thread::hardware_concurrency();
    if (nth < 1) nth = 1;
    if (nth > trials) nth = trials;
    std::vector<int> out;
    out.reserve((size_t)(only >= 0 ? 1 : trials) * n);
    std::vector<int> cols(n);
    for (int t = 0; t < nth; ++t) {
        const int lo = (int)((long)trials * t / nth);
        const int hi = (int)((long)trials * (t + 1) / nth);
        if (only >= 0 && (only < lo || only >= hi)) continue;
        std::mt19937 rng(nth == 1 ? seed : seed + 0x9e3779b9u * (unsigned)(t + 1));
        for (int it = lo; it < hi; ++it) {
            std::iota(cols.begin(), cols.end(), 0);
            std::shuffle(cols.begin(), cols.end(), rng);
            if (only < 0 || it == only) out.insert(out.end(), cols.begin(), cols.end());
            if (it == only) return out;
        }
    }
    return out;
}
}  // namespace

void BzSide::apply_device_seed(unsigned key) {
    seed_pending = false;
    seed_perm.reset();
    if (key == 0xffffffffu) return;
    const int w = (int)(key >> 15);
    if (w < inner) {
        inner = w;
        inner0 = w;
        seed_trial = (int)((key >> 7) & 0xff);
        seed_row = (int)(key & 0x7f);
        best_word.clear();
    }
}

// ------------------------------------------------------------------ side
int BzSide::setup_host(const Problem& p, const BzOptions& opt, const char* t) {
    tag = t;
    prob = &p;
    K = p.code_gen.rows;
    even = p.even;
    has_logicals = !(K == 0 || (!p.count_all && p.check.rows == 0));
    if (!has_logicals) { resolved = resolved0 = true; return kOk; }
    const bool dev_sets = opt.device_infosets && K <= kInfosetMaxK && p.n <= kInfosetMaxN;
    if (!dev_sets) {
        sets = information_sets(p.code_gen);
        ng = (int)sets.size();
        ranks.resize(ng);
        for (int g = 0; g < ng; ++g) ranks[g] = sets[g].rank;
    }
    inner = p.seed_upper > 0 ? p.seed_upper : kWeightNone;
    if (p.seed_upper > 0) best_word = p.seed_word;
    if (opt.device_seed && K <= kSeedMaxK && p.n <= kSeedMaxN && opt.seed_trials <= 256 &&
        opt.seed_trials > 0) {
        // the eliminations run on the GPU (setup_jobs); draw the column orders here
        seed_pending = true;
        seed_trials = opt.seed_trials;
        seed_perm = seed_order_bytes(p.n, seed_trials, 0x9e3779b9u);
    } else {
        std::vector<u64> w;
        const int seeded = random_is_seed(p, inner, opt.seed_trials, 0x9e3779b9u,
                                          opt.parallel_seed, &w);
        if (seeded < inner) { inner = seeded; best_word = w; }
    }
    maxw = K;
    inner0 = inner;
    resolved0 = resolved;
    if (dev_sets) {
        infoset_pending = true;   // built by setup_jobs_device
        return kOk;
    }
    return dev.prepare(p, sets);
}

int BzSide::adopt_sets(std::vector<InfoSet>&& s, uint32_t* red, uint32_t* syn, int W32, int SWP,
                       Device* d, Arena* arena) {
    infoset_pending = false;
    sets = std::move(s);
    ng = (int)sets.size();
    ranks.resize(ng);
    for (int g = 0; g < ng; ++g) ranks[g] = sets[g].rank;
    if (!red) return dev.prepare(*prob, sets);
    return dev.adopt_device(*prob, sets, red, syn, W32, SWP, d, arena);
}

void BzSide::reset() {
    inner = inner0;
    resolved = resolved0;
    outer = 0;
    level = 0;
    proven = false;
    best_from_level = false;
    best_g = -1;
    for (auto& kv : dev.lists) kv.second.ready = kv.second.pm_ready = false;
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
        if (best_word.empty() && seed_trial >= 0) {
            // replay the winning trial's elimination on the host
            const std::vector<int> ord = seed_orders(prob->n, seed_trials, 0x9e3779b9u, seed_trial);
            Mat M = prob->code_gen;
            restricted_rref(M, ord);
            if (seed_row >= M.rows) return false;
            out.assign(M.row(seed_row), M.row(seed_row) + M.stride);
            return true;
        }
        out = best_word;
        return !out.empty();
    }
    if (best_shift != 0 || best_g < 0 || best_g >= ng) return false;
    // Unrank the lexicographic rank (the order of cpp/qsf/combinatorics.hpp:52-61).
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

// ------------------------------------------------------------------ job
BzJob::BzJob(Problem p0, const BzOptions& o) : pair(false), opt(o) { p[0] = std::move(p0); }

BzJob::BzJob(Problem pz, Problem px, const BzOptions& o) : pair(true), opt(o) {
    p[0] = std::move(pz);
    p[1] = std::move(px);
}

BzJob::BzJob(Builder build, bool is_pair, const BzOptions& o)
    : pair(is_pair), opt(o), build_(std::move(build)) {}

int BzJob::setup_host() {
    t0_ = tl_ = now_seconds();
    if (build_) {
        zero = build_(p[0], p[1]) == 1;
        build_ = nullptr;
        if (zero) {
            done_ = true;
            return kOk;
        }
    }
    const int nsides = pair ? 2 : 1;
    for (int i = 0; i < nsides; ++i) {
        const int rc = s[i].setup_host(p[i], opt, pair ? (i == 0 ? "Z" : "X") : "");
        if (rc != kOk) return rc;
    }
    finish_setup();
    return kOk;
}

void BzJob::finish_setup() {
    if (zero) return;
    if (!pair) {
        done_ = !s[0].has_logicals;
        maxw_ = s[0].maxw;
        no_stop_ = opt.no_early_stop || std::getenv("DISTFIND_NO_EARLY_STOP") != nullptr;
    } else {
        best_ = kWeightNone;
        maxw_ = 0;
        for (int i = 0; i < 2; ++i)
            if (s[i].has_logicals) {
                best_ = std::min(best_, s[i].inner);
                maxw_ = std::max(maxw_, s[i].maxw);
            }
        done_ = s[0].resolved && s[1].resolved;
    }
}

void BzJob::reset() {
    final_.reset();
    if (zero) return;
    for (int i = 0; i < (pair ? 2 : 1); ++i) s[i].reset();
    w_ = 0;
    stats = RunStats();
    trace.clear();
    t0_ = tl_ = now_seconds();
    if (!pair) {
        done_ = !s[0].has_logicals;
    } else {
        best_ = kWeightNone;
        for (int i = 0; i < 2; ++i)
            if (s[i].has_logicals) best_ = std::min(best_, s[i].inner);
        done_ = s[0].resolved && s[1].resolved;
    }
}

std::vector<SideDev*> BzJob::device_sides() {
    std::vector<SideDev*> v;
    for (int i = 0; i < (pair ? 2 : 1); ++i)
        if (s[i].has_logicals) v.push_back(&s[i].dev);
    return v;
}

void BzJob::requests(std::vector<LevelReq>& q, std::vector<int>& side) {
    if (done_) return;
    const int w = w_ + 1;
    for (int i = 0; i < (pair ? 2 : 1); ++i) {
        BzSide& S = s[i];
        if (pair && (S.resolved || w > S.maxw || S.outer >= best_)) continue;
        const int active = S.active_at(w);
        if (active == 0) continue;
        LevelReq r;
        r.side = &S.dev;
        r.w = w;
        r.active = active;
        // candidates must beat the side's upper bound strictly; ties among new finds stay
        // inside the level so that its witness is deterministic
        r.bound = S.inner >= kWeightNone ? kWeightNone : S.inner - 1;
        q.push_back(r);
        side.push_back(i);
    }
}

void BzJob::apply(const std::vector<const LevelOut*>& outs, const std::vector<int>& side) {
    if (done_) return;
    const int w = ++w_;
    const double now = now_seconds();
    auto out_for = [&](int i) -> LevelOut {
        for (size_t k = 0; k < side.size(); ++k)
            if (side[k] == i) return *outs[k];
        return LevelOut();
    };
    auto record = [&](int i, const LevelOut& o) {
        trace.push_back({i, w, s[i].active_at(w), o.counts});
    };
    if (!pair) {
        BzSide& S = s[0];
        const LevelOut o = out_for(0);
        S.absorb(w, o);
        record(0, o);
        if (profile_on() && S.has_logicals) {
            const unsigned long long total = host_binom(S.K, w);
            const int act = S.active_at(w);
            std::fprintf(stderr, "[prof cuda] d=%d K=%d ng=%d/%d stride=%d total=%llu "
                         "work=%llu -> %.3f ms\n", w, S.K, act, S.ng, words_for(p[0].n), total,
                         total * (unsigned long long)act, 1e3 * (now - tl_));
        }
        if (S.inner <= S.outer && !no_stop_) {
            S.proven = true;
            done_ = true;
            if (opt.verbose) verbose_final(S.inner, now - t0_, "");
        } else if (opt.verbose) {
            verbose_bound(std::max(0, S.outer - 1), now - tl_, "");
        }
        if (w >= maxw_) done_ = true;
    } else {
        for (int i = 0; i < 2; ++i) {
            BzSide& S = s[i];
            if (S.resolved || w > S.maxw) continue;
            if (S.outer >= best_) { S.resolved = true; continue; }
            const LevelOut o = out_for(i);
            S.absorb(w, o);
            record(i, o);
            best_ = std::min(best_, S.inner);
            if (S.inner <= S.outer) {
                S.proven = true;
                S.resolved = true;
                if (opt.verbose) verbose_final(S.inner, now - t0_, S.tag);
            } else {
                if (opt.verbose) verbose_bound(std::max(0, S.outer - 1), now - tl_, S.tag);
                if (S.outer >= best_) S.resolved = true;
            }
        }
        if ((s[0].resolved && s[1].resolved) || w >= maxw_) done_ = true;
    }
    tl_ = now;
}

namespace {
void finish_witness(const BzSide& S, const Problem& p, BzResult& r, int side_idx) {
    std::vector<u64> c;
    r.witness_side = side_idx;
    if (r.distance >= 0 && S.witness(c)) {
        r.witness = c;
        r.witness_ok = verify_witness(p, c.data(), r.distance);
    }
}
}  // namespace

BzResult BzJob::result() { return final_result(); }

const BzResult& BzJob::final_result() {
    if (!final_) final_.reset(new BzResult(compute_result()));
    return *final_;
}

BzResult BzJob::compute_result() {
    BzResult r;
    r.stats = stats;
    r.trace = trace;
    r.seconds = now_seconds() - t0_;
    if (zero) {
        r.distance = 0;
        r.proven = true;
        r.witness_ok = true;
        return r;
    }
    if (!pair) {
        const BzSide& S = s[0];
        if (!S.has_logicals) return r;
        r.distance = S.inner >= kWeightNone ? -1 : S.inner;
        r.levels = S.level;
        r.lower_bound = S.outer;
        r.proven = S.proven;
        finish_witness(S, p[0], r, 0);
        return r;
    }
    auto v = [](const BzSide& S) { return S.has_logicals ? S.inner : kWeightNone; };
    const int dist = std::min(v(s[0]), v(s[1]));
    r.distance = dist >= kWeightNone ? -1 : dist;
    const int lb = std::min(s[0].has_logicals ? s[0].outer : kWeightNone,
                            s[1].has_logicals ? s[1].outer : kWeightNone);
    r.lower_bound = lb >= kWeightNone ? 0 : lb;
    r.levels = std::max(s[0].level, s[1].level);
    r.proven = s[0].resolved && s[1].resolved && dist < kWeightNone;
    if (r.distance >= 0) {
        if (v(s[0]) <= v(s[1])) finish_witness(s[0], p[0], r, 0);
        else finish_witness(s[1], p[1], r, 1);
    }
    return r;
}

// ------------------------------------------------------------------ rounds
cudaError_t launch_seed_trials(int W, const SeedDesc* d_descs, int ndesc, int total_trials,
                               cudaStream_t st);

namespace {
// Seed trials in flight: launched by seeds_begin, folded into the bounds by seeds_end.
struct SeedLaunch {
    std::vector<BzSide*> sides;   // in the order of `keys`
    unsigned* keys = nullptr;     // pinned host copy of the keys
    const unsigned* d_keys = nullptr;
    cudaStream_t st = nullptr;
    bool launched = false;
    int launches = 0;
    double t0 = 0.0;
};

// Every pending seed trial of every job, one launch per row width, on the session's
// `urgent2` stream: staging in the session's seed buffer, so that other preparation work
// may use the main staging while the trials run.
int seeds_begin(Session* s, Arena* arena, std::vector<BzJob*>& jobs, SeedLaunch* L) {
    L->t0 = now_seconds();
    std::vector<BzSide*> pend[5];   // by row words W = 1 .. 4
    for (BzJob* j : jobs)
        for (int i = 0; i < (j->pair ? 2 : 1); ++i)
            if (j->s[i].seed_pending) pend[words_for(j->s[i].prob->n)].push_back(&j->s[i]);
    for (int W = 1; W <= 4; ++W) L->sides.insert(L->sides.end(), pend[W].begin(), pend[W].end());
    const size_t n = L->sides.size();
    if (n == 0) return kOk;
    // layout: keys (all sides) | descs (all sides, W = 1 first) | per side: gen, check |
    // the column orders, shared by every side of the same length (one copy each)
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    size_t off = 0;
    const size_t off_keys = off;
    off = al(off + n * 4);
    const size_t off_desc = off;
    off = al(off + n * sizeof(SeedDesc));
    std::vector<size_t> og(n), oc(n), op(n);
    std::map<const std::vector<uint8_t>*, size_t> perm_off;
    for (size_t i = 0; i < n; ++i) {
        const Problem& p = *L->sides[i]->prob;
        const int W = words_for(p.n);
        og[i] = off; off = al(off + (size_t)p.code_gen.rows * W * 8);
        oc[i] = off; off = al(off + (size_t)std::max(1, p.check.rows) * W * 8);
        const std::vector<uint8_t>* pp = L->sides[i]->seed_perm.get();
        auto it = perm_off.find(pp);
        if (it == perm_off.end()) {
            it = perm_off.emplace(pp, off).first;
            off = al(off + pp->size());
        }
        op[i] = it->second;
    }
    char* d = (char*)arena->alloc(off);
    if (!d) return kErrMemory;
    int rc = s->grow_pinned(s->h_seed, off);
    if (rc != kOk) return rc;
    char* h = (char*)s->h_seed.h;
    SeedDesc* hd = (SeedDesc*)(h + off_desc);
    unsigned* hk = (unsigned*)(h + off_keys);
    int trials[5] = {0, 0, 0, 0, 0};
    for (size_t i = 0; i < n; ++i) {
        const BzSide& S = *L->sides[i];
        const Problem& p = *S.prob;
        const int W = words_for(p.n);
        u64* g = (u64*)(h + og[i]);
        for (int r = 0; r < p.code_gen.rows; ++r)
            for (int w = 0; w < W; ++w) g[(size_t)r * W + w] = p.code_gen.row(r)[w];
        u64* c = (u64*)(h + oc[i]);
        for (int r = 0; r < p.check.rows; ++r)
            for (int w = 0; w < W; ++w) c[(size_t)r * W + w] = p.check.row(r)[w];
        SeedDesc& D = hd[i];
        D.gen = (const unsigned long long*)(d + og[i]);
        D.check = (const unsigned long long*)(d + oc[i]);
        D.perm = (const uint8_t*)(d + op[i]);
        D.key = (unsigned*)(d + off_keys) + i;
        D.trial_base = trials[W];
        D.K = p.code_gen.rows;
        D.n = p.n;
        D.kcheck = p.count_all ? 0 : p.check.rows;
        D.count_all = p.count_all ? 1 : 0;
        D.init_best = S.inner;
        D.pad_ = 0;
        hk[i] = 0xffffffffu;
        trials[W] += S.seed_trials;
    }
    for (const auto& po : perm_off) std::memcpy(h + po.second, po.first->data(), po.first->size());
    // on a stream above the rounds' priority: in a pipelined batch or a server, the rounds
    // of other codes fill the SMs meanwhile, and these codes wait for the result
    const SeedDesc* dd = (const SeedDesc*)(d + off_desc);
    // the keys' read-back is queued by seeds_end: queued here, behind the trials, it would
    // hold back every later device-to-host copy of the preparation on the same copy engine
    L->st = s->urgent2;
    L->keys = hk;
    L->d_keys = (const unsigned*)(d + off_keys);
    L->launched = true;
    bool ok = cudaMemcpyAsync(d, h, off, cudaMemcpyHostToDevice, L->st) == cudaSuccess;
    size_t first = 0;   // descriptors are grouped by W, W = 1 first
    for (int W = 1; W <= 4 && ok; ++W) {
        const size_t nw = pend[W].size();
        if (nw > 0)
            ok = launch_seed_trials(W, dd + first, (int)nw, trials[W], L->st) == cudaSuccess;
        first += nw;
        L->launches += nw > 0 ? 1 : 0;
    }
    if (!ok) {
        cudaGetLastError();
        cudaStreamSynchronize(L->st);
        cudaGetLastError();
        L->launched = false;
        return kErrDevice;
    }
    return kOk;
}

// Waits for the trials of seeds_begin and folds the per-side keys into the bounds.
int seeds_end(std::vector<BzJob*>& jobs, SeedLaunch* L, RunStats* stats) {
    if (L->launched) {
        const double tw0 = now_seconds();
        L->launched = false;
        if (cudaMemcpyAsync(L->keys, L->d_keys, L->sides.size() * 4, cudaMemcpyDeviceToHost,
                            L->st) != cudaSuccess ||
            cudaStreamSynchronize(L->st) != cudaSuccess) {
            cudaGetLastError();
            return kErrDevice;
        }
        if (stats) {
            stats->device_seed_wait_s += now_seconds() - tw0;
            stats->launches += L->launches;
        }
        for (size_t i = 0; i < L->sides.size(); ++i) L->sides[i]->apply_device_seed(L->keys[i]);
    }
    if (!L->sides.empty())
        for (BzJob* j : jobs) j->finish_setup();
    if (stats) stats->device_seed_s += now_seconds() - L->t0;
    return kOk;
}
}  // namespace

int setup_jobs_host(std::vector<BzJob*>& jobs, int host_threads, RunStats* stats) {
    const double th0 = now_seconds();
    int nth = host_threads > 0 ? host_threads : (int)std::thread::hardware_concurrency();
    nth = std::max(1, std::min<int>(nth, (int)jobs.size()));
    std::atomic<int> err{kOk};
    host_parallel_for(jobs.size(), [&](size_t i) {
        const int rc = jobs[i]->setup_host();
        if (rc != kOk) err.store(rc);
    }, nth);
    if (err.load() != kOk) return err.load();
    if (stats) stats->host_setup_s += now_seconds() - th0;
    return kOk;
}

int setup_jobs_device(Device* dev, Session* s, Arena* arena, std::vector<BzJob*>& jobs,
                      RunStats* stats) {
    // the seed trials and the information-set eliminations are independent: the trials run
    // on one stream while the sets are built on another and finished on the host
    SeedLaunch L;
    int rc = seeds_begin(s, arena, jobs, &L);
    std::vector<BzSide*> pend;
    for (BzJob* j : jobs)
        if (!j->zero)
            for (int i = 0; i < (j->pair ? 2 : 1); ++i)
                if (j->s[i].infoset_pending) pend.push_back(&j->s[i]);
    if (rc == kOk) rc = device_infosets(s, arena, pend, stats);
    const int rc2 = seeds_end(jobs, &L, stats);   // also after a failure: nothing left in flight
    if (rc != kOk) return rc;
    if (rc2 != kOk) return rc2;
    std::vector<SideDev*> sides;
    for (BzJob* j : jobs)
        for (SideDev* sd : j->device_sides()) sides.push_back(sd);
    return upload_sides(dev, s, arena, sides);
}

int setup_jobs(Device* dev, Session* s, Arena* arena, std::vector<BzJob*>& jobs,
               int host_threads, RunStats* stats) {
    const int rc = setup_jobs_host(jobs, host_threads, stats);
    return rc != kOk ? rc : setup_jobs_device(dev, s, arena, jobs, stats);
}


namespace {
// Computes the final results (witness rebuilt and verified on the host) of the jobs a round
// finished, on a thread of its own, so that the round loop goes straight on to launching
// the next round.  The results are all in when the finisher is destroyed.
class Finisher {
public:
    Finisher() : th_([this]() { loop(); }) {}
    ~Finisher() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_one();
        th_.join();
    }
    void push(const std::vector<BzJob*>& v) {
        if (v.empty()) return;
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.insert(q_.end(), v.begin(), v.end());
        }
        cv_.notify_one();
    }

private:
    void loop() {
        for (;;) {
            std::vector<BzJob*> take;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this]() { return stop_ || !q_.empty(); });
                take.swap(q_);
                if (take.empty() && stop_) return;
            }
            for (BzJob* j : take) j->final_result();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<BzJob*> q_;
    bool stop_ = false;
    std::thread th_;
};
}  // namespace

int run_rounds(Session* s, std::vector<BzJob*>& jobs, RunStats* stats, int* rounds,
               double* span_ms, const JobFeed* feed) {
    int nround = 0;
    // a batch's answers are computed beside its rounds (a single job's by its caller)
    std::unique_ptr<Finisher> finisher;
    if (jobs.size() > 1 || feed) finisher.reset(new Finisher());
    std::vector<LevelReq> q;
    std::vector<int> side, owner;
    std::vector<LevelOut> outs;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (span_ms) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s->stream);
    }
    int rc = kOk;
    for (;;) {
        if (feed) (*feed)(jobs, false);
        bool any = false;
        q.clear(); side.clear(); owner.clear();
        for (size_t j = 0; j < jobs.size(); ++j) {
            if (jobs[j]->done()) continue;
            any = true;
            const size_t before = q.size();
            jobs[j]->requests(q, side);
            for (size_t k = before; k < q.size(); ++k) owner.push_back((int)j);
        }
        if (!any) {
            if (feed && (*feed)(jobs, true)) continue;
            break;
        }
        ++nround;
        RunStats rs;
        outs.clear();
        if (!q.empty()) {
            nvtxRangePushA("qsfb round");   // one range per round for profilers (no-op alone)
            rc = run_levels(s, q, outs, &rs);
            nvtxRangePop();
            if (rc != kOk) break;
        }
        // per-job slices (requests of one job are contiguous)
        const double ta0 = now_seconds();
        size_t k = 0;
        std::vector<BzJob*> finished;
        for (size_t j = 0; j < jobs.size(); ++j) {
            if (jobs[j]->done()) continue;
            std::vector<const LevelOut*> o;
            std::vector<int> sd;
            unsigned long long cw = 0;
            while (k < q.size() && owner[k] == (int)j) {
                o.push_back(&outs[k]);
                sd.push_back(side[k]);
                for (unsigned long long c : outs[k].counts) cw += c;
                ++k;
            }
            jobs[j]->stats.codewords += cw;
            jobs[j]->apply(o, sd);
            if (jobs[j]->done()) finished.push_back(jobs[j]);
        }
        rs.host_apply_s += now_seconds() - ta0;
        if (stats) {
            stats->host_plan_s += rs.host_plan_s;
            stats->host_apply_s += rs.host_apply_s;
            stats->ms_gen += rs.ms_gen;
            stats->ms_pairs += rs.ms_pairs;
            stats->ms_tc += rs.ms_tc;
            stats->jobs += rs.jobs;
            stats->codewords += rs.codewords;
            stats->popc_issued += rs.popc_issued;
            stats->zero_codewords += rs.zero_codewords;
            stats->tc_codewords += rs.tc_codewords;
            stats->tc_operand_bytes += rs.tc_operand_bytes;
            stats->list_bytes_written += rs.list_bytes_written;
            stats->launches += rs.launches;
        }
        if (jobs.size() == 1) {
            // a single job owns the whole device time of its rounds
            jobs[0]->stats.ms_gen += rs.ms_gen;
            jobs[0]->stats.ms_pairs += rs.ms_pairs;
            jobs[0]->stats.launches += rs.launches;
            jobs[0]->stats.jobs += rs.jobs;
        }
        // answers of the jobs this round finished (witnesses rebuilt and verified) are
        // computed on the finisher's thread while the next rounds run
        if (finisher) finisher->push(finished);
    }
    if (span_ms) {
        cudaEventRecord(e1, s->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        *span_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (rounds) *rounds = nround;
    return rc;
}

int run_jobs(Device* dev, std::vector<BzJob*>& jobs, int host_threads, RunStats* stats,
             int* rounds) {
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    Arena arena(dev);
    int rc = setup_jobs(dev, lease.s, &arena, jobs, host_threads, stats);
    if (rc != kOk) return rc;
    return run_rounds(lease.s, jobs, stats, rounds);
}

int bz_distance(Device* dev, const Problem& p, const BzOptions& opt, BzResult& r) {
    BzJob job(p, opt);
    std::vector<BzJob*> jobs{&job};
    const int rc = run_jobs(dev, jobs, 1, nullptr);
    if (rc != kOk) return rc;
    r = job.result();
    return kOk;
}

int bz_min_interleaved(Device* dev, const Problem& pz, const Problem& px, const BzOptions& opt,
                       BzResult& r) {
    BzJob job(pz, px, opt);
    std::vector<BzJob*> jobs{&job};
    const int rc = run_jobs(dev, jobs, 1, nullptr);
    if (rc != kOk) return rc;
    r = job.result();
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
