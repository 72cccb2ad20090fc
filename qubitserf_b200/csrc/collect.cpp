// Host driver and C ABI of the low-weight collector (codeaut_bz_*).
//
// The reference's handle (cpp/codeaut/bz.cpp:55-138) packs G, runs the collect mode of its
// enumeration backend once per subset size and sorts + deduplicates the hits.  Here one call
// does: pack G; find each row's private column (the probe words skip them, the pivot count
// stands in for them); choose the probe width; generate every prefix/suffix list the levels
// need in one launch; one pair-sweep launch per subset size into one output buffer; one
// synchronisation.  The sweeps append the rare pairs that pass their lower bound as
// candidates; one more kernel evaluates those exactly and appends the hits.  Both counters
// are exact even when their buffers are too small, so an overflow re-runs the stage once
// with the exact capacity (the reference recomputes the level on its CPU backend instead;
// there is no CPU path here).  The sort and
// deduplication stay on the host as in the reference.
#include "../../include/qsf_b200.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <utility>
#include <vector>

#include "collect_types.hpp"
#include "engine.hpp"
#include "filter_plan.hpp"

namespace qsfb {

cudaError_t launch_collect_gen(const CollectListDesc* d_lists, int nlists, unsigned long long runs,
                               const CollectShared& S, const unsigned long long* d_binom,
                               int num_sms, cudaStream_t st);
cudaError_t launch_collect_exact(const CollectLevelDesc* d_levels, const CollectShared& S,
                                 const unsigned long long* d_binom, int num_sms, cudaStream_t st);
cudaError_t launch_collect_pairs(const CollectLevelDesc* d_levels, int level,
                                 unsigned long long jobs, const CollectShared& S,
                                 const unsigned long long* d_binom, int num_sms,
                                 cudaStream_t st);

namespace {

constexpr long long kComboCap = 1LL << 62;     // bz.cpp:29
constexpr unsigned long long kFirstCap = 1ull << 16;   // output rows before the first run
constexpr unsigned long long kFirstCand = 1ull << 20;  // candidate pairs before the first run

struct CollectHandle {
    int n = 0, stride = 0;
    bool ok = false;
    long long combos = 0, count = 0;
    std::vector<uint64_t> rows;   // count x stride, sorted, distinct
    std::string backend;
    QsfbCollectStats st{};
};

// C(n, k) with the reference's per-level cap (bz.cpp:87-88): min(C(n,k), 2^62).
long long capped_binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    unsigned __int128 c = 1;
    for (int i = 1; i <= k; ++i) {
        c = c * (unsigned)(n - k + i) / (unsigned)i;
        if (c > (unsigned __int128)kComboCap) return kComboCap;
    }
    return (long long)c;
}

// P(Binomial(bits, 1/2) <= t), bits <= 256 (the probe filter's pass rate on random rows).
double binom_cdf_half(int bits, int t) {
    if (t < 0) return 0.0;
    if (t >= bits) return 1.0;
    double acc = 0.0;
    for (int i = 0; i <= t; ++i)
        acc += std::exp(std::lgamma(bits + 1.0) - std::lgamma(i + 1.0) -
                        std::lgamma(bits - i + 1.0) - bits * std::log(2.0));
    return std::min(acc, 1.0);
}

// Probe variant (width HP, bound FILT of collect.cu's probe_bound): the least expected cost
// per pair in POPC-pipe cycles, max(POPCs, other integer ops / 4) (the ALU pipe issues four
// times the POPC rate), plus ~256 for every pair that passes to the exact evaluation, at
// the fair-coin pass rates of filter_plan.cpp.  QSFB_COLLECT_HP / QSFB_COLLECT_FILT force
// a width / bound (tests cover every variant this way).
struct ProbeVariant { int hp, filt; };

ProbeVariant choose_probe(int n_np, int t) {
    struct Cand { int hp, filt; double popc, alu; };
    const Cand cands[7] = {{1, 0, 1, 2.5}, {2, 0, 2, 4.5}, {2, 2, 1, 3.5}, {4, 0, 4, 8.5},
                           {4, 4, 1, 5.5}, {4, 6, 2, 11.5}, {8, 0, 8, 16.5}};
    int force_hp = 0, force_f = -1;
    if (const char* e = std::getenv("QSFB_COLLECT_HP")) force_hp = std::atoi(e);
    if (const char* e = std::getenv("QSFB_COLLECT_FILT")) force_f = std::atoi(e);
    const int need = std::max(1, (n_np + 31) / 32);
    ProbeVariant best{1, 0};
    double best_cost = 1e300;
    for (const Cand& c : cands) {
        if (force_hp > 0 && c.hp != force_hp) continue;
        if (force_f >= 0 && c.filt != force_f) continue;
        // wider probes than the non-private columns only add zero words
        if (force_hp <= 0 && c.hp > 1 && c.hp / 2 >= need) continue;
        const double pass = c.filt == 0 ? binom_cdf_half(std::min(32 * c.hp, n_np), t)
                                        : filter_pass_rate(c.filt, n_np, t);
        const double cost = std::max(c.popc, c.alu / 4.0) + 256.0 * pass;
        if (cost < best_cost) { best_cost = cost; best = {c.hp, c.filt}; }
    }
    return best;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Device allocations of one call, released together.
struct DevBufs {
    Device* dev;
    std::vector<std::pair<void*, size_t>> held;
    explicit DevBufs(Device* d) : dev(d) {}
    ~DevBufs() { for (auto& h : held) dev->release(h.first, h.second); }
    void* get(size_t bytes) {
        void* p = dev->alloc(bytes ? bytes : 16);
        if (p) held.emplace_back(p, bytes ? bytes : 16);
        return p;
    }
};

// Sort rows of `s` words (word 0 first, as RowLess of bz.cpp:38-50) and drop repeats.
void sort_unique(std::vector<uint64_t>& v, int s, long long* count) {
    const size_t nr = v.size() / (size_t)s;
    if (s == 1) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        *count = (long long)v.size();
        return;
    }
    std::vector<size_t> idx(nr);
    std::iota(idx.begin(), idx.end(), (size_t)0);
    const uint64_t* base = v.data();
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
        const uint64_t* pa = base + (size_t)a * s;
        const uint64_t* pb = base + (size_t)b * s;
        for (int i = 0; i < s; ++i)
            if (pa[i] != pb[i]) return pa[i] < pb[i];
        return false;
    });
    std::vector<uint64_t> out;
    out.reserve(v.size());
    for (size_t i = 0; i < nr; ++i) {
        const uint64_t* r = base + (size_t)idx[i] * s;
        if (!out.empty() && std::memcmp(out.data() + out.size() - s, r, (size_t)s * 8) == 0)
            continue;
        out.insert(out.end(), r, r + s);
    }
    v.swap(out);
    *count = (long long)(v.size() / (size_t)s);
}

int run_collect(const uint8_t* G, int m, int n, int p, int keep, CollectHandle* H) {
    const int S64 = (n + 63) / 64;
    const int maxsw = std::min(p, m);
    if (n > 64 * kCollectMaxWords || m > kBinomMaxN || maxsw > kCollectMaxSize)
        return kErrUnsupported;
    int rc = kOk;
    Device* dev = Device::get(&rc);
    if (!dev) return rc;
    if (cudaSetDevice(dev->id) != cudaSuccess) { cudaGetLastError(); return kErrDevice; }

    // ---- host: packed rows, private columns, probe rows
    std::vector<uint64_t> rows((size_t)m * S64, 0ull);
    std::vector<int> colcount(n, 0);
    for (int r = 0; r < m; ++r)
        for (int j = 0; j < n; ++j)
            if (G[(size_t)r * n + j] & 1) {
                rows[(size_t)r * S64 + (j >> 6)] |= 1ull << (j & 63);
                ++colcount[j];
            }
    std::vector<uint8_t> piv(m, 0);
    std::vector<char> is_private(n, 0);
    int npiv = 0;
    for (int r = 0; r < m; ++r)
        for (int j = 0; j < n; ++j)
            if ((G[(size_t)r * n + j] & 1) && colcount[j] == 1) {
                piv[r] = 1;
                is_private[j] = 1;
                ++npiv;
                break;
            }
    std::vector<int> np_cols;
    for (int j = 0; j < n; ++j)
        if (!is_private[j]) np_cols.push_back(j);
    const int n_np = (int)np_cols.size();
    // threshold on the probe weight of the heaviest level's pairs (their fewest pivots)
    const int t = keep - std::max(0, maxsw - (m - npiv));
    const ProbeVariant pv = choose_probe(n_np, t);
    const int HP = pv.hp;
    std::vector<uint32_t> probe_rows((size_t)m * HP, 0u);
    for (int r = 0; r < m; ++r)
        for (int b = 0; b < 32 * HP && b < n_np; ++b)
            if (G[(size_t)r * n + np_cols[b]] & 1)
                probe_rows[(size_t)r * HP + (b >> 5)] |= 1u << (b & 31);
    H->st.probe_words = HP;
    H->st.filter = pv.filt;
    H->st.pivots = npiv;

    // ---- lists: colex a-subsets (a = ceil(sw/2)) and reflected b-subsets (b = floor(sw/2))
    const int amax = (maxsw + 1) / 2, bmax = maxsw / 2;
    std::vector<unsigned long long> xcount(amax + 1, 0), ycount(bmax + 1, 0);
    for (int sw = 1; sw <= maxsw; ++sw) {
        const int a = (sw + 1) / 2, b = sw / 2;
        // prefixes live in [0, m - b), suffixes in [a, m)
        xcount[a] = std::max(xcount[a], dev->binom(m - b, a));
        ycount[b] = std::max(ycount[b], dev->binom(m - a, b));
    }
    struct ListPlan { int size, reflect; unsigned long long count; size_t off_p, off_c; };
    std::vector<ListPlan> lp;
    for (int a = 1; a <= amax; ++a) lp.push_back({a, 0, xcount[a], 0, 0});
    for (int b = 0; b <= bmax; ++b) lp.push_back({b, 1, ycount[b], 0, 0});
    // every list must be addressable: a saturated binomial means astronomically many pairs
    size_t list_bytes = 0;
    for (ListPlan& l : lp) {
        if (l.count >= (1ull << 40)) return kErrMemory;
        l.off_p = list_bytes;
        list_bytes += (l.count * (size_t)HP * 4 + 255) / 256 * 256;
        l.off_c = list_bytes;
        list_bytes += (l.count + 255) / 256 * 256;
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); return kErrDevice; }
    if (list_bytes > free_b / 2 + dev->bytes_cached() / 2) return kErrMemory;

    // ---- levels: terms and jobs
    std::vector<CollectTerm> terms;
    std::vector<CollectLevelDesc> levels(maxsw);
    std::vector<size_t> term_off(maxsw);
    for (int sw = 1; sw <= maxsw; ++sw) {
        const int a = (sw + 1) / 2, b = sw / 2;
        CollectLevelDesc& L = levels[sw - 1];
        L.a = a; L.b = b;
        term_off[sw - 1] = terms.size();
        unsigned long long jobs = 0;
        for (int q = a - 1; q <= m - 1 - b; ++q) {
            CollectTerm T;
            T.x0 = dev->binom(q, a);
            T.nx = dev->binom(q, a - 1);
            T.ny = dev->binom(m - 1 - q, b);
            if (T.nx == 0 || T.ny == 0) continue;
            const unsigned long long xt = (T.nx + kCollectTileX - 1) / kCollectTileX;
            T.ychunks = (T.ny + kCollectChunkY - 1) / kCollectChunkY;
            T.job_base = jobs;
            jobs += xt * T.ychunks;
            terms.push_back(T);
        }
        L.nterms = (int)(terms.size() - term_off[sw - 1]);
        L.jobs = jobs;
    }

    // ---- device buffers
    DevBufs bufs(dev);
    const unsigned long long runs_total = [&] {
        unsigned long long r = 0;
        for (const ListPlan& l : lp) r += (l.count + kGenRun - 1) / kGenRun;
        return r;
    }();
    std::vector<CollectListDesc> ld(lp.size());
    const size_t b_rows = rows.size() * 8, b_probe = probe_rows.size() * 4, b_piv = (size_t)m;
    const size_t b_ld = ld.size() * sizeof(CollectListDesc);
    const size_t b_lv = levels.size() * sizeof(CollectLevelDesc);
    const size_t b_tm = std::max<size_t>(1, terms.size()) * sizeof(CollectTerm);
    const size_t b_ctr = (2 + (size_t)maxsw) * 8;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o_rows = 0, o_probe = al(b_rows), o_piv = o_probe + al(b_probe);
    const size_t o_ld = o_piv + al(b_piv), o_lv = o_ld + al(b_ld), o_tm = o_lv + al(b_lv);
    const size_t o_ctr = o_tm + al(b_tm), b_static = o_ctr + al(b_ctr);
    char* d_static = (char*)bufs.get(b_static);
    char* d_lists = (char*)bufs.get(list_bytes);
    if (!d_static || !d_lists) return kErrMemory;
    unsigned long long cap = kFirstCap;
    unsigned long long* d_out = (unsigned long long*)bufs.get(cap * S64 * 8);
    if (!d_out) return kErrMemory;

    for (size_t i = 0; i < lp.size(); ++i) {
        ld[i].probe = (uint32_t*)(d_lists + lp[i].off_p);
        ld[i].pc = (uint8_t*)(d_lists + lp[i].off_c);
        ld[i].count = lp[i].count;
        ld[i].size = lp[i].size;
        ld[i].reflect = lp[i].reflect;
    }
    {
        unsigned long long rb = 0;
        for (size_t i = 0; i < lp.size(); ++i) {
            ld[i].run_base = rb;
            rb += (lp[i].count + kGenRun - 1) / kGenRun;
        }
    }
    // lists with zero entries never own a run; the search over run_base skips them
    for (int sw = 1; sw <= maxsw; ++sw) {
        CollectLevelDesc& L = levels[sw - 1];
        const ListPlan& X = lp[L.a - 1];
        const ListPlan& Y = lp[amax + L.b];
        L.xp = (const uint32_t*)(d_lists + X.off_p);
        L.xpc = (const uint8_t*)(d_lists + X.off_c);
        L.yp = (const uint32_t*)(d_lists + Y.off_p);
        L.ypc = (const uint8_t*)(d_lists + Y.off_c);
        L.terms = (const CollectTerm*)(d_static + o_tm) + term_off[sw - 1];
    }
    std::vector<char> h_static(b_static, 0);
    std::memcpy(h_static.data() + o_rows, rows.data(), b_rows);
    std::memcpy(h_static.data() + o_probe, probe_rows.data(), b_probe);
    std::memcpy(h_static.data() + o_piv, piv.data(), b_piv);
    std::memcpy(h_static.data() + o_ld, ld.data(), b_ld);
    std::memcpy(h_static.data() + o_lv, levels.data(), b_lv);
    if (!terms.empty()) std::memcpy(h_static.data() + o_tm, terms.data(), terms.size() * sizeof(CollectTerm));

    CollectShared S;
    S.probe_rows = (const uint32_t*)(d_static + o_probe);
    S.piv = (const uint8_t*)(d_static + o_piv);
    S.rows = (const unsigned long long*)(d_static + o_rows);
    S.ctr = (unsigned long long*)(d_static + o_ctr);
    S.job_ctr = S.ctr + 2;
    S.m = m; S.S64 = S64; S.HP = HP; S.keep = keep; S.filt = pv.filt;
    const CollectLevelDesc* d_levels = (const CollectLevelDesc*)(d_static + o_lv);

    SessionLease lease(dev);
    Session* s = lease.s;
    if (!s) return kErrDevice;
    cudaStream_t st = s->stream;
    auto fail = [&]() { cudaStreamSynchronize(st); cudaGetLastError(); return kErrDevice; };
    if (cudaMemcpyAsync(d_static, h_static.data(), b_static, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return fail();
    // the session's second event pair brackets the list generation
    if (cudaEventRecord(s->ev_tc0, st) != cudaSuccess) return fail();
    if (launch_collect_gen((const CollectListDesc*)(d_static + o_ld), (int)ld.size(), runs_total, S,
                           dev->d_binom, dev->num_sms, st) != cudaSuccess)
        return fail();
    if (cudaEventRecord(s->ev_tc1, st) != cudaSuccess) return fail();
    H->st.launches = runs_total ? 1 : 0;

    unsigned long long cand_cap = kFirstCand;
    unsigned long long* d_cand = (unsigned long long*)bufs.get(cand_cap * 16);
    if (!d_cand) return kErrMemory;
    unsigned long long h_ctr[2] = {0, 0};
    auto read_ctr = [&]() -> bool {
        return cudaMemcpyAsync(h_ctr, S.ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
               cudaStreamSynchronize(st) == cudaSuccess;
    };
    for (int pass = 0; pass < 2; ++pass) {
        S.out = d_out;
        S.cap = cap;
        S.cand = d_cand;
        S.cand_cap = cand_cap;
        if (cudaMemsetAsync(S.ctr, 0, b_ctr, st) != cudaSuccess) return fail();
        if (cudaEventRecord(s->ev0, st) != cudaSuccess) return fail();
        for (int sw = 1; sw <= maxsw; ++sw) {
            if (levels[sw - 1].jobs == 0) continue;
            if (launch_collect_pairs(d_levels, sw - 1, levels[sw - 1].jobs, S, dev->d_binom,
                                     dev->num_sms, st) != cudaSuccess)
                return fail();
            ++H->st.launches;
        }
        if (launch_collect_exact(d_levels, S, dev->d_binom, dev->num_sms, st) != cudaSuccess)
            return fail();
        ++H->st.launches;
        if (cudaEventRecord(s->ev1, st) != cudaSuccess) return fail();
        if (!read_ctr()) return fail();
        if (pass == 0) {
            float gen_ms = 0.f;
            cudaEventElapsedTime(&gen_ms, s->ev_tc0, s->ev_tc1);
            H->st.gen_ms = gen_ms;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        H->st.pairs_ms = ms;
        if (h_ctr[1] <= cand_cap) break;
        // more candidates than slots (the counter is exact): sweep again into enough slots
        ++H->st.reruns;
        cand_cap = h_ctr[1];
        d_cand = (unsigned long long*)bufs.get(cand_cap * 16);
        if (!d_cand) return kErrMemory;
    }
    if (h_ctr[1] > cand_cap) return kErrDevice;
    if (h_ctr[0] > cap) {
        // more hits than output rows: evaluate the (complete) candidates again into enough rows
        ++H->st.reruns;
        cap = h_ctr[0];
        d_out = (unsigned long long*)bufs.get(cap * S64 * 8);
        if (!d_out) return kErrMemory;
        S.out = d_out;
        S.cap = cap;
        if (cudaMemsetAsync(S.ctr, 0, 8, st) != cudaSuccess) return fail();
        if (launch_collect_exact(d_levels, S, dev->d_binom, dev->num_sms, st) != cudaSuccess)
            return fail();
        ++H->st.launches;
        if (!read_ctr()) return fail();
        if (h_ctr[0] > cap) return kErrDevice;
    }
    const unsigned long long hits = h_ctr[0];
    H->st.hits = (int64_t)hits;
    H->st.passes = (int64_t)h_ctr[1];
    std::vector<uint64_t> out(hits * (size_t)S64);
    if (hits) {
        if (cudaMemcpyAsync(out.data(), d_out, out.size() * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return fail();
        if (cudaStreamSynchronize(st) != cudaSuccess) return fail();
    }
    sort_unique(out, S64, &H->count);
    H->rows.swap(out);
    return kOk;
}

}  // namespace
}  // namespace qsfb

using namespace qsfb;

extern "C" {

void* codeaut_bz_collect(const uint8_t* G, int32_t m, int32_t n, int32_t p, int32_t keep_weight,
                         int32_t backend, int32_t threads) {
    (void)threads;
    const auto t0 = std::chrono::steady_clock::now();
    CollectHandle* H = new (std::nothrow) CollectHandle();
    if (!H) return nullptr;
    H->n = n;
    H->stride = n > 0 ? (n + 63) / 64 : 0;
    // empty problems are complete before any backend is chosen (bz.cpp:60)
    if (m <= 0 || n <= 0 || p <= 0) { H->ok = true; return H; }
    if (!G) { H->st.status = kErrNull; return H; }
    if (backend == 0) { H->st.status = kErrUnsupported; return H; }
    H->backend = "cuda";
    const int maxsw = std::min<int>(p, m);
    for (int sw = 1; sw <= maxsw; ++sw) {
        const long long total = capped_binom(m, sw);
        H->combos = (H->combos > kComboCap - total) ? kComboCap : H->combos + total;
    }
    H->st.combos = H->combos;
    // a nonpositive keep collects nothing (the emit test is 0 < wt <= keep)
    int rc = kOk;
    if (keep_weight > 0) {
        try {
            rc = run_collect(G, m, n, p, keep_weight, H);
        } catch (const std::bad_alloc&) {
            rc = kErrMemory;
        }
    }
    H->st.status = rc;
    H->ok = rc == kOk;
    if (!H->ok) { H->rows.clear(); H->count = 0; }
    H->st.seconds = ms_since(t0) / 1e3;
    return H;
}

int32_t codeaut_bz_ok(void* h) { return h && ((CollectHandle*)h)->ok ? 1 : 0; }
int64_t codeaut_bz_count(void* h) { return h ? ((CollectHandle*)h)->count : -1; }
int64_t codeaut_bz_combos(void* h) { return h ? ((CollectHandle*)h)->combos : -1; }

void codeaut_bz_copy_rows(void* h, uint8_t* buf) {
    CollectHandle* H = (CollectHandle*)h;
    if (!H || !buf) return;
    const int s = H->stride, n = H->n;
    for (long long r = 0; r < H->count; ++r) {
        const uint64_t* src = H->rows.data() + (size_t)r * s;
        uint8_t* dst = buf + (size_t)r * n;
        for (int j = 0; j < n; ++j) dst[j] = (uint8_t)((src[j >> 6] >> (j & 63)) & 1ull);
    }
}

const char* codeaut_bz_backend(void* h) { return h ? ((CollectHandle*)h)->backend.c_str() : ""; }

void codeaut_bz_free(void* h) { delete (CollectHandle*)h; }

int32_t codeaut_backend_available(const char* name) {
    if (!name) return 0;
    const std::string b = name;
    if (b == "gpu" || b == "cuda" || b == "auto") return Device::available() ? 1 : 0;
    return 0;
}

const char* codeaut_version(void) { return "0.1.0"; }

int qsfb_collect_stats(void* h, QsfbCollectStats* out) {
    if (!h || !out) return kErrNull;
    *out = ((CollectHandle*)h)->st;
    return kOk;
}

}  // extern "C"
