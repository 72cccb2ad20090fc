// Host driver of the meet-in-the-middle distance (method "mitm") on the device join of
// mitm.cu.  The level loop, the seed-bound rule and the Z/X interleave keep the reference's
// semantics (cpp/distfind/mitm.cpp:318-552):
//   for d = 1 .. target (seed_upper if set, else the coordinate count): level d hits when
//   some split d = wL + wR matches; the first hit is the distance; with no hit up to a seed
//   target the seed itself is the distance; levels = levels stepped; lower_bound = distance
//   (0 when none); proven = a distance was found.
// Where the reference rebuilds the left hash map for every (d, wL), the table of a left
// weight is built once and probed by every later level (the parts it holds do not depend
// on d), and a level's probes run back to back with one synchronisation.
#include "mitm.hpp"

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "mitm_types.hpp"

namespace qsfb {

cudaError_t launch_mitm_build(const MitmShared& S, const MitmTable& T, int first, int count,
                              int w, unsigned long long n, unsigned long long pw3,
                              const unsigned long long* d_binom, int num_sms, cudaStream_t st);
cudaError_t launch_mitm_probe(const MitmShared& S, const MitmTable& T, int first, int count,
                              int w, unsigned long long n, unsigned long long pw3, int count_all,
                              const unsigned long long* d_binom, int num_sms, cudaStream_t st);

namespace {

constexpr unsigned long long kMaxParts = 1ull << 36;   // parts of one table

unsigned long long pow3(int w) {
    unsigned long long p = 1;
    for (int i = 0; i < w; ++i) p *= 3ull;
    return p;
}

struct DevTable {
    MitmTable t{};
    void* mem = nullptr;
    size_t bytes = 0;
};

// One MITM subproblem stepped level by level (the reference's MitmSide, cpp/distfind/mitm.cpp:403-448).
class MitmSide {
public:
    ~MitmSide() { release(); }

    bool has_logicals = false, sym = false, count_all = false;
    int ncoord = 0, target = 0, seed_upper = 0;
    int found = -1, level = 0;
    bool resolved = false, confirmed = false;
    RunStats stats;

    int setup(Device* d, Session* s, const Problem& p) {
        dev = d;
        sess = s;
        const int K = p.code_gen.rows;
        has_logicals = !(K == 0 || (!p.count_all && p.check.rows == 0));
        if (!has_logicals) { resolved = true; confirmed = true; return kOk; }
        sym = p.symplectic;
        count_all = p.count_all;
        qubits = p.qubits;
        ncoord = sym ? p.qubits : p.n;
        // parts are unranked over the device binomial table (kBinomMaxN + 1 rows)
        if (ncoord > kBinomMaxN) return kErrUnsupported;
        nL = ncoord / 2;
        nR = ncoord - nL;
        seed_upper = p.seed_upper;
        target = seed_upper > 0 ? std::min(seed_upper, ncoord) : ncoord;
        // column views of the parity check H = nullspace(code_gen) and of the detector
        const Mat H = nullspace(p.code_gen);
        const int ncols = p.n;
        SW = (H.rows + 31) / 32;
        LW = count_all ? 0 : (p.check.rows + 31) / 32;
        if (SW > kMitmMaxSynWords || LW > kMitmMaxLogWords) return kErrUnsupported;
        std::vector<uint32_t> cols((size_t)ncols * (SW + LW) + 1, 0u);
        for (int i = 0; i < H.rows; ++i)
            for (int j = 0; j < ncols; ++j)
                if (H.get(i, j)) cols[(size_t)j * SW + (i >> 5)] |= 1u << (i & 31);
        const size_t log_off = (size_t)ncols * SW;
        if (!count_all)
            for (int i = 0; i < p.check.rows; ++i)
                for (int j = 0; j < ncols; ++j)
                    if (p.check.get(i, j)) cols[log_off + (size_t)j * LW + (i >> 5)] |= 1u << (i & 31);
        // the column views, then four status words on a 16-byte boundary
        const size_t status_off = (cols.size() * 4 + 15) / 16 * 16;
        cols_bytes = status_off + 16;
        d_cols = (uint32_t*)dev->alloc(cols_bytes);
        if (!d_cols) return kErrMemory;
        int* st_ptr = (int*)((char*)d_cols + status_off);
        if (cudaMemcpyAsync(d_cols, cols.data(), cols.size() * 4, cudaMemcpyHostToDevice,
                            sess->stream) != cudaSuccess) {
            cudaGetLastError();
            return kErrDevice;
        }
        S.syn_cols = d_cols;
        S.log_cols = d_cols + log_off;
        S.SW = SW;
        S.LW = LW;
        S.sym = sym ? 1 : 0;
        S.qubits = qubits;
        S.status = st_ptr;
        return kOk;
    }

    // Level d: sets *hit; returns a Status.
    int step(int d, bool* hit) {
        ++level;
        *hit = false;
        const auto t0 = std::chrono::steady_clock::now();
        int rc = kOk;
        for (int attempt = 0; attempt < 4; ++attempt) {
            rc = run_level(d, hit);
            if (rc != kRetry) break;
            // two different syndromes shared a 64-bit tag in some table: new seeds
            seed_base += 0x9e3779b97f4a7c15ull;
            for (auto& kv : tables) free_table(kv.second);
            tables.clear();
        }
        if (rc == kRetry) rc = kErrDevice;
        stats.host_plan_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (rc == kOk && *hit) found = d;
        return rc;
    }

private:
    static constexpr int kRetry = -1;
    Device* dev = nullptr;
    Session* sess = nullptr;
    int qubits = 0, nL = 0, nR = 0, SW = 0, LW = 0;
    uint32_t* d_cols = nullptr;
    size_t cols_bytes = 0;
    MitmShared S{};
    std::map<int, DevTable> tables;
    static constexpr unsigned long long kSeed0 = 0x5851f42d4c957f2dull;
    unsigned long long seed_base = kSeed0;
    const bool weak_tags = std::getenv("QSFB_MITM_WEAK_TAGS") != nullptr;

    unsigned long long parts(int count, int w) const {
        const unsigned long long c = dev->binom(count, w);
        if (!sym) return c;
        const unsigned long long p3 = pow3(w);
        if (c != 0 && p3 > ~0ull / c) return ~0ull;
        return c * p3;
    }

    void free_table(DevTable& t) {
        if (t.mem) dev->release(t.mem, t.bytes);
        t.mem = nullptr;
    }

    void release() {
        for (auto& kv : tables) free_table(kv.second);
        tables.clear();
        if (d_cols) dev->release(d_cols, cols_bytes);
        d_cols = nullptr;
    }

    // Build the table of left weight w (parts over coordinates [0, nL)); kRetry on a tag
    // collision.
    int build(int w) {
        const unsigned long long n = parts(nL, w);
        if (n > kMaxParts || w > kMitmMaxWeight) return kErrMemory;
        unsigned long long cap = 2;
        while (cap < n + n / 2 + 1) cap <<= 1;
        const int KW = SW + LW;
        const size_t b_tag = cap * 8, b_key = cap * 4 * (size_t)KW, b_flags = cap * 4;
        DevTable t;
        t.bytes = b_tag + b_key + b_flags + 64;
        t.mem = dev->alloc(t.bytes);
        if (!t.mem) return kErrMemory;
        t.t.tag = (unsigned long long*)t.mem;
        t.t.key = (uint32_t*)((char*)t.mem + b_tag);
        t.t.flags = (uint32_t*)((char*)t.mem + b_tag + b_key);
        t.t.mask = cap - 1;
        t.t.seed = seed_base + (unsigned long long)w * 0x632be59bd9b4e019ull;
        // collision drill: QSFB_MITM_WEAK_TAGS keeps 4 bits of the first seed's tags, so
        // that different syndromes share tags and the rebuild path runs
        t.t.tag_mask = (weak_tags && seed_base == kSeed0) ? 0xfull : ~0ull;
        cudaStream_t st = sess->stream;
        if (cudaMemsetAsync(t.t.tag, 0, b_tag, st) != cudaSuccess ||
            cudaMemsetAsync(t.t.flags, 0, b_flags, st) != cudaSuccess ||
            cudaMemsetAsync(S.status, 0, 16, st) != cudaSuccess ||
            launch_mitm_build(S, t.t, 0, nL, w, n, sym ? pow3(w) : 1ull, dev->d_binom,
                              dev->num_sms, st) != cudaSuccess) {
            cudaGetLastError();
            dev->release(t.mem, t.bytes);
            return kErrDevice;
        }
        stats.launches += 2;
        int status[4] = {0, 0, 0, 0};
        if (cudaMemcpyAsync(status, S.status, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            dev->release(t.mem, t.bytes);
            return kErrDevice;
        }
        tables[w] = t;
        if (status[kMitmOverrun]) return kErrDevice;
        if (status[kMitmCollision]) return kRetry;
        stats.codewords += n;
        return kOk;
    }

    int run_level(int d, bool* hit) {
        // tables first (each build synchronises once to read its collision flag)
        for (int wL = 0; wL <= d; ++wL) {
            const int wR = d - wL;
            if (wL > nL || wR > nR) continue;
            if (tables.count(wL)) continue;
            const int rc = build(wL);
            if (rc != kOk) return rc;
        }
        cudaStream_t st = sess->stream;
        if (cudaMemsetAsync(S.status, 0, 16, st) != cudaSuccess) { cudaGetLastError(); return kErrDevice; }
        for (int wL = 0; wL <= d; ++wL) {
            const int wR = d - wL;
            if (wL > nL || wR > nR) continue;
            const unsigned long long n = parts(nR, wR);
            if (n > (1ull << 50) || wR > kMitmMaxWeight) return kErrMemory;
            if (launch_mitm_probe(S, tables[wL].t, nL, nR, wR, n, sym ? pow3(wR) : 1ull,
                                  count_all ? 1 : 0, dev->d_binom, dev->num_sms, st) != cudaSuccess) {
                cudaGetLastError();
                return kErrDevice;
            }
            ++stats.launches;
            stats.codewords += n;
        }
        int status[4] = {0, 0, 0, 0};
        if (cudaMemcpyAsync(status, S.status, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return kErrDevice;
        }
        if (status[kMitmOverrun]) return kErrDevice;
        *hit = status[kMitmFound] != 0;
        return kOk;
    }
};

void finish(const MitmSide& s, BzResult& r) {
    r.distance = s.found;
    r.levels = s.level;
    r.lower_bound = s.found >= 0 ? s.found : 0;
    r.proven = s.found >= 0;
    r.stats = s.stats;
}

}  // namespace

int mitm_distance(Device* dev, const Problem& p, BzResult& r) {
    const auto t0 = std::chrono::steady_clock::now();
    r = BzResult();
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    MitmSide side;
    int rc = side.setup(dev, lease.s, p);
    if (rc != kOk) return rc;
    if (side.has_logicals) {
        for (int d = 1; d <= side.target; ++d) {
            bool hit = false;
            rc = side.step(d, &hit);
            if (rc != kOk) return rc;
            if (hit) break;
        }
        // stopped at the seed bound without a hit: the seed certifies that weight
        if (side.found < 0 && side.seed_upper > 0 && side.target == side.seed_upper)
            side.found = side.seed_upper;
    }
    finish(side, r);
    r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return kOk;
}

int mitm_min_interleaved(Device* dev, const Problem& pz, const Problem& px, BzResult& r) {
    const auto t0 = std::chrono::steady_clock::now();
    r = BzResult();
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    MitmSide Z, X;
    int rc = Z.setup(dev, lease.s, pz);
    if (rc == kOk) rc = X.setup(dev, lease.s, px);
    if (rc != kOk) return rc;
    // cpp/distfind/mitm.cpp:467-516 with cap_to_min
    MitmSide* sides[2] = {&Z, &X};
    int best = kWeightNone;
    if (Z.has_logicals && Z.seed_upper > 0) best = std::min(best, Z.seed_upper);
    if (X.has_logicals && X.seed_upper > 0) best = std::min(best, X.seed_upper);
    const int maxd = std::max(Z.has_logicals ? Z.target : 0, X.has_logicals ? X.target : 0);
    for (int d = 1; d <= maxd; ++d) {
        for (MitmSide* S : sides) {
            if (S->resolved) continue;
            if (d > S->target) {
                if (S->seed_upper > 0 && S->target == S->seed_upper) {
                    S->found = S->seed_upper;
                    S->confirmed = true;
                    best = std::min(best, S->found);
                }
                S->resolved = true;
                continue;
            }
            if (d >= best) {
                S->confirmed = true;
                if (S->seed_upper > 0 && best == S->seed_upper) S->found = best;
                S->resolved = true;
                continue;
            }
            bool hit = false;
            rc = S->step(d, &hit);
            if (rc != kOk) return rc;
            if (hit) {
                best = std::min(best, d);
                S->confirmed = true;
                S->resolved = true;
            }
        }
        if (Z.resolved && X.resolved) break;
    }
    auto v = [](const MitmSide& s) { return s.found >= 0 ? s.found : kWeightNone; };
    const int dist = std::min(v(Z), v(X));
    r.distance = dist >= kWeightNone ? -1 : dist;
    r.lower_bound = dist >= kWeightNone ? 0 : dist;
    r.levels = std::max(Z.level, X.level);
    r.proven = Z.confirmed && X.confirmed && dist < kWeightNone;
    r.stats = Z.stats;
    r.stats.launches += X.stats.launches;
    r.stats.codewords += X.stats.codewords;
    r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return kOk;
}

}  // namespace qsfb
