// Host side of the device engine: context, allocator, side upload and the level runner.
#include "engine.hpp"
#include "filter_plan.hpp"
#include "tuning.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>

namespace qsfb {

cudaError_t launch_gen_lists(const GenDesc* d_descs, int ndesc, unsigned long long total,
                             const unsigned long long* d_binom, int num_sms, cudaStream_t st);
cudaError_t launch_pairs(int filt, int HP, int mode, const LevelDesc* d, int nd,
                         unsigned long long jobs, unsigned long long* ctr,
                         const unsigned long long* B, int num_sms, cudaStream_t st);
cudaError_t launch_expand_pm(const ExpandDesc* d, int nd, unsigned long long total_rows,
                             int num_sms, cudaStream_t st);
cudaError_t launch_zero_pads(int8_t* const* d_pads, int npads, int num_sms, cudaStream_t st);
cudaError_t launch_pairs_tc(const LevelDesc* d, int nd, unsigned long long jobs,
                            const unsigned long long* B, void* job_recs, int* err, int num_sms,
                            cudaStream_t st);
size_t tc_job_record_bytes();
int tc_tile_rows();
int tc_tile_cols();

namespace {
constexpr unsigned long long kSat = ~0ull;
size_t round_bucket(size_t b) {
    if (b < 256) return 256;
    size_t r = 256;
    while (r < b) r <<= 1;
    return r;
}
size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
constexpr size_t kMinHostStage = 8ull << 20;   // pinned staging of a new session
constexpr size_t kMinSeedStage = 4ull << 20;   // and its seed-trial staging
}  // namespace

// ------------------------------------------------------------------ Device
Device* Device::get(int* rc) {
    static Device* inst = nullptr;
    static int status = -1;
    static std::mutex once;
    std::lock_guard<std::mutex> lk(once);
    if (status < 0) {
        Device* d = new Device();
        status = d->init();
        if (status == kOk) inst = d; else delete d;
    }
    if (rc) *rc = status;
    return inst;
}

bool Device::available() {
    int rc = 0;
    return get(&rc) != nullptr;
}

int Device::init() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return kErrDevice;
    }
    const char* env = std::getenv("QSFB_DEVICE");
    id = env ? std::atoi(env) : 0;
    if (id < 0 || id >= count) return kErrDevice;
    if (cudaSetDevice(id) != cudaSuccess) return kErrDevice;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, id) != cudaSuccess) return kErrDevice;
    // The kernels are built for sm_100a only.
    if (prop.major != 10 || prop.minor != 0) return kErrDevice;
    num_sms = prop.multiProcessorCount;
    name = prop.name;
    // Pool-backed cache misses (QSFB_PLAIN_MALLOC=1: cudaMalloc instead).
    if (!std::getenv("QSFB_PLAIN_MALLOC")) {
        unsigned long long keep = ~0ull;
        if (cudaDeviceGetDefaultMemPool(&pool_, id) != cudaSuccess ||
            cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep) !=
                cudaSuccess ||
            cudaStreamCreateWithFlags(&alloc_stream_, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            pool_ = nullptr;
        }
    }
    const int ld = kBinomMaxK + 1;
    h_binom_.assign((size_t)(kBinomMaxN + 1) * ld, 0ull);
    for (int n = 0; n <= kBinomMaxN; ++n) {
        h_binom_[(size_t)n * ld] = 1ull;
        for (int k = 1; k <= std::min(n, kBinomMaxK); ++k) {
            const unsigned long long a = h_binom_[(size_t)(n - 1) * ld + k - 1];
            const unsigned long long b = (k <= n - 1) ? h_binom_[(size_t)(n - 1) * ld + k] : 0ull;
            h_binom_[(size_t)n * ld + k] = (a == kSat || b == kSat || a > kSat - b) ? kSat : a + b;
        }
    }
    const size_t bytes = h_binom_.size() * sizeof(unsigned long long);
    if (cudaMalloc((void**)&d_binom, bytes) != cudaSuccess) return kErrDevice;
    if (cudaMemcpy(d_binom, h_binom_.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return kErrDevice;
    return kOk;
}

unsigned long long Device::binom(int n, int k) const {
    if (k < 0 || n < 0 || k > n) return 0ull;
    if (n > kBinomMaxN || k > kBinomMaxK) return kSat;
    return h_binom_[(size_t)n * (kBinomMaxK + 1) + k];
}

void* Device::alloc(size_t bytes) {
    // Host-side fault injection for tests: QSFB_FAIL_ALLOC makes every allocation fail
    // (cached blocks included), so callers exercise their out-of-memory paths.
    if (std::getenv("QSFB_FAIL_ALLOC") != nullptr) return nullptr;
    const size_t b = round_bucket(bytes);
    {
        std::lock_guard<std::mutex> lk(mu_);
        // The smallest cached block of this bucket or up to three buckets above it: a miss
        // maps new memory (milliseconds for large blocks, kept by the pool for good), while
        // the number of blocks of one size live at once varies with the timing of
        // concurrent work.  A block keeps its own size through later releases.
        auto it = free_.lower_bound(b);
        if (it != free_.end() && it->first > 8 * b) it = free_.end();
        if (it != free_.end()) {
            void* p = it->second;
            const size_t sz = it->first;
            free_.erase(it);
            cached_ -= sz;
            in_use_ += sz;
            live_[p] = sz;
            return p;
        }
    }
    cudaSetDevice(id);
    void* p = nullptr;
    auto driver_alloc = [&]() -> bool {
        if (!pool_) return cudaMalloc(&p, b) == cudaSuccess;
        if (cudaMallocAsync(&p, b, alloc_stream_) != cudaSuccess) return false;
        return cudaStreamSynchronize(alloc_stream_) == cudaSuccess;
    };
    const double tm0 = now_seconds();
    const bool got = driver_alloc();
    n_device_malloc.fetch_add(1);
    ns_device_malloc.fetch_add((long long)((now_seconds() - tm0) * 1e9));
    if (!got) {
        cudaGetLastError();
        // Drop the cache (after all work that may still use its blocks) and retry once.
        std::multimap<size_t, void*> drop;
        {
            std::lock_guard<std::mutex> lk(mu_);
            drop.swap(free_);
            cached_ = 0;
        }
        cudaDeviceSynchronize();
        for (auto& kv : drop) {
            if (pool_) cudaFreeAsync(kv.second, alloc_stream_);
            else cudaFree(kv.second);
        }
        if (pool_) {
            cudaStreamSynchronize(alloc_stream_);
            cudaMemPoolTrimTo(pool_, 0);
        }
        cudaGetLastError();
        if (!driver_alloc()) {
            cudaGetLastError();
            return nullptr;
        }
    }
    std::lock_guard<std::mutex> lk(mu_);
    in_use_ += b;
    live_[p] = b;
    return p;
}

void Device::reserve(size_t bytes) {
    if (!pool_ || bytes == 0) return;
    cudaSetDevice(id);
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes, alloc_stream_) == cudaSuccess)
        cudaFreeAsync(p, alloc_stream_);   // the pool keeps the memory (release threshold)
    cudaStreamSynchronize(alloc_stream_);
    cudaGetLastError();
}

void Device::release(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu_);
    size_t b = round_bucket(bytes);
    auto it = live_.find(p);
    if (it != live_.end()) {
        b = it->second;
        live_.erase(it);
    }
    free_.emplace(b, p);
    in_use_ -= b;
    cached_ += b;
}

Session* Device::acquire() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (!idle_.empty()) {
            Session* s = idle_.back();
            idle_.pop_back();
            return s;
        }
    }
    cudaSetDevice(id);
    Session* s = new Session();
    s->dev = this;
    int prio_least = 0, prio_greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) != cudaSuccess) {
        cudaGetLastError();
        prio_greatest = 0;
    }
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithPriority(&s->urgent, cudaStreamNonBlocking, prio_greatest) !=
            cudaSuccess ||
        cudaStreamCreateWithPriority(&s->urgent2, cudaStreamNonBlocking,
                                     std::min(prio_least, prio_greatest + 1)) != cudaSuccess ||
        cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess ||
        cudaEventCreate(&s->ev_tc0) != cudaSuccess || cudaEventCreate(&s->ev_tc1) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return nullptr;
    }
    for (int k = 0; k < Session::kAux; ++k)
        if (cudaStreamCreateWithFlags(&s->aux[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->ev_join[k], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            delete s;
            return nullptr;
        }
    // Pinned staging sized up front for a chunk's seed trials and information sets: growing
    // it later (cudaFreeHost + cudaMallocHost, several ms) would stall a preparation that
    // overlaps running rounds.  Sessions are pooled, so this is paid once per session.
    if (s->ensure(0, kMinHostStage) != kOk || s->grow_pinned(s->h_seed, kMinSeedStage) != kOk) {
        delete s;
        return nullptr;
    }
    return s;
}

void Device::give_back(Session* s) {
    std::lock_guard<std::mutex> lk(mu_);
    idle_.push_back(s);
}

int Session::ensure(size_t dbytes, size_t hbytes) {
    if (d_stage.cap < dbytes) {
        if (d_stage.d) dev->release(d_stage.d, d_stage.cap);
        d_stage.cap = round_bucket(dbytes);
        d_stage.d = dev->alloc(d_stage.cap);
        if (!d_stage.d) { d_stage.cap = 0; return kErrMemory; }
    }
    const int rc = grow_pinned(h_stage, hbytes);
    if (rc != kOk) return rc;
    if (!d_ctr.d) {
        d_ctr.cap = 64 * sizeof(unsigned long long);
        d_ctr.d = dev->alloc(d_ctr.cap);
        if (!d_ctr.d) return kErrMemory;
    }
    return kOk;
}

int Session::grow_pinned(HostScratch& hs, size_t hbytes) {
    if (hs.cap >= hbytes) return kOk;
    const double tm0 = now_seconds();
    if (hs.h) cudaFreeHost(hs.h);
    hs.cap = round_bucket(hbytes);
    const cudaError_t he = cudaMallocHost(&hs.h, hs.cap);
    dev->n_pinned_alloc.fetch_add(1);
    dev->ns_pinned_alloc.fetch_add((long long)((now_seconds() - tm0) * 1e9));
    if (he != cudaSuccess) {
        cudaGetLastError();
        hs.h = nullptr;
        hs.cap = 0;
        return kErrMemory;
    }
    return kOk;
}

// ------------------------------------------------------------------ Arena
Arena::~Arena() {
    for (auto& c : chunks_) dev_->release(c.first, c.second);
}

void* Arena::alloc(size_t bytes) {
    std::lock_guard<std::mutex> lk(mu_);
    bytes = align_up(std::max<size_t>(bytes, 16), 256);
    if (chunks_.empty() || used_ + bytes > chunks_.back().second) {
        const size_t sz = round_bucket(std::max<size_t>(bytes, min_chunk_));
        char* p = (char*)dev_->alloc(sz);
        if (!p) return nullptr;
        chunks_.push_back({p, sz});
        used_ = 0;
        total_ += sz;
    }
    char* p = chunks_.back().first + used_;
    used_ += bytes;
    return p;
}

// ------------------------------------------------------------------ SideDev
SideDev::~SideDev() {
    if (!dev) return;
    if (owns) {
        dev->release(d_red, bytes_red);
        dev->release(d_syn, bytes_syn);
    }
    for (auto& kv : lists) {
        if (kv.second.arena) continue;
        dev->release(kv.second.words, kv.second.bytes_w);
        dev->release(kv.second.pc, kv.second.bytes_pc);
        dev->release(kv.second.pm, kv.second.bytes_pm);
    }
}

int SideDev::prepare(const Problem& p, const std::vector<InfoSet>& sets) {
    n = p.n;
    K = p.code_gen.rows;
    ng = (int)sets.size();
    count_all = p.count_all;
    kcheck = p.count_all ? 0 : p.check.rows;
    if (K > kBinomMaxN || ng > 255 || ng == 0) return kErrUnsupported;
    int max_red = 1;
    ranks.resize(ng);
    nonpivot.assign(ng, {});
    for (int g = 0; g < ng; ++g) {
        ranks[g] = sets[g].rank;
        std::vector<char> isp(n, 0);
        for (int c : sets[g].pivots) isp[c] = 1;
        for (int c = 0; c < n; ++c)
            if (!isp[c]) nonpivot[g].push_back(c);
        max_red = std::max(max_red, (int)nonpivot[g].size());
    }
    W32 = (max_red + 31) / 32;
    SW = (kcheck + 31) / 32;
    if (W32 > 32 || SW > 32) return kErrUnsupported;
    const int swp = std::max(SW, 1);
    h_red.assign((size_t)ng * K * W32, 0u);
    h_syn.assign((size_t)ng * K * swp, 0u);
    for (int g = 0; g < ng; ++g) {
        const Mat& G = sets[g].g;
        const std::vector<int>& np = nonpivot[g];
        for (int r = 0; r < K; ++r) {
            uint32_t* o = &h_red[((size_t)g * K + r) * W32];
            const u64* row = G.row(r);
            for (size_t i = 0; i < np.size(); ++i) {
                const int c = np[i];
                if ((row[c >> 6] >> (c & 63)) & 1u) o[i >> 5] |= 1u << (i & 31);
            }
            uint32_t* so = &h_syn[((size_t)g * K + r) * swp];
            for (int c = 0; c < kcheck; ++c)
                if (vec_dot(p.check.row(c), row, G.stride)) so[c >> 5] |= 1u << (c & 31);
        }
    }
    bytes_red = h_red.size() * 4;
    bytes_syn = h_syn.size() * 4;
    return kOk;
}

int SideDev::adopt_device(const Problem& p, const std::vector<InfoSet>& sets, uint32_t* red,
                          uint32_t* syn, int W32_, int SWP, Device* d, Arena* a) {
    n = p.n;
    K = p.code_gen.rows;
    ng = (int)sets.size();
    count_all = p.count_all;
    kcheck = p.count_all ? 0 : p.check.rows;
    if (K > kBinomMaxN || ng > 255 || ng == 0) return kErrUnsupported;
    ranks.resize(ng);
    nonpivot.assign(ng, {});
    for (int g = 0; g < ng; ++g) {
        ranks[g] = sets[g].rank;
        std::vector<char> isp(n, 0);
        for (int c : sets[g].pivots) isp[c] = 1;
        for (int c = 0; c < n; ++c)
            if (!isp[c]) nonpivot[g].push_back(c);
    }
    W32 = W32_;
    SW = (kcheck + 31) / 32;
    if (W32 > 32 || SW > 32 || std::max(SW, 1) != SWP) return kErrUnsupported;
    h_red.clear();
    h_syn.clear();
    bytes_red = (size_t)ng * K * W32 * 4;
    bytes_syn = (size_t)ng * K * SWP * 4;
    dev = d;
    arena = a;
    owns = false;
    d_red = red;
    d_syn = syn;
    device_rows = true;
    return kOk;
}

int SideDev::upload(Device* d, Session* s) {
    dev = d;
    owns = true;
    d_red = (uint32_t*)dev->alloc(bytes_red);
    d_syn = (uint32_t*)dev->alloc(bytes_syn);
    if (!d_red || !d_syn) return kErrMemory;
    if (cudaMemcpyAsync(d_red, h_red.data(), bytes_red, cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaMemcpyAsync(d_syn, h_syn.data(), bytes_syn, cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess) {
        cudaGetLastError();
        return kErrDevice;
    }
    return kOk;
}

int upload_sides(Device* dev, Session* s, Arena* arena, const std::vector<SideDev*>& sides) {
    size_t total = 0;
    for (SideDev* S : sides)
        if (!S->device_rows) total += align_up(S->bytes_red, 256) + align_up(S->bytes_syn, 256);
    if (total == 0) return kOk;
    char* d = (char*)arena->alloc(total);
    if (!d) return kErrMemory;
    int rc = s->ensure(0, total);
    if (rc != kOk) return rc;
    char* h = (char*)s->h_stage.h;
    size_t off = 0;
    for (SideDev* S : sides) {
        if (S->device_rows) continue;   // built in place by the information-set kernel
        S->dev = dev;
        S->arena = arena;
        S->owns = false;
        std::memcpy(h + off, S->h_red.data(), S->bytes_red);
        S->d_red = (uint32_t*)(d + off);
        off += align_up(S->bytes_red, 256);
        std::memcpy(h + off, S->h_syn.data(), S->bytes_syn);
        S->d_syn = (uint32_t*)(d + off);
        off += align_up(S->bytes_syn, 256);
    }
    if (cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess) {
        cudaGetLastError();
        return kErrDevice;
    }
    return kOk;
}

// ------------------------------------------------------------------ level runner
namespace {

int words_of(int bits) { return (bits + 31) / 32; }

// Initial witness key: weight field = bound + 1 (the strict bound), every other bit set.
unsigned long long key_init(int bound) {
    const int f = std::max(0, std::min(bound + 1, 4095));
    return ((unsigned long long)f << kKeyWtShift) | ((1ull << kKeyWtShift) - 1);
}

// QSFB_DEBUG=<level>: diagnostics on stderr (1 failures, 2 plans of heavy levels, 3
// tensor-core launch statistics, 4 planner phase times, 5 pairs by sweep, 6 CUDA-core job
// statistics, 7 a device timeline line per round); read once.
int debug_level() {
    static const int lvl = [] {
        const char* e = std::getenv("QSFB_DEBUG");
        return e ? std::atoi(e) : 0;
    }();
    return lvl;
}

// Rank-deficient sets on the tensor-core sweep (QSFB_TENSOR_RD=0: on the CUDA cores).
bool rd_tensor() {
    static const bool on = [] {
        const char* e = std::getenv("QSFB_TENSOR_RD");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Tensor-core sweep switch: QSFB_TENSOR=0 keeps every level on the CUDA-core kernels.
bool tensor_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("QSFB_TENSOR");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Tensor-core sweep for a full-rank set: worth it when the exact Hamming filter over the
// first 64 non-pivot columns (two K = 32 MMA steps) is clearly cheaper than the CUDA-core
// filter.  Costs are SM cycles per 32768 pairs (one 256 x 128 tile): the four MMAs take
// ~262 cycles, a 64-column slice the filter passes costs ~1300 cycles of exact rescan on
// one of the eight read-back warps; the CUDA-core sweep costs ~2048 cycles per POPC per
// pair, ~1280 in zero-test mode.  Returns the MMA steps (2) or 0.
int tc_depth(int n_enc, int t, int popcs, int* n_live) {
    const int nl = std::min(n_enc, 64);
    // the filter would reject (almost) nothing; up to 32 live columns (one probe word) the
    // +-1 rows carry zeros beyond them, and the 64-column filter is exact over the set's
    // non-pivot columns
    if (nl < 8 || t >= nl / 2) return 0;
    const double pass = hamming_pass_rate(nl, t);
    const double cost = 262.0 + 512.0 * 64.0 * pass * 1300.0 / 8.0;
    const double cc = popcs > 0 ? 2048.0 * popcs : 1280.0;
    if (cost >= tuning().tc_cost_ratio * cc) return 0;
    *n_live = nl;
    return 2;
}

struct Plan {
    int req, g, a, b, filt, popcs, HP, full, mode;
    bool tc = false;                 // tensor-core sweep of terms [p_lo, p_lo + nterms)
    int ksteps = 0, n_live = 0;
    unsigned long long pairs;        // C(K, w) of the level (witness rank width)
    unsigned long long range_pairs;  // pairs of this plan's terms
    int p_lo, nterms;
    int table = -1;                  // term job table (prefix sums, nterms + 1 entries)
    ListBuf* list[2] = {nullptr, nullptr};   // prefix (a) and suffix (b) lists of its set
    unsigned long long jobs;
};

}  // namespace

unsigned long long level_pairs(const Device* dev, int K, int w) { return dev->binom(K, w); }

unsigned long long host_binom(int n, int k) {
    if (k < 0 || n < 0 || k > n) return 0ull;
    k = std::min(k, n - k);   // C(n, i) grows with i up to n/2: the running value never shrinks
    unsigned __int128 r = 1;
    for (int i = 0; i < k; ++i) {
        r = r * (unsigned)(n - i) / (unsigned)(i + 1);   // exact: C(n, i) * (n - i) = C(n, i + 1) * (i + 1)
        if (r >> 64) return kSat;
    }
    return (unsigned long long)r;
}

void level_split(unsigned long long pairs, int w, int* a, int* b) {
    *a = pairs <= (1ull << 14) ? w : (w + 1) / 2;
    *b = w - *a;
}

int level_size_rc(int K, int w) {
    if (w < 1 || w > K || w > kBinomMaxK || K > kBinomMaxN) return kErrUnsupported;
    const unsigned long long pairs = host_binom(K, w);
    if (pairs == kSat || pairs >= (1ull << 62)) return kErrUnsupported;
    int a, b;
    level_split(pairs, w, &a, &b);
    if (host_binom(K, a) > kMaxListEntries || host_binom(K, b) > kMaxListEntries)
        return kErrMemory;
    return kOk;
}

// The reference point of the QSFB_DEBUG=7 timelines: one event, recorded on the stream of
// the first round that asks for it.
static cudaEvent_t timeline_base(cudaStream_t st) {
    static const cudaEvent_t base = [st] {
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        return e;
    }();
    return base;
}

int run_levels(Session* s, const std::vector<LevelReq>& reqs, std::vector<LevelOut>& outs,
               RunStats* stats) {
    Device* dev = s->dev;
    const auto tp0 = std::chrono::steady_clock::now();
    outs.assign(reqs.size(), LevelOut());
    if (reqs.empty()) return kOk;
    const int tcM = tc_tile_rows(), tcN = tc_tile_cols();

    // 1) plan every (request, set); a full-rank set may split into a tensor-core plan for
    //    the terms whose rectangles fill the MMA tiles and CUDA-core plans for the rest
    std::vector<Plan> plans;
    unsigned long long cc_pairs = 0;
    // QSFB_DEBUG=5: pairs of this call by sweep and by why a plan stays on the CUDA cores
    // (rank-deficient, zero test, one probe word, no second list, list over 2^28 entries,
    // the cost model, the terms outside the tensor range)
    unsigned long long why[8] = {0, 0, 0, 0, 0, 0, 0, 0}, tc_sum = 0, edge_lo = 0, edge_hi = 0;
    for (size_t r = 0; r < reqs.size(); ++r) {
        const LevelReq& q = reqs[r];
        SideDev* S = q.side;
        const int K = S->K, w = q.w;
        const int size_rc = level_size_rc(K, w);
        if (size_rc != kOk) return size_rc;
        const unsigned long long pairs = dev->binom(K, w);
        int a, b;
        level_split(pairs, w, &a, &b);
        // tensor-core term range of this level (the same for every set): terms whose
        // rectangles fill at least 1/div of a tile's rows and of its columns (div from the
        // tuning table, 2 by default); nx grows and ny shrinks with p
        int p1 = -1, p2 = -1;
        unsigned long long tc_pairs = 0, lo_pairs = 0, hi_pairs = 0;
        bool range_done = false;
        auto tc_range = [&]() {
            range_done = true;
            const int plo = a - 1, pend = K - b;   // terms p in [plo, pend)
            const int div = tuning().tc_edge_div;
            const unsigned long long min_rows = std::max(1, tcM / div), min_cols = std::max(1, tcN / div);
            int lo = plo, hi = pend;               // first p with nx >= min_rows
            while (lo < hi) {
                const int mid = (lo + hi) / 2;
                if (dev->binom(mid, a - 1) >= min_rows) hi = mid; else lo = mid + 1;
            }
            int l2 = plo - 1, h2 = pend - 1;       // last p with ny >= min_cols
            while (l2 < h2) {
                const int mid = (l2 + h2 + 1) / 2;
                if (dev->binom(K - 1 - mid, b) >= min_cols) l2 = mid; else h2 = mid - 1;
            }
            if (lo > l2) return;
            p1 = lo;
            p2 = l2;
            for (int p = plo; p < p1; ++p) lo_pairs += dev->binom(p, a - 1) * dev->binom(K - 1 - p, b);
            for (int p = p2 + 1; p < pend; ++p) hi_pairs += dev->binom(p, a - 1) * dev->binom(K - 1 - p, b);
            tc_pairs = pairs - lo_pairs - hi_pairs;
        };
        for (int g = 0; g < q.active; ++g) {
            Plan P;
            P.req = (int)r; P.g = g; P.a = a; P.b = b;
            const int rank = S->ranks[g];
            const int nred = (int)S->nonpivot[g].size();
            const int wg = std::max(1, words_of(nred));
            P.HP = wg >= 3 ? 4 : wg;
            P.full = rank == K;
            // mode: 0 rank-deficient, 1 full rank, 2 full rank with no room above the
            // pivot bits (every candidate needs an all-zero non-pivot part)
            const int T = std::max(0, std::min(q.bound + 1, 4095));
            const int pcmin = std::max(0, w - (K - rank));
            P.mode = !P.full ? 0 : (T - 1 - w <= 0 ? 2 : 1);
            const FilterChoice fc = choose_filter(P.HP, nred, T - 1 - pcmin, P.mode == 2);
            P.filt = fc.filt;
            P.popcs = fc.popcs;
            P.pairs = pairs;
            P.p_lo = a - 1;
            P.nterms = K - b - a + 1;
            int ks = 0, nl = 0;
            // (+-1 lists hold 64 bytes per entry: keep them, and their 32-bit row indices, modest)
            // a rank-deficient set: the sweep adds each prefix entry's own pivot-row count and
            // the fewest a suffix entry can hold, b - (K - rank); for the cost model a prefix
            // entry typically holds all a of its rows as pivots
            const int rd_allow = T - 1 - (a + std::max(0, b - (K - rank)));
            if (tensor_enabled() && b > 0 && (P.full || rd_tensor()) &&
                dev->binom(K, a) < (1ull << 28) && dev->binom(K, b) < (1ull << 28))
                ks = tc_depth(nred, P.full ? T - 1 - w : rd_allow, P.popcs, &nl);
            if (debug_level() == 2 && pairs > (1ull << 26))
                std::fprintf(stderr, "qsfb plan: K=%d w=%d a=%d b=%d nred=%d rank=%d HP=%d T=%d "
                             "mode=%d filt=%d ks=%d\n", K, w, a, b, nred, rank, P.HP, T, P.mode,
                             P.filt, ks);
            if (ks > 0 && !range_done) tc_range();
            if (ks == 0 || p1 < 0) {
                P.range_pairs = pairs;
                cc_pairs += pairs;
                if (debug_level() == 5)
                    why[!P.full ? 0 : P.mode == 2 ? 1 : P.HP < 2 ? 2 : b == 0 ? 3
                        : (dev->binom(K, a) >= (1ull << 28) || dev->binom(K, b) >= (1ull << 28)) ? 4
                        : ks == 0 ? 5 : 6] += pairs;
                plans.push_back(std::move(P));
                continue;
            }
            if (debug_level() == 5) {
                why[6] += lo_pairs + hi_pairs;
                edge_lo += lo_pairs;
                edge_hi += hi_pairs;
                tc_sum += tc_pairs;
            }
            const int p_end = P.p_lo + P.nterms;   // one past the last term
            Plan TP = P;
            TP.tc = true;
            TP.ksteps = ks;
            TP.n_live = nl;
            TP.p_lo = p1;
            TP.nterms = p2 - p1 + 1;
            TP.range_pairs = tc_pairs;
            if (p1 > P.p_lo) {
                Plan L = P;
                L.nterms = p1 - P.p_lo;
                L.range_pairs = lo_pairs;
                cc_pairs += lo_pairs;
                plans.push_back(std::move(L));
            }
            if (p2 + 1 < p_end) {
                Plan R = P;
                R.p_lo = p2 + 1;
                R.nterms = p_end - R.p_lo;
                R.range_pairs = hi_pairs;
                cc_pairs += hi_pairs;
                plans.push_back(std::move(R));
            }
            plans.push_back(std::move(TP));
        }
    }
    if (debug_level() == 5)
        std::fprintf(stderr, "qsfb plan pairs: tc %llu | cc rank-deficient %llu zero-test %llu "
                     "one-word %llu one-list %llu big-list %llu cost-model %llu edge-terms %llu "
                     "(few prefix rows %llu, few suffix columns %llu)\n",
                     tc_sum, why[0], why[1], why[2], why[3], why[4], why[5], why[6], edge_lo,
                     edge_hi);
    // loop tile: enough jobs to keep every resident warp busy several times over
    // ~16 jobs per resident warp: the launch tail (one job) stays a few % of the level
    const unsigned long long want_jobs =
        (unsigned long long)dev->num_sms * 24 * (unsigned long long)tuning().cc_jobs_per_warp;
    unsigned long long lt = cc_pairs / ((unsigned long long)kRegTile * want_jobs);
    lt = std::max<unsigned long long>(32, std::min<unsigned long long>(1024, lt));
    const int loop_tile = (int)((lt + 31) / 32 * 32);

    const auto tp1 = std::chrono::steady_clock::now();
    // 2) lists to build: packed probe words for every plan, +-1 rows for tensor plans
    // A list generated in this call writes its +-1 rows in the same pass when a tensor plan
    // needs them; a list generated earlier gets them from the expansion kernel.
    struct GenReq {
        SideDev* S;
        int g, size, reflect, HP;
        bool pm;
        int n_enc;
        unsigned long long pm_lo, pm_hi;
        const ListBuf* src = nullptr;   // complete list one size smaller (built from it)
    };
    // The list one size smaller of the same set and orientation, when an earlier round left
    // it complete (ready and not being rebuilt in this call): the new list is built from it
    // by one XOR per entry instead of unranking.  Its pivot counts are needed when the new
    // list stores them.
    auto smaller_list = [](SideDev* S, int g, int size, int side, bool full) -> const ListBuf* {
        if (size < 2) return nullptr;
        auto it = S->lists.find(std::make_tuple(g, size - 1, side));
        if (it == S->lists.end()) return nullptr;
        const ListBuf& L = it->second;
        if (!L.ready || L.queued || !L.words || (!full && !L.pc)) return nullptr;
        return &L;
    };
    struct ExpReq {
        SideDev* S;
        int g, size, reflect, HP, n_enc;
        unsigned long long lo, hi;
    };
    std::vector<GenReq> gens;
    std::vector<ExpReq> exps;
    std::vector<int8_t*> pad_zero;   // new +-1 buffers: their kPmPadRows tail rows, zeroed
    // the `queued` marks only live for this call, whatever path it leaves by
    struct ClearQueued {
        std::vector<GenReq>& g;
        std::vector<ExpReq>& e;
        ~ClearQueued() {
            for (const GenReq& G : g) {
                ListBuf& L = G.S->lists[std::make_tuple(G.g, G.size, G.reflect)];
                L.queued = L.pm_queued = false;
                L.gen_idx = -1;
            }
            for (const ExpReq& E : e) {
                ListBuf& L = E.S->lists[std::make_tuple(E.g, E.size, E.reflect)];
                L.pm_queued = false;
                L.exp_idx = -1;
            }
        }
    } clear_queued{gens, exps};
    // per list, the hull of the +-1 rows this call's tensor plans read (operand bytes)
    std::unordered_map<const ListBuf*, std::pair<unsigned long long, unsigned long long>> tc_rows;
    for (Plan& P : plans) {
        SideDev* S = reqs[P.req].side;
        for (int side = 0; side < 2; ++side) {
            const int size = side == 0 ? P.a : P.b;   // b = 0: one empty entry
            auto key = std::make_tuple(P.g, size, side);
            ListBuf& L = S->lists[key];   // map nodes are stable: kept in the plan
            P.list[side] = &L;
            if (!(L.ready || L.queued)) {
                if (L.words) {   // allocated by an earlier execution: regenerate in place
                    L.queued = true;
                    L.gen_idx = (int)gens.size();
                    gens.push_back({S, P.g, size, side, P.HP, false, 0, 0, 0,
                                    smaller_list(S, P.g, size, side, P.full)});
                } else {
                    L.queued = true;
                    L.count = dev->binom(S->K, size);
                    L.bytes_w = std::max<size_t>((size_t)L.count * P.HP * 4, 16);
                    L.arena = S->arena != nullptr;
                    L.words = (uint32_t*)(L.arena ? S->arena->alloc(L.bytes_w) : dev->alloc(L.bytes_w));
                    if (!L.words) { L.queued = false; return kErrMemory; }
                    if (!P.full) {
                        L.bytes_pc = std::max<size_t>((size_t)L.count, 16);
                        L.pc = (uint8_t*)(L.arena ? S->arena->alloc(L.bytes_pc) : dev->alloc(L.bytes_pc));
                        if (!L.pc) { L.queued = false; return kErrMemory; }
                    }
                    S->list_bytes += L.bytes_w + L.bytes_pc;
                    L.gen_idx = (int)gens.size();
                    gens.push_back({S, P.g, size, side, P.HP, false, 0, 0, 0,
                                    smaller_list(S, P.g, size, side, P.full)});
                }
            }
            if (!P.tc) continue;
            // +-1 rows this tensor plan reads: the prefix blocks of its terms, and the
            // suffix prefix of its first term plus one tile (columns past a term's end
            // must hold real entries or zeros, not stale memory)
            unsigned long long n_lo, n_hi;
            if (side == 0) {
                n_lo = dev->binom(P.p_lo, P.a);
                n_hi = dev->binom(P.p_lo + P.nterms, P.a);
            } else {
                n_lo = 0;
                n_hi = std::min(L.count, dev->binom(S->K - 1 - P.p_lo, P.b) + (unsigned long long)tcN);
            }
            {
                auto ins = tc_rows.emplace(&L, std::make_pair(n_lo, n_hi));
                if (!ins.second) {
                    ins.first->second.first = std::min(ins.first->second.first, n_lo);
                    ins.first->second.second = std::max(ins.first->second.second, n_hi);
                }
            }
            if (L.pm_ready && n_lo >= L.pm_lo && n_hi <= L.pm_hi) continue;   // already written
            if (!L.pm) {
                L.bytes_pm = (size_t)(L.count + kPmPadRows) * kPmRowBytes;
                L.pm = (int8_t*)(L.arena ? S->arena->alloc(L.bytes_pm) : dev->alloc(L.bytes_pm));
                if (!L.pm) return kErrMemory;
                S->list_bytes += L.bytes_pm;
                pad_zero.push_back(L.pm + (size_t)L.count * kPmRowBytes);
            }
            const int nred = (int)S->nonpivot[P.g].size();
            const int n_enc = std::min(nred, kPmRowBytes);
            if (L.queued && L.gen_idx >= 0) {   // generated in this call: fused, hull of needs
                GenReq& G = gens[L.gen_idx];
                if (!G.pm) {
                    G.pm = true;
                    G.n_enc = n_enc;
                    G.pm_lo = n_lo;
                    G.pm_hi = n_hi;
                } else {
                    G.pm_lo = std::min(G.pm_lo, n_lo);
                    G.pm_hi = std::max(G.pm_hi, n_hi);
                }
                L.pm_queued = true;
            } else {   // built earlier: expand the hull of what is written and what is needed
                if (L.pm_ready) {
                    n_lo = std::min(n_lo, L.pm_lo);
                    n_hi = std::max(n_hi, L.pm_hi);
                }
                if (L.pm_queued && L.exp_idx >= 0) {
                    ExpReq& E = exps[L.exp_idx];
                    E.lo = std::min(E.lo, n_lo);
                    E.hi = std::max(E.hi, n_hi);
                } else {
                    L.exp_idx = (int)exps.size();
                    exps.push_back({S, P.g, size, side, P.HP, n_enc, n_lo, n_hi});
                    L.pm_queued = true;
                }
            }
        }
    }

    const auto tp2 = std::chrono::steady_clock::now();
    // 3) term tables and job counts, shared by every plan with the same level shape (K, a,
    //    b), sweep and term range: sets of a level and levels of equal shape across codes
    //    differ only in their lists
    unsigned long long tc_jobs = 0;
    std::vector<std::vector<unsigned long long>> tables;
    std::vector<int> table_jb;                              // tensor-core job tiles per table
    std::unordered_map<unsigned long long, int> table_of;   // packed (K, a, b, tc, p_lo, nterms)
    for (Plan& P : plans) {
        const unsigned long long tkey =
            ((unsigned long long)reqs[P.req].side->K << 42) | ((unsigned long long)P.a << 35) |
            ((unsigned long long)P.b << 28) | ((unsigned long long)(P.tc ? 1 : 0) << 27) |
            ((unsigned long long)P.p_lo << 14) | (unsigned long long)P.nterms;
        auto it = table_of.find(tkey);
        if (it == table_of.end()) {
            const int K = reqs[P.req].side->K;
            std::vector<unsigned long long> tj(P.nterms + 1, 0ull);
            unsigned long long acc = 0;
            // tensor-core plans: suffix tiles per job by the level's size class (tuned)
            int jb = 0;
            if (P.tc) {
                unsigned long long tiles = 0;
                for (int t = 0; t < P.nterms; ++t) {
                    const int p = P.p_lo + t;
                    const unsigned long long xoff = dev->binom(p, P.a);
                    const unsigned long long na = ((xoff & 7ull) + dev->binom(p, P.a - 1) + tcM - 1) / tcM;
                    tiles += na * ((dev->binom(K - 1 - p, P.b) + tcN - 1) / tcN);
                }
                jb = tc_job_tiles_for(tiles);
            }
            for (int t = 0; t < P.nterms; ++t) {
                const int p = P.p_lo + t;
                const unsigned long long nx = dev->binom(p, P.a - 1);
                const unsigned long long ny = dev->binom(K - 1 - p, P.b);
                tj[t] = acc;
                if (P.tc) {
                    // prefix tiles from the 8-aligned start of the block x suffix-tile chunks
                    const unsigned long long xoff = dev->binom(p, P.a);
                    const unsigned long long na = ((xoff & 7ull) + nx + tcM - 1) / tcM;
                    const unsigned long long nbt = (ny + tcN - 1) / tcN;
                    acc += na * ((nbt + jb - 1) / jb);
                } else {
                    const unsigned long long rn = std::max(nx, ny), ln = std::min(nx, ny);
                    acc += ((rn + kRegTile - 1) / kRegTile) * ((ln + loop_tile - 1) / loop_tile);
                }
            }
            tj[P.nterms] = acc;
            it = table_of.emplace(tkey, (int)tables.size()).first;
            tables.push_back(std::move(tj));
            table_jb.push_back(jb);
        }
        P.table = it->second;
        P.jobs = tables[P.table].back();
        if (P.tc) tc_jobs += P.jobs;
    }
    if (tc_jobs && debug_level() == 3) {
        unsigned long long tiles = 0, pairs = 0, atiles = 0;
        for (const Plan& P : plans) {
            if (!P.tc) continue;
            const int K = reqs[P.req].side->K;
            for (int t = 0; t < P.nterms; ++t) {
                const int p = P.p_lo + t;
                const unsigned long long nx = dev->binom(p, P.a - 1), ny = dev->binom(K - 1 - p, P.b);
                const unsigned long long xoff = dev->binom(p, P.a);
                const unsigned long long na = ((xoff & 7ull) + nx + tcM - 1) / tcM;
                tiles += na * ((ny + tcN - 1) / tcN);
                const unsigned long long jb = (unsigned long long)table_jb[P.table];
                atiles += na * ((((ny + tcN - 1) / tcN) + jb - 1) / jb);
                pairs += nx * ny;
            }
        }
        std::fprintf(stderr, "qsfb tc launch: jobs=%llu tiles=%llu pairs=%llu tile_util=%.3f tiles_per_job=%.2f\n",
                     tc_jobs, tiles, pairs, (double)pairs / ((double)tiles * tcM * tcN),
                     (double)tiles / (double)tc_jobs);
    }

    if (debug_level() == 6) {   // CUDA-core jobs of this call: how many, how big, how short
        unsigned long long jobs = 0, pairs = 0, sjobs = 0, spairs = 0;
        for (const Plan& P : plans) {
            if (P.tc) continue;
            const int K = reqs[P.req].side->K;
            for (int t = 0; t < P.nterms; ++t) {
                const int p = P.p_lo + t;
                const unsigned long long nx = dev->binom(p, P.a - 1), ny = dev->binom(K - 1 - p, P.b);
                const unsigned long long rn = std::max(nx, ny), ln = std::min(nx, ny);
                const unsigned long long j = ((rn + kRegTile - 1) / kRegTile) *
                                             ((ln + loop_tile - 1) / loop_tile);
                jobs += j;
                pairs += nx * ny;
                if (ln < (unsigned long long)loop_tile / 4) { sjobs += j; spairs += nx * ny; }
            }
        }
        if (jobs)
            std::fprintf(stderr, "qsfb cc launch: jobs=%llu pairs=%llu loop_tile=%d pairs_per_job=%.0f "
                         "short-loop (< tile/4) jobs=%llu pairs=%llu pairs_per_job=%.0f\n",
                         jobs, pairs, loop_tile, (double)pairs / (double)jobs, sjobs, spairs,
                         sjobs ? (double)spairs / (double)sjobs : 0.0);
    }

    // launch groups: CUDA-core variants (filter, HP, mode), then one tensor-core group
    std::vector<int> order(plans.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return std::make_tuple(plans[x].tc, plans[x].filt, plans[x].HP, plans[x].mode) <
               std::make_tuple(plans[y].tc, plans[y].filt, plans[y].HP, plans[y].mode);
    });

    const auto tp3 = std::chrono::steady_clock::now();
    // 4) staging layout
    const size_t nplans = plans.size();
    size_t off = 0;
    const size_t off_gen = off;
    off = align_up(off + gens.size() * sizeof(GenDesc), 64);
    const size_t off_exp = off;
    off = align_up(off + exps.size() * sizeof(ExpandDesc), 64);
    const size_t off_lvl = off;
    off = align_up(off + nplans * sizeof(LevelDesc), 64);
    const size_t off_terms = off;
    size_t terms_total = 0;
    for (const auto& tj : tables) terms_total += tj.size();
    off = align_up(off + terms_total * 8, 64);
    const size_t off_keys = off;
    off = align_up(off + reqs.size() * 8, 64);
    const size_t off_counts = off;
    off = off + nplans * 8;
    const size_t off_err = off;
    off = align_up(off + 8, 64);
    const size_t off_pads = off;                    // new +-1 lists' pad areas to zero
    off = align_up(off + pad_zero.size() * sizeof(int8_t*), 64);
    const size_t total_bytes = off;                 // host-written part
    const size_t off_recs = off;                    // device-only: decoded tensor-core jobs
    off = align_up(off + tc_jobs * tc_job_record_bytes(), 64);
    int rc = s->ensure(off, total_bytes);
    if (rc != kOk) return rc;
    char* h = (char*)s->h_stage.h;
    char* d = (char*)s->d_stage.d;
    std::memset(h, 0, total_bytes);

    GenDesc* hg = (GenDesc*)(h + off_gen);
    unsigned long long gen_total = 0;
    unsigned long long list_written = 0;   // algorithmic bytes of the list generation
    for (size_t i = 0; i < gens.size(); ++i) {
        const GenReq& G = gens[i];
        ListBuf& L = G.S->lists[std::make_tuple(G.g, G.size, G.reflect)];
        GenDesc& D = hg[i];
        D.red = G.S->d_red + (size_t)G.g * G.S->K * G.S->W32;
        D.out = L.words;
        D.pc = L.pc;
        D.pm = G.pm ? L.pm : nullptr;
        D.n_enc = G.n_enc;
        D.pm_lo = G.pm_lo;
        D.pm_hi = G.pm_hi;
        D.entry_base = gen_total;   // in runs of kGenRun entries
        D.count = L.count;
        D.K = G.S->K;
        D.size = G.size;
        D.W32 = G.S->W32;
        D.HP = G.HP;
        D.rank = G.S->ranks[G.g];
        D.reflect = G.reflect;
        D.src = G.src ? G.src->words : nullptr;
        D.src_pc = G.src ? G.src->pc : nullptr;
        gen_total += (L.count + kGenRun - 1) / kGenRun;
        list_written += L.count * (unsigned long long)G.HP * 4 + (L.pc ? L.count : 0) +
                        (G.pm ? (G.pm_hi - G.pm_lo) * kPmRowBytes : 0);
    }
    ExpandDesc* he = (ExpandDesc*)(h + off_exp);
    unsigned long long exp_total = 0;
    for (size_t i = 0; i < exps.size(); ++i) {
        const ExpReq& E = exps[i];
        ListBuf& L = E.S->lists[std::make_tuple(E.g, E.size, E.reflect)];
        ExpandDesc& D = he[i];
        D.words = L.words;
        D.out = L.pm;
        D.row_base = exp_total;
        D.count = L.count;
        D.row_lo = E.lo;
        D.rows = E.hi - E.lo;
        D.HP = E.HP;
        D.n_enc = E.n_enc;
        exp_total += D.rows;
        list_written += D.rows * kPmRowBytes;
    }

    int8_t** hpads = (int8_t**)(h + off_pads);
    for (size_t i = 0; i < pad_zero.size(); ++i) hpads[i] = pad_zero[i];

    unsigned long long* hkeys = (unsigned long long*)(h + off_keys);
    for (size_t r = 0; r < reqs.size(); ++r)
        hkeys[r] = key_init(reqs[r].bound);

    LevelDesc* hl = (LevelDesc*)(h + off_lvl);
    unsigned long long* hterms = (unsigned long long*)(h + off_terms);
    std::vector<size_t> table_off(tables.size());
    {
        size_t cur = 0;
        for (size_t i = 0; i < tables.size(); ++i) {
            std::memcpy(hterms + cur, tables[i].data(), tables[i].size() * 8);
            table_off[i] = cur;
            cur += tables[i].size();
        }
    }
    struct Group { bool tc; int filt, HP, mode, first, count; unsigned long long jobs; };
    std::vector<Group> groups;
    for (size_t oi = 0; oi < order.size(); ++oi) {
        const Plan& P = plans[order[oi]];
        if (groups.empty() || groups.back().tc != P.tc ||
            (!P.tc && (groups.back().filt != P.filt || groups.back().HP != P.HP ||
                       groups.back().mode != P.mode)))
            groups.push_back({P.tc, P.filt, P.HP, P.mode, (int)oi, 0, 0ull});
        Group& Gp = groups.back();
        SideDev* S = reqs[P.req].side;
        LevelDesc& D = hl[oi];
        const ListBuf& La = *P.list[0];
        const ListBuf& Rb = *P.list[1];
        D.red = S->d_red + (size_t)P.g * S->K * S->W32;
        D.syn = S->d_syn + (size_t)P.g * S->K * std::max(S->SW, 1);
        D.la = La.words;
        D.pca = La.pc;
        D.rb = Rb.words;
        D.pcb = Rb.pc;
        D.term_jobs = (const uint64_t*)(d + off_terms + table_off[P.table] * 8);
        D.key = (unsigned long long*)(d + off_keys + (size_t)P.req * 8);
        D.count = (unsigned long long*)(d + off_counts + (size_t)order[oi] * 8);
        D.job_base = Gp.jobs;
        D.K = S->K; D.w = reqs[P.req].w; D.a = P.a; D.b = P.b;
        D.W32 = S->W32; D.SW = S->SW; D.HP = P.HP;
        D.rank = S->ranks[P.g];
        D.g = P.g;
        D.p_lo = P.p_lo;
        D.nterms = P.nterms;
        D.loop_tile = loop_tile;
        int bits = 0;
        while (bits < 64 && (P.pairs - 1) >> bits) ++bits;
        D.rank_shift = std::max(0, bits - kKeyGShift);
        D.count_all = S->count_all ? 1 : 0;
        D.tc_job_tiles = 0;
        if (P.tc) {
            D.ksteps = P.ksteps;
            D.n_live = P.n_live;
            D.xpm = La.pm;
            D.ypm = Rb.pm;
            D.tc_job_tiles = table_jb[P.table];
        }
        Gp.jobs += P.jobs;
        Gp.count += 1;
    }
    if (groups.size() > 64) return kErrUnsupported;

    // 5) launch
    if (debug_level() == 4) {
        const auto tp4 = std::chrono::steady_clock::now();
        auto us = [](std::chrono::steady_clock::time_point x, std::chrono::steady_clock::time_point y) {
            return std::chrono::duration<double, std::micro>(y - x).count();
        };
        std::fprintf(stderr, "qsfb plan: reqs=%zu plans=%zu gens=%zu exps=%zu tables=%zu | plan %.0f us, lists %.0f us, "
                     "terms %.0f us, staging %.0f us\n", reqs.size(), plans.size(), gens.size(),
                     exps.size(), tables.size(), us(tp0, tp1), us(tp1, tp2), us(tp2, tp3), us(tp3, tp4));
    }
    if (stats)
        stats->host_plan_s +=
            std::chrono::duration<double>(std::chrono::steady_clock::now() - tp0).count();
    cudaStream_t st = s->stream;
    // QSFB_DEBUG=7: this round's device timeline (staging copy, end of list generation,
    // tensor sweep, join) against one base event of the process, a line per round
    const bool timeline = debug_level() == 7;
    const double plan_ms =
        1e3 * std::chrono::duration<double>(std::chrono::steady_clock::now() - tp0).count();
    cudaEvent_t tl[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    if (timeline) {
        timeline_base(st);
        for (cudaEvent_t& e : tl) cudaEventCreate(&e);
        cudaEventRecord(tl[0], st);
    }
    if (cudaMemcpyAsync(d, h, total_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(s->d_ctr.d, 0, s->d_ctr.cap, st) != cudaSuccess) {
        cudaGetLastError();
        return kErrDevice;
    }
    // one launch for every new +-1 list's pad rows (a memset per list cost a launch each,
    // thousands in a batch's first execution)
    if (launch_zero_pads((int8_t* const*)(d + off_pads), (int)pad_zero.size(), dev->num_sms,
                         st) != cudaSuccess) {
        cudaGetLastError();
        return kErrDevice;
    }
    cudaEventRecord(s->ev0, st);
    int launches = 0;
    if (!gens.empty()) {
        if (launch_gen_lists((const GenDesc*)(d + off_gen), (int)gens.size(), gen_total,
                             dev->d_binom, dev->num_sms, st) != cudaSuccess)
            return kErrDevice;
        ++launches;
    }
    if (!exps.empty()) {
        if (launch_expand_pm((const ExpandDesc*)(d + off_exp), (int)exps.size(), exp_total,
                             dev->num_sms, st) != cudaSuccess)
            return kErrDevice;
        ++launches;
    }
    cudaEvent_t evm;
    cudaEventCreate(&evm);
    cudaEventRecord(evm, st);
    if (timeline) cudaEventRecord(tl[1], st);
    // fork: the pair launches (independent levels; they share only the atomic witness keys)
    // go round-robin over the auxiliary streams, the tensor-core sweep first.
    // QSFB_SERIAL_PAIRS (read per call): all on one stream, so that each kernel's events
    // time it alone (benchmarks' per-kernel statistics).
    const bool serial_pairs = std::getenv("QSFB_SERIAL_PAIRS") != nullptr;
    cudaEventRecord(s->ev_fork, st);
    for (int k = 0; k < Session::kAux; ++k) cudaStreamWaitEvent(s->aux[k], s->ev_fork, 0);
    unsigned long long all_jobs = 0;
    bool tc_timed = false;
    int next_aux = 0;
    for (size_t gi0 = 0; gi0 < groups.size(); ++gi0) {
        // tensor-core group (sorted last) launched first
        const size_t gi = (groups.back().tc ? (gi0 == 0 ? groups.size() - 1 : gi0 - 1) : gi0);
        const Group& Gp = groups[gi];
        const LevelDesc* gd = (const LevelDesc*)(d + off_lvl) + Gp.first;
        cudaStream_t gs = s->aux[serial_pairs ? 0 : next_aux];
        next_aux = (next_aux + 1) % Session::kAux;
        if (Gp.tc) cudaEventRecord(s->ev_tc0, gs);
        if (Gp.tc && timeline) cudaEventRecord(tl[2], gs);
        const cudaError_t e =
            Gp.tc ? launch_pairs_tc(gd, Gp.count, Gp.jobs, dev->d_binom, d + off_recs,
                                    (int*)(d + off_err), dev->num_sms, gs)
                  : launch_pairs(Gp.filt, Gp.HP, Gp.mode, gd, Gp.count, Gp.jobs,
                                 (unsigned long long*)s->d_ctr.d + gi, dev->d_binom,
                                 dev->num_sms, gs);
        if (e != cudaSuccess) {
            if (debug_level() >= 1)
                std::fprintf(stderr, "qsfb: pair launch failed: %s\n", cudaGetErrorString(e));
            cudaGetLastError();
            // nothing launched so far may still run when the staging is reused
            for (int k = 0; k < Session::kAux; ++k) cudaStreamSynchronize(s->aux[k]);
            cudaGetLastError();
            cudaEventDestroy(evm);
            return kErrDevice;
        }
        if (Gp.tc) {
            cudaEventRecord(s->ev_tc1, gs);
            if (timeline) cudaEventRecord(tl[3], gs);
            tc_timed = true;
            launches += 1;   // the job-decode kernel
        }
        ++launches;
        all_jobs += Gp.jobs;
    }
    // join
    for (int k = 0; k < Session::kAux; ++k) {
        cudaEventRecord(s->ev_join[k], s->aux[k]);
        cudaStreamWaitEvent(st, s->ev_join[k], 0);
    }
    cudaEventRecord(s->ev1, st);
    if (timeline) cudaEventRecord(tl[4], st);
    cudaError_t se = cudaMemcpyAsync(h + off_keys, d + off_keys, off_err + 8 - off_keys,
                                     cudaMemcpyDeviceToHost, st);
    if (se == cudaSuccess) se = cudaStreamSynchronize(st);
    if (se != cudaSuccess) {
        if (debug_level() >= 1)
            std::fprintf(stderr, "qsfb: level run failed: %s\n", cudaGetErrorString(se));
        cudaGetLastError();
        cudaEventDestroy(evm);
        return kErrDevice;
    }
    if (*(const int*)(h + off_err) != 0) {   // a tensor-core wait ran out
        if (debug_level() >= 1)
            std::fprintf(stderr, "qsfb: tensor-core sweep wait ran out (role %d)\n",
                         *(const int*)(h + off_err));
        cudaEventDestroy(evm);
        return kErrDevice;
    }
    for (const GenReq& G : gens) {
        ListBuf& L = G.S->lists[std::make_tuple(G.g, G.size, G.reflect)];
        L.ready = true;
        L.queued = false;
        L.gen_idx = -1;
        if (G.pm) {
            L.pm_ready = true;
            L.pm_queued = false;
            L.pm_lo = G.pm_lo;
            L.pm_hi = G.pm_hi;
        }
    }
    for (const ExpReq& E : exps) {
        ListBuf& L = E.S->lists[std::make_tuple(E.g, E.size, E.reflect)];
        L.pm_ready = true;
        L.pm_queued = false;
        L.exp_idx = -1;
        L.pm_lo = E.lo;
        L.pm_hi = E.hi;
    }

    // 6) decode
    unsigned long long* hcounts = (unsigned long long*)(h + off_counts);
    unsigned long long cw = 0;
    for (size_t r = 0; r < reqs.size(); ++r) {
        LevelOut& O = outs[r];
        O.counts.assign(reqs[r].active, 0ull);
        const unsigned long long k0 = key_init(reqs[r].bound);
        const unsigned long long k = hkeys[r];
        if (k < k0) {
            O.found = true;
            O.wt = (int)(k >> kKeyWtShift) - 1;
            O.g = (int)((k >> kKeyGShift) & 0xff);
            O.rank = k & kKeyRankMask;
        }
    }
    unsigned long long popc = 0, zcw = 0, tcw = 0;
    for (size_t oi = 0; oi < order.size(); ++oi) {
        const Plan& P = plans[order[oi]];
        const unsigned long long c = hcounts[order[oi]];
        outs[P.req].counts[P.g] += c;
        cw += c;
        if (P.tc) tcw += c;
        else if (P.mode == 2) zcw += c;
        else popc += c * (unsigned long long)P.popcs;
        const LevelDesc& D = hl[oi];
        if (outs[P.req].found && outs[P.req].g == P.g) outs[P.req].rank_shift = D.rank_shift;
    }
    if (stats) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, s->ev0, evm);
        cudaEventElapsedTime(&b, evm, s->ev1);
        stats->ms_gen += a;
        stats->ms_pairs += b;
        if (tc_timed) {
            float c = 0.f;
            cudaEventElapsedTime(&c, s->ev_tc0, s->ev_tc1);
            stats->ms_tc += c;
        }
        stats->jobs += all_jobs;
        stats->codewords += cw;
        stats->popc_issued += popc;
        stats->zero_codewords += zcw;
        stats->tc_codewords += tcw;
        stats->list_bytes_written += list_written;
        for (const auto& kv : tc_rows)
            stats->tc_operand_bytes += (kv.second.second - kv.second.first) * kPmRowBytes;
        stats->launches += launches;
    }
    if (timeline) {
        float t[5] = {0.f, 0.f, -1.f, -1.f, 0.f};
        const cudaEvent_t b = timeline_base(st);
        for (int i = 0; i < 5; ++i)
            if ((i != 2 && i != 3) || tc_timed) cudaEventElapsedTime(&t[i], b, tl[i]);
        std::fprintf(stderr, "qsfb timeline %p plan_ms %.3f h2d %.3f gen_end %.3f tc %.3f %.3f "
                     "join %.3f\n", (void*)s, plan_ms, t[0], t[1], t[2], t[3], t[4]);
        for (cudaEvent_t e : tl) cudaEventDestroy(e);
    }
    cudaEventDestroy(evm);
    return kOk;
}

}  // namespace qsfb
