// Device side of the BZ engine: one context per process (device selected by
// QSFB_DEVICE, default 0), a size-bucketed caching allocator, and pooled sessions (one
// CUDA stream + staging buffers each) so that concurrent ABI calls never share a stream.
//
// A SideDev is the device image of one BZ subproblem: per information set the rows
// restricted to the set's non-pivot columns, the per-row detector syndromes, and the
// lazily built subset lists.  run_levels() enumerates any number of (side, level)
// requests in ONE list-generation launch plus one pair-sweep launch per kernel variant,
// which is what both the plain per-code path (one request) and the batched engine
// (every unresolved side of a round) use.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "engine_types.hpp"
#include "infoset.hpp"
#include "problem.hpp"

namespace qsfb {

// Status codes shared with the C ABI (0..3 are the reference's own, capi.cpp).
enum Status : int {
    kOk = 0,
    kErrNull = 1,
    kErrShape = 2,
    kErrMethod = 3,     // cc on non-CSS (reference rc 3)
    kErrDevice = 4,     // no usable device, CUDA error, or device wait timeout
    kErrUnsupported = 5,  // method/backend/size this engine does not run
    kErrMemory = 6,     // admission / device memory exhausted
};

struct Session;

double now_seconds();   // steady clock, seconds

// f(0..n-1) on the calling thread and up to max_threads - 1 threads of a process-wide pool
// (threads of the call's own while the pool serves another caller); returns when all ran
void host_parallel_for(size_t n, const std::function<void(size_t)>& f, int max_threads = 16);

class Device {
public:
    // The process-wide device context; nullptr (with *rc = kErrDevice) without a GPU.
    static Device* get(int* rc);
    static bool available();

    int id = 0;
    int num_sms = 0;
    std::string name;
    unsigned long long* d_binom = nullptr;   // (kBinomMaxN+1) x (kBinomMaxK+1), saturating

    void* alloc(size_t bytes);               // caching; nullptr on failure
    void release(void* p, size_t bytes);
    // Grow the device memory pool behind alloc()'s cache misses by `bytes` of mapped memory
    // that it keeps (a server calls it at start, so that a first allocation of a new size
    // during serving does not map memory while requests wait).
    void reserve(size_t bytes);
    size_t bytes_in_use() const { return in_use_; }
    size_t bytes_cached() const { return cached_; }
    // allocation calls that reach the driver (cache misses, pinned staging growth) and
    // their wall time: both can stall other threads' work
    std::atomic<long long> n_device_malloc{0}, ns_device_malloc{0};
    std::atomic<long long> n_pinned_alloc{0}, ns_pinned_alloc{0};

    Session* acquire();
    void give_back(Session* s);

    // Host-side binomial (same saturating table the kernels read).
    unsigned long long binom(int n, int k) const;

private:
    Device() = default;
    int init();
    std::mutex mu_;
    std::multimap<size_t, void*> free_;           // cached blocks by size
    std::unordered_map<void*, size_t> live_;      // size of every block handed out
    // Cache misses are served by the stream-ordered allocator from the device's default
    // memory pool (release threshold: keep everything), on a stream of their own that is
    // synchronised before the pointer is handed out, so any stream may use it at once.
    cudaMemPool_t pool_ = nullptr;
    cudaStream_t alloc_stream_ = nullptr;
    size_t in_use_ = 0, cached_ = 0;
    std::vector<Session*> idle_;
    std::vector<unsigned long long> h_binom_;
};

// Grow-only device / pinned-host scratch owned by a session.
struct DevScratch {
    void* d = nullptr;
    size_t cap = 0;
};
struct HostScratch {
    void* h = nullptr;
    size_t cap = 0;
};

struct Session {
    Device* dev = nullptr;
    cudaStream_t stream = nullptr;
    // the device's greatest stream priority: work that others wait on while rounds fill the
    // SMs (the random-information-set seed eliminations of a preparation) goes here, so its
    // blocks are scheduled first as SMs free up
    cudaStream_t urgent = nullptr;
    // one priority step below `urgent` (still above the rounds): a preparation's seed
    // trials run on it while its information-set eliminations, a short kernel on the
    // critical path, run on `urgent` and take the SMs first as blocks retire
    cudaStream_t urgent2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_tc0 = nullptr, ev_tc1 = nullptr;   // around the tensor-core sweep
    // pair launches of a round are spread over these streams (forked after the list
    // generation, joined before the results are read back): their tails overlap
    static constexpr int kAux = 3;
    cudaStream_t aux[kAux] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[kAux] = {nullptr, nullptr, nullptr};
    DevScratch d_stage;    // descriptors + term tables + keys/counts
    HostScratch h_stage;   // pinned mirror of d_stage
    HostScratch h_seed;    // pinned staging of the seed trials, in flight beside h_stage's
    DevScratch d_ctr;      // job counters (one per kernel variant)
    int ensure(size_t dbytes, size_t hbytes);
    int grow_pinned(HostScratch& hs, size_t hbytes);   // contents are not kept
};

// RAII lease of a session from the device pool.
struct SessionLease {
    Device* dev;
    Session* s;
    explicit SessionLease(Device* d) : dev(d), s(d->acquire()) {}
    ~SessionLease() { if (s) dev->give_back(s); }
};

struct ListBuf {
    uint32_t* words = nullptr;
    uint8_t* pc = nullptr;
    int8_t* pm = nullptr;  // +-1 rows for the tensor-core sweep (count + kPmPadRows rows)
    unsigned long long count = 0;
    size_t bytes_w = 0, bytes_pc = 0, bytes_pm = 0;
    bool ready = false;
    bool pm_ready = false;
    bool arena = false;   // carved from an Arena (released with it)
    bool queued = false;  // scheduled for generation in the current run_levels call
    bool pm_queued = false;
    unsigned long long pm_lo = 0, pm_hi = 0;   // rows of `pm` written (when pm_ready)
    int gen_idx = -1;     // position in the current call's generation list (while queued)
    int exp_idx = -1;     // position in the current call's expansion list (while pm_queued)
};

// Bump allocator over device chunks taken from the caching allocator; everything carved
// from it is released together when the arena is destroyed (one batch).
class Arena {
public:
    // min_chunk: smallest device chunk taken from the caching allocator (a whole batch
    // carves from 64 MiB chunks; a single serving request from much smaller ones)
    explicit Arena(Device* d, size_t min_chunk = 64ull << 20) : dev_(d), min_chunk_(min_chunk) {}
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;
    ~Arena();
    void* alloc(size_t bytes);
    size_t bytes() const { return total_; }

private:
    Device* dev_;
    size_t min_chunk_;
    std::mutex mu_;   // the rounds of several job groups may carve lists concurrently
    std::vector<std::pair<char*, size_t>> chunks_;
    size_t used_ = 0, total_ = 0;
};

class SideDev {
public:
    SideDev() = default;
    SideDev(const SideDev&) = delete;
    SideDev& operator=(const SideDev&) = delete;
    ~SideDev();

    // Host half: pack every information set's rows over its non-pivot columns and the
    // per-row detector syndromes.  Returns a Status (no device work).
    int prepare(const Problem& p, const std::vector<InfoSet>& sets);
    // Device half for a single side: own allocation + copy on the session stream.
    int upload(Device* dev, Session* s);
    // The rows were built on the device (the information-set kernel wrote red/syn into
    // `arena` with row strides W32 and SWP): take the host-side description of the sets.
    int adopt_device(const Problem& p, const std::vector<InfoSet>& sets, uint32_t* red,
                     uint32_t* syn, int W32, int SWP, Device* dev, Arena* arena);
    bool device_rows = false;    // red/syn built on the device (nothing to upload)

    int n = 0, K = 0, ng = 0, W32 = 0, SW = 0, kcheck = 0;
    bool count_all = false;
    std::vector<int> ranks;
    std::vector<std::vector<int>> nonpivot;   // per set: non-pivot columns (bit order of red)
    std::vector<uint32_t> h_red, h_syn;       // host images (ng x K x W32, ng x K x max(SW,1))
    Device* dev = nullptr;
    Arena* arena = nullptr;      // list storage (null: caching allocator per list)
    bool owns = false;           // d_red/d_syn allocated by upload()
    uint32_t* d_red = nullptr;
    uint32_t* d_syn = nullptr;
    size_t bytes_red = 0, bytes_syn = 0;
    std::map<std::tuple<int, int, int>, ListBuf> lists;   // (g, size, reflect)
    size_t list_bytes = 0;
};

// Upload many prepared sides with one allocation (from `arena`) and one host->device copy.
int upload_sides(Device* dev, Session* s, Arena* arena, const std::vector<SideDev*>& sides);

struct LevelReq {
    SideDev* side = nullptr;
    int w = 0;
    int active = 0;      // information sets [0, active) are enumerated
    int bound = kWeightNone;  // current upper bound (candidates of weight <= bound count)
};

struct LevelOut {
    bool found = false;  // some candidate of weight <= bound was seen
    int wt = kWeightNone;
    int g = -1;
    unsigned long long rank = 0;   // lexicographic rank (shifted by rank_shift)
    int rank_shift = 0;
    std::vector<unsigned long long> counts;   // evaluated codewords per set [0, active)
};

struct RunStats {
    double ms_gen = 0.0;     // device time of list generation
    double ms_pairs = 0.0;   // device time of the pair sweep
    double ms_tc = 0.0;      // device time of the tensor-core sweep launches alone
    unsigned long long jobs = 0;
    unsigned long long codewords = 0;
    unsigned long long popc_issued = 0;    // POPC the pair kernels issue (H per pair, 0 in zero mode)
    unsigned long long zero_codewords = 0; // codewords swept by the zero-test mode
    unsigned long long tc_codewords = 0;   // codewords swept by the tensor-core kernel
    // +-1 row bytes the tensor-core launches must read at least once: per round, the union
    // of the row ranges its tensor plans read from each list
    unsigned long long tc_operand_bytes = 0;
    // bytes the list generation must write: probe words, pivot counts and +-1 rows of the
    // generated lists, +-1 rows added to earlier lists
    unsigned long long list_bytes_written = 0;
    int launches = 0;
    double host_setup_s = 0.0;
    double device_seed_s = 0.0;   // wall time of the device seed phase (copy + kernel)
    double device_seed_wait_s = 0.0;   // of which: waiting for the copies and the kernel
    double device_sets_s = 0.0;   // wall time of the device information-set phase
    double host_plan_s = 0.0;     // run_levels host work before the launches
    double host_apply_s = 0.0;    // schedule updates after each round
};

// Enumerate every request; blocking.  Returns a Status.
int run_levels(Session* s, const std::vector<LevelReq>& reqs, std::vector<LevelOut>& outs,
               RunStats* stats = nullptr);

// Enumeration counts are the per-set C(K,w); used by tests of the job decomposition.
unsigned long long level_pairs(const Device* dev, int K, int w);

// Subset lists above this many entries are never built: at 4 bytes per probe word plus the
// 64-byte +-1 row they would exceed any device's memory, and every product of a list
// count with a per-entry byte size stays far from 2^64 below it.
constexpr unsigned long long kMaxListEntries = 1ull << 36;

// C(n, k) computed on the host without a table, saturating to ~0ull at 2^64.
unsigned long long host_binom(int n, int k);

// The prefix/suffix split of a level's w-subsets: a = w (single list) when C(K, w) is
// small, else a = ceil(w/2), b = w - a.
void level_split(unsigned long long pairs, int w, int* a, int* b);

// Size guard of one level of a K-row set, without a device: kOk, kErrUnsupported (w or K
// beyond the binomial table, C(K, w) saturated or >= 2^62) or kErrMemory (a subset list
// beyond kMaxListEntries).  Every path that sizes buffers from binomials calls it first.
int level_size_rc(int K, int w);

}  // namespace qsfb
