// Brouwer-Zimmermann schedule on the device engine.
//
// A BzJob is one certificate: a single subproblem (classical, one CSS side, a coset, the
// non-CSS isometry) or an interleaved Z/X pair (CSS which='min').  Jobs are stepped one
// weight level per ROUND; every unresolved job of a round contributes its level to ONE
// run_levels() call, so a single code (the plain drop-in) and a batch of a thousand codes
// run through the same code path.  Bounds, termination and the Z/X cap keep the
// reference's semantics (cpp/distfind/bz.cpp:72-370):
//   outer(w) = sum_g max(0, (w+1) - (K - rank_g))  (+1 if odd and every codeword is even)
//   stop when inner <= outer; a pair side is capped once its outer reaches the best found.
// In a pair both sides' level w run in the same round; the X result is folded in only if
// the sequential Z-then-X order would have stepped X (capped levels are discarded), which
// leaves every reported number identical to the sequential schedule.
#pragma once
#include <cstdlib>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "engine.hpp"
#include "infoset.hpp"
#include "problem.hpp"

namespace qsfb {

struct BzOptions {
    bool verbose = false;
    bool no_early_stop = false;  // enumerate every level up to K (single sides; count parity)
    int seed_trials = 256;
    bool parallel_seed = true;   // host seed trials on hardware_concurrency threads
    // eliminations of the seed trials on the GPU when K <= 128 and n <= 256 (QSFB_HOST_SEEDS=1:
    // on the host threads, with the same streams and results)
    bool device_seed = std::getenv("QSFB_HOST_SEEDS") == nullptr;
    // information sets (and the packed rows) built on the GPU when K, n <= 128;
    // QSFB_HOST_INFOSETS=1 builds them on the host instead (same results)
    bool device_infosets = std::getenv("QSFB_HOST_INFOSETS") == nullptr;
};

// One enumerated level, for the per-(information set, w) count record.
struct LevelRecord {
    int side = 0;      // 0 = single / Z, 1 = X
    int w = 0;
    int active = 0;
    std::vector<unsigned long long> counts;
};

struct BzResult {
    int distance = -1;
    int levels = 0;
    int lower_bound = 0;
    bool proven = false;
    double seconds = 0.0;
    std::vector<u64> witness;   // problem-space codeword of weight `distance` (if any)
    bool witness_ok = false;    // verified on the host against the problem
    int witness_side = 0;
    RunStats stats;
    std::vector<LevelRecord> trace;
};

// Upper bound from `trials` random column orders (reference cpp/distfind/bz.cpp:24-70):
// same generator, seeds and split of the trials over hardware_concurrency() streams, so
// the bound equals the reference's on the same host.  parallel=false replays the streams
// one after another (same result).  `word` receives a logical row achieving the bound.
int random_is_seed(const Problem& p, int init_best, int trials, unsigned seed, bool parallel,
                   std::vector<u64>* word);

// The column orders of those trials (trials x n, trial-major), drawn exactly as the
// reference draws them; `only` >= 0 returns just that trial's order.
std::vector<int> seed_orders(int n, int trials, unsigned seed, int only = -1);
// The same orders as bytes (n <= 256), one shared copy per (n, trials, seed).
std::shared_ptr<const std::vector<uint8_t>> seed_order_bytes(int n, int trials, unsigned seed);

// One BZ subproblem stepped level by level.
class BzSide {
public:
    int setup_host(const Problem& p, const BzOptions& opt, const char* tag);
    bool has_logicals = false;
    int K = 0, ng = 0, maxw = 0;
    bool even = false;
    std::vector<int> ranks;
    int inner = kWeightNone, outer = 0, level = 0;
    bool proven = false, resolved = false;
    const char* tag = "";
    const Problem* prob = nullptr;
    std::vector<InfoSet> sets;
    SideDev dev;
    // witness: the seed word, or (set g, lexicographic rank at weight w)
    std::vector<u64> best_word;
    int best_w = 0, best_g = -1;
    unsigned long long best_rank = 0;
    int best_shift = 0;
    bool best_from_level = false;

    int active_at(int w) const;
    int outer_at(int w) const;
    void absorb(int w, const LevelOut& o);
    bool witness(std::vector<u64>& out) const;
    // state right after setup (for re-execution)
    int inner0 = kWeightNone;
    bool resolved0 = false;
    void reset();
    // device-seed bookkeeping: trials pending on the GPU, and the winning (trial, row)
    bool seed_pending = false;
    int seed_trials = 0;
    int seed_trial = -1, seed_row = -1;
    std::shared_ptr<const std::vector<uint8_t>> seed_perm;   // trials x n, shared by length
    void apply_device_seed(unsigned key);
    // information sets pending on the GPU (setup_jobs_device builds them and the packed rows)
    bool infoset_pending = false;
    bool sets_from_classes = false;   // built on the device from matroid-partition classes
    // Take the sets built on the device (or, with red == nullptr, build the rows on the host
    // for upload): fills ng, ranks and the device image.
    int adopt_sets(std::vector<InfoSet>&& s, uint32_t* red, uint32_t* syn, int W32, int SWP,
                   Device* d, Arena* arena);
};

class BzJob {
public:
    // Single subproblem, or (pair=true) the interleaved min over two.
    BzJob(Problem p0, const BzOptions& opt);
    BzJob(Problem pz, Problem px, const BzOptions& opt);
    // Deferred construction: `build` fills p[0] (and p[1] for a pair) inside setup_host, on
    // the worker thread; returning 1 marks a certificate that is trivially 0 (an operator
    // already in the group) and needs no enumeration.
    using Builder = std::function<int(Problem& p0, Problem& p1)>;
    BzJob(Builder build, bool pair, const BzOptions& opt);
    bool zero = false;                      // trivially weight 0 (see Builder)
    BzJob(const BzJob&) = delete;
    BzJob& operator=(const BzJob&) = delete;

    int setup_host();                       // information sets, seeds, packed rows
    void finish_setup();                    // after the (device) seeds are in
    std::vector<SideDev*> device_sides();   // sides that need device data
    // Level requests of this round (w = next level); side index per request.
    void requests(std::vector<LevelReq>& q, std::vector<int>& side);
    // Fold the round's results (one per request, in order) into the schedule.
    void apply(const std::vector<const LevelOut*>& outs, const std::vector<int>& side);
    bool done() const { return done_; }
    void reset();                           // back to the post-setup state
    BzResult result();                      // final numbers + verified witness
    // The result of a finished job, computed once (witness rebuilt and verified) and kept:
    // the rounds call it as soon as a job is done, so that the answers of a batch are
    // ready when its last round ends.
    const BzResult& final_result();

    bool pair = false;
    Problem p[2];
    BzSide s[2];
    BzOptions opt;
    RunStats stats;
    std::vector<LevelRecord> trace;

private:
    BzResult compute_result();
    std::unique_ptr<BzResult> final_;
    Builder build_;
    int w_ = 0;                // last stepped level
    int maxw_ = 0;
    int best_ = kWeightNone;   // pair: best distance found so far
    bool done_ = false;
    double t0_ = 0.0, tl_ = 0.0;
    bool no_stop_ = false;
};

// Run jobs to completion on one device: host setup on `host_threads` threads (0 = all
// cores), one bulk upload, then rounds.  Per-job results in `out`.  Returns a Status.
int run_jobs(Device* dev, std::vector<BzJob*>& jobs, int host_threads, RunStats* stats,
             int* rounds = nullptr);

// The two halves of run_jobs, for callers that keep the device data resident and run the
// rounds repeatedly: host setup of every job + one upload into `arena`, then the rounds.
int setup_jobs(Device* dev, Session* s, Arena* arena, std::vector<BzJob*>& jobs,
               int host_threads, RunStats* stats);
// setup_jobs in two phases: the host setup of every job (no device work), then the seed
// eliminations and the upload (a pipeline runs the next batch's host phase meanwhile).
int setup_jobs_host(std::vector<BzJob*>& jobs, int host_threads, RunStats* stats);
int setup_jobs_device(Device* dev, Session* s, Arena* arena, std::vector<BzJob*>& jobs,
                      RunStats* stats);
// The information sets of every side whose construction is pending, on the device (one
// warp per side), with their packed rows and syndromes written into `arena`; sides the
// kernel cannot hold fall back to the host construction (rows uploaded by upload_sides).
int device_infosets(Session* s, Arena* arena, const std::vector<BzSide*>& sides,
                    RunStats* stats);
// `feed` (optional) is called at the top of every round with idle = false and may append
// jobs to `jobs` (they start from their first level in that round); when every job is done
// it is called with idle = true, may block until it has more, and returns whether it
// appended any (false ends the rounds).
using JobFeed = std::function<bool(std::vector<BzJob*>&, bool idle)>;
int run_rounds(Session* s, std::vector<BzJob*>& jobs, RunStats* stats, int* rounds,
               double* span_ms = nullptr, const JobFeed* feed = nullptr);

int bz_distance(Device* dev, const Problem& p, const BzOptions& opt, BzResult& r);
int bz_min_interleaved(Device* dev, const Problem& pz, const Problem& px, const BzOptions& opt,
                       BzResult& r);
// Non-CSS: isometry to a 3q-column Hamming problem, BZ, then halve.
int symplectic_bz_distance(Device* dev, const Problem& sp, const BzOptions& opt, BzResult& r);

double now_seconds();

}  // namespace qsfb
