// Brouwer-Zimmermann schedule on the device engine: information sets, the random
// information-set upper bound, the weight-level loop with the BZ lower bound
//   outer(w) = sum_g max(0, (w+1) - (K - rank_g))   (+1 if odd and every codeword is even)
// and the early stop inner <= outer (reference cpp/distfind/bz.cpp:118-228), the Z/X
// interleave with the cap-to-min (cpp/distfind/bz.cpp:242-403), and witness tracking.
#pragma once
#include <string>
#include <vector>

#include "engine.hpp"
#include "infoset.hpp"
#include "problem.hpp"

namespace qsfb {

struct BzOptions {
    bool verbose = false;
    int threads = 0;          // host threads for the seed trials (0 = hardware concurrency)
    bool no_early_stop = false;  // enumerate every level up to K (count parity)
    int seed_trials = 256;
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

// Upper bound from `trials` random column orders (reference cpp/distfind/bz.cpp:70-116):
// same generator, seeds and thread split, so the bound matches the reference run on the
// same host.  `word` receives the logical row that achieved it.
int random_is_seed(const Problem& p, int init_best, int trials, unsigned seed, int threads,
                   std::vector<u64>* word);

// One BZ subproblem stepped level by level on the device.
class BzSide {
public:
    int setup(Device* dev, Session* s, const Problem& p, const BzOptions& opt, const char* tag);
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
    // Rebuild the witness codeword (problem columns) from the recorded source.
    bool witness(std::vector<u64>& out) const;
};

int bz_distance(Device* dev, const Problem& p, const BzOptions& opt, BzResult& r);
int bz_min_interleaved(Device* dev, const Problem& pz, const Problem& px, const BzOptions& opt,
                       BzResult& r);
// Non-CSS: isometry to a 3q-column Hamming problem, BZ, then halve.
int symplectic_bz_distance(Device* dev, const Problem& sp, const BzOptions& opt, BzResult& r);

}  // namespace qsfb
