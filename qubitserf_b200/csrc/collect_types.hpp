// Plain-old-data descriptors shared by the host driver of the low-weight collector
// (collect.cpp) and its kernels (collect.cu).
//
// The collector enumerates, for one generator matrix of m rows, every sw-subset of rows
// (sw = 1..p) and keeps the XORs of weight 1..keep.  A subset S is split at its a-th
// smallest row q (a = ceil(sw/2), b = sw - a): the a smallest rows form an entry of the
// colex list of a-subsets whose largest element is q, the b largest rows an entry of the
// reflected-colex list of b-subsets of (q, m).  Every subset is one (prefix, suffix) pair
// of exactly one term q, so a level is a set of rectangles of independent pairs.
//
// Per list entry the device keeps HP probe words (the entry's XOR over up to 32 * HP
// columns that are nobody's private column) and its pivot count (rows of the subset that
// own a private column).  A row's private column is a column whose only 1 is in that row;
// a subset sets it exactly when the row is in the subset, so
//     weight(S) >= pivots(S) + popc(probe(S)),
// which is the sweep's filter; the pairs under keep + 1 become candidates that a second
// kernel re-evaluates over the full rows.
#pragma once
#include <cstdint>

namespace qsfb {

constexpr int kCollectMaxProbe = 8;     // probe words per entry (1, 2, 4 or 8)
constexpr int kCollectMaxWords = 16;    // 64-bit words per codeword: n <= 1024
constexpr int kCollectMaxSize = 64;     // subset size (binomial table columns)
constexpr int kCollectTileX = 256;      // prefix entries per warp job (32 lanes x 8)
constexpr int kCollectChunkY = 256;     // suffix entries per warp job (staged in shared memory)

// One list: `count` entries of `size`-subsets of [0, m), colex (reflect = 0) or reflected
// colex (rows m - 1 - c, reflect = 1).  `run_base` numbers the runs of kGenRun entries of
// all lists of a launch consecutively.
struct CollectListDesc {
    uint32_t* probe;                 // count x HP
    uint8_t* pc;                     // count
    unsigned long long count;
    unsigned long long run_base;
    int size;
    int reflect;
};

// Term q of a level: prefix entries [x0, x0 + nx) (the a-subsets with largest element q),
// suffix entries [0, ny) (the b-subsets of (q, m)); jobs [job_base, job_base + xtiles *
// ychunks) of the level's launch.
struct CollectTerm {
    unsigned long long x0, nx, ny;
    unsigned long long job_base;
    unsigned long long ychunks;
};

struct CollectLevelDesc {
    const uint32_t* xp;     // prefix list probe words (HP per entry)
    const uint8_t* xpc;     // prefix list pivot counts
    const uint32_t* yp;     // suffix list probe words
    const uint8_t* ypc;     // suffix list pivot counts
    const CollectTerm* terms;
    int nterms;
    int a, b;               // prefix and suffix subset sizes
    unsigned long long jobs;
};

// Launch-wide constants of the collector.
struct CollectShared {
    const uint32_t* probe_rows;   // m x HP probe words per row
    const uint8_t* piv;           // m: 1 if the row owns a private column
    const unsigned long long* rows;   // m x S64 full rows (the caller's column order)
    unsigned long long* out;      // cap x S64 collected codewords
    unsigned long long* cand;     // cand_cap x 2: pairs that passed the filter
                                  //   [0] prefix entry | subset size << 56, [1] suffix entry
    unsigned long long* ctr;      // [0] hits, [1] candidates (both counted past capacity)
    unsigned long long* job_ctr;  // one dynamic job counter per level
    unsigned long long cap, cand_cap;
    int m, S64, HP, keep;
    int filt;                     // probe_bound variant (collect.cu): 0 exact, 2/4 OR, 6 CSA
};

}  // namespace qsfb
