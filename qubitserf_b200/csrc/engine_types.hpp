// Descriptors shared by the host scheduler and the sm_100a kernels.
//
// Enumeration scheme (one BZ level of one information set g, combination weight w):
// every w-subset S of the K generator rows is split at its a-th smallest element p into
//   P = S ∩ [0, p]   (a rows, max p)          -- a block of the colex-ordered list L_a
//   Q = S ∩ (p, K)   (b = w - a rows, all > p) -- a prefix of the reflected-colex list R_b
// so level g,w is a union over p of rectangles  L_a[C(p,a) .. C(p+1,a)) x R_b[0 .. C(K-1-p,b)),
// which together hold every w-subset exactly once (sum_p C(p,a-1) C(K-1-p,b) = C(K,w)).
// A list entry is the XOR of its rows restricted to the set's NON-pivot columns ("red"
// words); the pivot columns of a systematic row contribute exactly one bit per selected
// pivot row, so  wt(c) = popc(red(P) ^ red(Q)) + pc(P) + pc(Q), pc = #rows below the rank.
#pragma once
#include <cstdint>

namespace qsfb {

constexpr int kWeightNone = 1 << 30;   // "no upper bound" (reference WEIGHT_NONE)
constexpr int kBinomMaxN = 4096;       // binomial table rows   (K <= 4096)
constexpr int kBinomMaxK = 64;         // binomial table columns (w <= 64)
constexpr int kRegTile = 256;          // register-side entries per warp job (32 lanes x 8)
constexpr int kKeyWtShift = 52;        // witness key = wt:12 | g:8 | rank:44
constexpr int kKeyGShift = 44;
constexpr unsigned long long kKeyRankMask = (1ull << 44) - 1;

// One (information set, weight level) enumeration, resident in device memory.
struct LevelDesc {
    // rows of the information set
    const uint32_t* red;      // K x W32 words (row restricted to non-pivot columns)
    const uint32_t* syn;      // K x SW words (row syndrome against the logical detector)
    // lists
    const uint32_t* la;       // colex a-subsets, HP words per entry
    const uint8_t* pca;       // pivot-row count per la entry (null when full rank)
    const uint32_t* rb;       // reflected-colex b-subsets, HP words per entry
    const uint8_t* pcb;       // (null when full rank)
    const uint64_t* term_jobs;  // nterms+1 prefix sums of job counts, by p = p_lo + t
    unsigned long long* key;    // packed witness key of this side (atomicMin)
    unsigned long long* count;  // evaluated codewords of (side, g)
    unsigned long long job_base;  // first global job index of this descriptor
    int K, w, a, b;
    int W32, SW, HP;          // red words, syndrome words, stored probe words per entry
    int rank;                 // rows [0, rank) are pivot rows
    int g;                    // information-set index inside its side (witness key)
    int p_lo, nterms;
    int loop_tile;            // loop-side entries per job
    int rank_shift;           // lex rank >> rank_shift goes into the key
    int count_all;            // 1: every nonzero codeword is a logical (no detector)
    // tensor-core sweep only (null / 0 elsewhere): the two lists as signed +-1 int8 rows
    // of kPmRowBytes (bit set -> +1, clear -> -1, beyond the live bits -> 0), 16-byte
    // chunk c of row e stored at c ^ ((e >> 1) & 3) (the 64-byte swizzle of the operand)
    int ksteps;               // 32-column MMA steps per pair (probe columns = 32 * ksteps)
    const int8_t* xpm;        // la rows
    const int8_t* ypm;        // rb rows
    int n_live;               // live +-1 columns among the first 32 * ksteps
    int tc_job_tiles;         // suffix tiles per tensor-core job of this level
};

constexpr int kGenRun = 4;         // consecutive list entries generated by one thread (measured: 2, 8 and 32 are slower)
constexpr int kPmRowBytes = 64;    // +-1 row: 64 int8 columns (the first two probe words)
constexpr int kPmPadRows = 256;    // zero rows after every +-1 list (whole-tile copies)

// One +-1 expansion: rows [row_lo, row_lo + rows) of `out` from the packed probe words of
// a list (rows at or beyond `count` are written as zeros).
struct ExpandDesc {
    const uint32_t* words;    // count x HP
    int8_t* out;              // (count + kPmPadRows) x kPmRowBytes
    unsigned long long row_base;  // first global row of this descriptor
    unsigned long long count, row_lo, rows;
    int HP, n_enc;            // live columns = min(non-pivot bits, 64)
};

// One list to generate: entries [0, count) of the colex (or reflected colex) order of the
// `size`-subsets of [0,K), XOR of the first HP red words of their rows.
struct GenDesc {
    const uint32_t* red;      // K x W32
    uint32_t* out;            // count x HP
    uint8_t* pc;              // count (null when full rank)
    int8_t* pm;               // +-1 rows (count + kPmPadRows), or null when not needed
    unsigned long long entry_base;  // first global run (kGenRun entries) of this descriptor
    unsigned long long count;
    unsigned long long pm_lo, pm_hi;  // entries whose +-1 rows are written (pm only)
    // the complete list one size smaller of the same set and orientation (HP words per
    // entry, and its pivot counts when `pc` is written), or null: entries are then built
    // from it instead of by unranking
    const uint32_t* src;
    const uint8_t* src_pc;
    int K, size, W32, HP, rank, reflect;
    int n_enc;                // live +-1 columns (pm only)
    int pad_;
};

}  // namespace qsfb
