// Choice of the pair sweep's probe filter (the device side is `fold_min` in enum_kernels.cu).
//
// A filter turns the XORed probe words of a pair into a lower bound on their popcount:
//   1..4  popc of the OR of the first 1..4 stored words (one POPC),
//   6     carry-save over four words, exact except that a column set in all four counts 2
//         (two POPCs).
// The bound only decides which chunks of the sweep are rescanned exactly, so every filter
// gives the same results; the choice is about speed.  The planner models the non-pivot bits
// of a pair as independent fair coins, takes P(filter <= t) as the rate at which a pair
// forces the rescan of its chunk, and picks the filter with the least expected cost.
// Host only; uses no heap (the probability tables live in static storage, filled once).
#pragma once

namespace qsfb {

struct FilterChoice {
    int filt;    // template argument of pairs_kernel
    int popcs;   // POPC instructions per pair
};

// HP: probe words stored per list entry (1, 2 or 4); nred: non-pivot bits of the set;
// t: largest probe weight that can still beat the bound (T - 1 - pivot rows);
// zero_test: the sweep only asks whether every probe word of the XOR is zero.
FilterChoice choose_filter(int HP, int nred, int t, bool zero_test);

// P(filter value <= t) under the fair-coin model (exposed for the tests of the planner).
double filter_pass_rate(int filt, int nred, int t);

// P(Binomial(bits, 1/2) <= t): pass rate of an exact Hamming-distance filter over `bits`
// random columns (the tensor-core sweep's).
double hamming_pass_rate(int bits, int t);

}  // namespace qsfb
