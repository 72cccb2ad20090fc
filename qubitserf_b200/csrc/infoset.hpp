// Information sets for Brouwer-Zimmermann: a partition of the n columns, and for each part
// the generator put in systematic form on it (restricted RREF), with its rank.
#pragma once
#include <vector>

#include "gf2.hpp"

namespace qsfb {

struct InfoSet {
    Mat g;                  // K x n, pivot i of this set in row i (i < rank)
    int rank = 0;
    std::vector<int> pivots;  // pivot column of row i, i < rank
};

// The sequence the reference's BZ driver enumerates (cpp/distfind/css.cpp:417-447):
// greedy peel, replaced by an Edmonds matroid partition when n <= 200 and the partition
// packs more full-rank sets; then stably sorted by rank, descending
// (cpp/distfind/bz.cpp:141-143).
std::vector<InfoSet> information_sets(const Mat& code_gen);

}  // namespace qsfb
