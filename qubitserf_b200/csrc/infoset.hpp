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

// The sequence the reference's BZ driver enumerates (cpp/distfind/css.cpp:336-366):
// greedy peel, replaced by an Edmonds matroid partition when n <= 200 and the partition
// packs more full-rank sets; then stably sorted by rank, descending
// (cpp/distfind/bz.cpp:95-97).
std::vector<InfoSet> information_sets(const Mat& code_gen);

// Number of sets of rank K.
int full_sets(const std::vector<InfoSet>& s, int K);

// The step after the greedy peel (cpp/distfind/css.cpp:341-365), given how many full-rank
// sets the peel found: true when the matroid partition replaces it, with the classes'
// column lists (each in the partition's own order) already in the final rank-sorted order
// and each class's rank (its number of nonzero columns).  Restricted RREF of a fresh copy
// of code_gen over each list gives the sets.
bool matroid_sets(const Mat& code_gen, int greedy_full, std::vector<std::vector<int>>* lists,
                  std::vector<int>* ranks);

}  // namespace qsfb
