// Reduction of every distance / operator-weight query to one BZ subproblem:
//   "minimum Hamming weight of a vector in rowspan(code_gen) that is a logical
//    (count_all, or check * c^T != 0)".
// Same contract as the reference's DistProblem (cpp/distfind/css.hpp:21-30), plus the
// codeword behind `seed_upper`, so that the engine can return a witness even when the
// starting upper bound is already the distance.
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include "gf2.hpp"

namespace qsfb {

struct Problem {
    int n = 0;                    // columns (3q after the symplectic isometry)
    Mat code_gen;                 // K x n basis of the searched space
    Mat check;                    // kcheck x n logical detector
    bool even = false;            // every codeword has even weight
    bool count_all = false;       // classical: every nonzero codeword counts
    int seed_upper = 0;           // a valid upper bound (0 = none)
    std::vector<u64> seed_word;   // a logical codeword of weight seed_upper (if any)
    bool symplectic = false;      // cost is symplectic weight (before isometry_extend)
    int qubits = 0;
};

// cpp/distfind/css.cpp:94-105
Mat quotient_basis(const Mat& self, const Mat& other);
// cpp/distfind/css.cpp:107-109 / 78-87
Problem css_problem(const Mat& Hx, const Mat& Hz, char which);
// Both sides of a CSS code at once: the same two problems as css_problem(·,'Z') and
// css_problem(·,'X'), sharing the two nullspaces and the two quotient bases.
std::pair<Problem, Problem> css_problem_pair(const Mat& Hx, const Mat& Hz);
// cpp/distfind/css.cpp:111-120
Problem classical_problem(const Mat& H);
// cpp/distfind/css.cpp:122-133
std::pair<Mat, Mat> css_center(const Mat& Gx, const Mat& Gz);
// cpp/distfind/css.cpp:135-139
Problem subsystem_problem(const Mat& Gx, const Mat& Gz, char which);
// cpp/distfind/css.cpp:141-148
bool in_rowspace(const Mat& G, const u8* vec);
// cpp/distfind/css.cpp:150-174
Problem coset_problem(const Mat& G, const u8* vec);

// Symplectic [z|x] helpers, cpp/distfind/stab.cpp:32-146.
Mat symplectic_swap(const Mat& m);
int symplectic_row_weight(const u64* row, int qubits);
bool is_css_symplectic(const Mat& S);
std::pair<Mat, Mat> split_css(const Mat& S);
Mat symplectic_center(const Mat& G);
Problem symplectic_problem(const Mat& Snorm, const Mat& Gtriv);
Problem symplectic_coset_problem(const Mat& G, const u8* op);
// (a|b) -> (a|b|a^b): symplectic weight doubles into Hamming weight, cpp/distfind/stab.cpp:147-178.
Problem isometry_extend(const Problem& sp);

// Independent host check of a witness codeword: c lies in rowspan(code_gen), is a logical
// (count_all, or some check row has odd overlap) and has Hamming weight `weight`.
bool verify_witness(const Problem& p, const u64* c, int weight);

}  // namespace qsfb
