// Test-infrastructure shim compiled TOGETHER with the reference's own CPU sources
// (cpp/qsf/*.cpp, cpp/distfind/*.cpp of Quantinuum/Qubitserf) into oracle/_ref/.
// It is never part of the product library: only tests/, the golden-fixture script and
// bench.py's reference arm load it.
//
// The reference exposes its per-level enumerator and its information-set construction
// only as C++ (qsf::Backend::enumerate, distfind::gamma_sequence).  These extern "C"
// wrappers make both reachable from ctypes so the C restatement in oracle/bz_oracle.c
// and the product's host reduction can be pinned against the reference itself:
//   ref_enumerate       -> qsf::cpu_backend()->enumerate(EnumPlan)   (cpp/qsf/backend_cpu.cpp:33-75)
//   ref_problem_gammas  -> classical_problem / css_problem / subsystem_problem + gamma_sequence
//                          + the rank-descending stable sort of bz_distance (cpp/distfind/bz.cpp:95-107)
#include "qsf/backend.hpp"
#include "qsf/combinatorics.hpp"
#include "distfind/css.hpp"
#include "distfind/stab.hpp"
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

using namespace distfind;

extern "C" {

// One BZ weight level through the reference CPU backend.  gamma is ng*K*stride words,
// check is kcheck*stride words (row-major).  threads<=0 => hardware concurrency.
int ref_enumerate(int n, int stride, int K, int d, int num_gamma, const uint64_t* gamma,
                  int kcheck, const uint64_t* check, int current_best, int threads) {
    qsf::BinomTable bt(K, K);
    qsf::EnumPlan p;
    p.n = n; p.stride = stride; p.K = K; p.d = d;
    p.num_gamma = num_gamma; p.num_gamma_total = num_gamma;
    p.gamma = gamma;
    p.kcheck = kcheck; p.check = check;
    p.binom = bt.c.data(); p.binom_maxN = bt.maxN; p.binom_maxK = bt.maxK;
    p.current_best = current_best;
    p.buffers_key = qsf::next_buffers_key();
    qsf::set_cpu_threads(threads);
    int r = qsf::cpu_backend()->enumerate(p);
    qsf::set_cpu_threads(0);
    return r;
}

// Build the reference's DistProblem for `kind` and its information-set sequence.
//   kind 0: classical_problem(H)                 (A = H)
//   kind 1: css_problem(Hx=A, Hz=B, 'Z')   kind 2: css_problem(A, B, 'X')
//   kind 3: subsystem_problem(Gx=A, Gz=B, 'Z')   kind 4: subsystem_problem(A, B, 'X')
//   kind 5: symplectic_problem(S=A, S=A) + isometry_extend (plain non-CSS stabilizer)
// Outputs (caller-sized, max_words words for gamma, max_check for check):
//   meta[0..7] = {n, K, num_gamma, kcheck, even, count_all, seed_upper, stride}
//   ranks[num_gamma]; gamma[ng*K*stride] in the rank-descending stable order of bz_distance;
//   check[kcheck*stride].
// Returns 0, or 1 if a buffer is too small.
int ref_problem_gammas(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br,
                       int bc, int* meta, int* ranks, int max_gamma, uint64_t* gamma,
                       long long max_words, uint64_t* check, long long max_check) {
    GF2Mat mA = from_dense(A, ar, ac);
    GF2Mat mB = (B && br > 0) ? from_dense(B, br, bc) : GF2Mat(0, ac);
    DistProblem p;
    switch (kind) {
        case 0: p = classical_problem(mA); break;
        case 1: p = css_problem(mA, mB, 'Z'); break;
        case 2: p = css_problem(mA, mB, 'X'); break;
        case 3: p = subsystem_problem(mA, mB, 'Z'); break;
        case 4: p = subsystem_problem(mA, mB, 'X'); break;
        default: p = isometry_extend(symplectic_problem(mA, mA)); break;
    }
    const int K = p.code_gen.rows, stride = words_for(p.n);
    std::vector<Gamma> seq;
    if (K > 0) {
        seq = gamma_sequence(p.code_gen);
        std::stable_sort(seq.begin(), seq.end(),
                         [](const Gamma& a, const Gamma& b) { return a.rank > b.rank; });
    }
    const int ng = (int)seq.size();
    const int kcheck = p.count_all ? 0 : p.check.rows;
    meta[0] = p.n; meta[1] = K; meta[2] = ng; meta[3] = kcheck;
    meta[4] = p.even ? 1 : 0; meta[5] = p.count_all ? 1 : 0; meta[6] = p.seed_upper;
    meta[7] = stride;
    if (ng > max_gamma || (long long)ng * K * stride > max_words ||
        (long long)kcheck * stride > max_check)
        return 1;
    for (int g = 0; g < ng; ++g) {
        ranks[g] = seq[g].rank;
        for (int r = 0; r < K; ++r)
            for (int w = 0; w < stride; ++w)
                gamma[((size_t)g * K + r) * stride + w] = seq[g].g.row(r)[w];
    }
    for (int c = 0; c < kcheck; ++c)
        for (int w = 0; w < stride; ++w) check[(size_t)c * stride + w] = p.check.row(c)[w];
    return 0;
}

}  // extern "C"
