/* CPU restatement of the reference Brouwer-Zimmermann distance path (Quantinuum/Qubitserf),
 * written in plain C as TEST INFRASTRUCTURE ONLY: the checker that tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg compare the GPU engine against.
 * The product library never links or loads it.
 *
 * Parity: pinned against the reference's own CPU library built from its sources
 * (oracle/_ref, see oracle/Makefile) and against committed golden vectors
 * (tests/golden/, made by tests/golden/make_golden.py).  Distances, lower bounds and
 * per-level counts agree with the reference; with seed_trials = 0 the upper bound starts
 * from the problem's seed_upper only (the reference adds 256 random information sets,
 * which changes how many levels run but never the distance).
 */
#ifndef BZ_ORACLE_H
#define BZ_ORACLE_H
#include <stdint.h>

#define ORC_WEIGHT_NONE (1 << 30)

typedef struct {
    int distance, lower_bound, proven, levels;
    unsigned long long codewords; /* sum over levels of C(K,w) * active */
} orc_result;

typedef struct {
    int no_early_stop;      /* enumerate every level up to K */
    int seed_trials;        /* random information-set trials (0 = none) */
    /* optional per-level record: levels_w[i], levels_active[i] (cap entries) */
    int cap;
    int* levels_w;
    int* levels_active;
    int* levels_side;
    int mitm;               /* method "mitm": meet in the middle (cpp/distfind/mitm.cpp) */
} orc_options;

/* One level, brute force: cpp/qsf/backend.hpp:84-100 evaluated over every combination in
 * lexicographic order (cpp/distfind/tests/cpu_enum_ref.cpp:27-42).  Returns
 * min(current_best, lightest logical < current_best); counts[g] = C(K,d); the arg-min with the
 * smallest (weight, g, lex rank) goes to *arg_g / *arg_rank (-1 when none). */
int orc_enumerate(int n, int stride, int K, int d, int ng, const uint64_t* gamma, int kcheck,
                  const uint64_t* check, int current_best, unsigned long long* counts,
                  int* arg_g, unsigned long long* arg_rank);

/* The reference's two-level CPU kernel (cpp/qsf/enum_core.hpp:109-194), one thread. */
int orc_enumerate_fast(int n, int stride, int K, int d, int ng, const uint64_t* gamma,
                       int kcheck, const uint64_t* check, int current_best);

int orc_classical_distance(const uint8_t* H, int rows, int cols, const orc_options* opt,
                           orc_result* out);
/* which: 'Z', 'X' or 'M' (interleaved min) */
int orc_css_distance(const uint8_t* Hx, int hxr, int hxc, const uint8_t* Hz, int hzr, int hzc,
                     char which, const orc_options* opt, orc_result* out);
int orc_subsystem_distance(const uint8_t* Gx, int gxr, int gxc, const uint8_t* Gz, int gzr,
                           int gzc, char which, const orc_options* opt, orc_result* out);
/* z_weight / x_weight of a CSS operator (cpp/distfind/op_weight.cpp:9-36) */
int orc_operator_weight(const uint8_t* Gx, int gxr, int gxc, const uint8_t* Gz, int gzr, int gzc,
                        const uint8_t* z, const uint8_t* x, const orc_options* opt, int* zw,
                        int* xw);
/* symplectic [z|x] inputs; subsystem selects the gauge center reduction */
int orc_stabilizer_distance(const uint8_t* S, int rows, int cols, int subsystem, char which,
                            const orc_options* opt, orc_result* out);
int orc_pauli_operator_weight(const uint8_t* G, int rows, int cols, const uint8_t* op,
                              const orc_options* opt, orc_result* out);

/* Problem + information sets as bz_distance sees them (kinds as in the engine's
 * qsfb_prepare_problem).  meta = {n, K, ng, kcheck, even, count_all, seed_upper, stride}. */
int orc_prepare(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br, int bc,
                int* meta, int* ranks, int max_gamma);

/* codeaut low-weight collection (cpp/codeaut/bz.cpp:55-117): the distinct nonzero XORs of
 * size-1..p subsets of the m x n 0/1 rows of G with weight <= keep, sorted by packed 64-bit
 * words (word 0 first).  Returns their count with the rows in *out (ceil(n/64) words each;
 * release with orc_free) and the saturating combination count in *combos; -1 if memory
 * runs out. */
long long orc_collect(const uint8_t* G, int m, int n, int p, int keep, uint64_t** out,
                      long long* combos);
void orc_free(void* ptr);

#endif
