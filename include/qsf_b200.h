/* C ABI of libqsfb200.so, the B200 (sm_100a) Brouwer-Zimmermann distance engine.
 *
 * Part 1 is the drop-in boundary: the nine distfind_* entry points with the exact
 * signatures, struct layouts and return codes of the reference's
 * cpp/distfind/capi.h:12-111 (Quantinuum/Qubitserf), which its Python layer binds with
 * ctypes (python/qubitserf/distfind/_native.py:15-107).  Pointing QUBITSERF_LIB at this
 * library makes the unchanged reference Python call it.  Methods "bz" (Brouwer-Zimmermann)
 * and "mitm" (meet in the middle) run on backend "gpu"/"auto", with the reference's
 * method dispatch (any other name is BZ; "cc" falls back where the reference falls back);
 * there is no CPU fallback.
 *
 * Return codes: 0 ok; 1 null pointer; 2 not a [z|x] matrix / bad operator length;
 * 3 method "cc" on a non-CSS code (the reference's own codes, cpp/distfind/capi.cpp:29-288);
 * 4 no usable sm_100 device or a CUDA error; 5 method/backend/size this engine does not
 * run (method "cc" where the reference runs its connected-cluster solver, backend "cpu",
 * n > 1024 after pivot removal); 6 device memory exhausted.  Codes 4-6 surface in the
 * reference Python as RuntimeError.
 *
 * Part 2 (qsfb_*) adds what the reference has no ABI for: the per-level enumeration on a
 * raw plan, the host problem reduction, the witness and per-level counts of the last
 * call, and the batched engine.
 */
#ifndef QSF_B200_H
#define QSF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- Part 1: drop-in */

/* Same layout as the reference DistfindResult (cpp/distfind/capi.h:12-19). */
typedef struct {
    int distance;       /* -1 if undefined (no logicals / empty code) */
    int lower_bound;
    int proven;
    int levels;
    double seconds;
    char backend[16];   /* "cuda" */
} DistfindResult;

/* Same layout as the reference DistfindOpResult (cpp/distfind/capi.h:39-45). */
typedef struct {
    int z_weight;
    int x_weight;
    int proven;
    double seconds;
    char backend[16];
} DistfindOpResult;

/* Replaces distfind_css_distance, cpp/distfind/capi.h:24-29 (which: 'Z','X','M'). */
int distfind_css_distance(const uint8_t* Hx, int hx_rows, int hx_cols,
                          const uint8_t* Hz, int hz_rows, int hz_cols,
                          const char* method, char which, const char* backend,
                          int threads, int verbose, DistfindResult* out);

/* Replaces distfind_classical_distance, cpp/distfind/capi.h:32-36. */
int distfind_classical_distance(const uint8_t* H, int rows, int cols,
                                const char* method, const char* backend,
                                int threads, int verbose, DistfindResult* out);

/* Replaces distfind_operator_weight, cpp/distfind/capi.h:52-58. */
int distfind_operator_weight(const uint8_t* Gx, int gx_rows, int gx_cols,
                             const uint8_t* Gz, int gz_rows, int gz_cols,
                             const uint8_t* z_op, const uint8_t* x_op, int n,
                             const char* method, const char* backend,
                             int threads, int verbose, DistfindOpResult* out);

/* Replaces distfind_subsystem_distance, cpp/distfind/capi.h:63-68. */
int distfind_subsystem_distance(const uint8_t* Gx, int gx_rows, int gx_cols,
                                const uint8_t* Gz, int gz_rows, int gz_cols,
                                const char* method, char which, const char* backend,
                                int threads, int verbose, DistfindResult* out);

/* Replaces distfind_stabilizer_distance, cpp/distfind/capi.h:81-85. */
int distfind_stabilizer_distance(const uint8_t* S, int rows, int cols,
                                 const char* method, char which, const char* backend,
                                 int threads, int verbose, DistfindResult* out);

/* Replaces distfind_subsystem_stabilizer_distance, cpp/distfind/capi.h:91-95. */
int distfind_subsystem_stabilizer_distance(const uint8_t* G, int rows, int cols,
                                           const char* method, char which, const char* backend,
                                           int threads, int verbose, DistfindResult* out);

/* Replaces distfind_stabilizer_operator_weight, cpp/distfind/capi.h:103-108. */
int distfind_stabilizer_operator_weight(const uint8_t* G, int rows, int cols,
                                        const uint8_t* op, int op_len,
                                        const char* method, const char* backend,
                                        int threads, int verbose, DistfindResult* out);

/* Replaces distfind_backend_available, cpp/distfind/capi.h:110: "gpu"/"cuda"/"auto" -> 1
 * when an sm_100 device is usable; "cpu"/"metal" -> 0. */
int distfind_backend_available(const char* name);

/* Replaces distfind_version, cpp/distfind/capi.h:111. */
const char* distfind_version(void);

/* ---------------------------------------------------------------- Part 2: engine */

/* Summary of the last distance call made on the calling thread. */
typedef struct {
    int distance;
    int lower_bound;
    int proven;
    int levels;
    int witness_ok;          /* 1: the witness was verified on the host */
    int witness_bits;        /* length of the witness (problem columns) */
    int witness_side;        /* 0 = single/Z side, 1 = X side */
    int kernel_launches;
    double seconds;          /* wall time of the call */
    double device_ms;        /* device time of list generation + pair sweeps */
    unsigned long long codewords;  /* evaluated (information set, combination) pairs */
} QsfbReport;

/* One weight level of one BZ subproblem on a raw plan: the semantics of the reference's
 * qsf::Backend::enumerate(EnumPlan) (cpp/qsf/backend.hpp:21-42, 53-61;
 * cpp/qsf/enum_core.hpp:74-88, 109-194).  gamma = num_gamma*K*stride words, check =
 * kcheck*stride words, row-major; kcheck == 0 means every codeword counts.  Rows need not be
 * systematic.  *out_best = min(current_best, lightest logical codeword < current_best);
 * out_counts[g] = evaluated combinations of set g (== C(K,d)); the arg-min is returned as
 * (*out_g, *out_rank) with rank in the lexicographic order of cpp/qsf/combinatorics.hpp:52-61
 * (-1 if nothing beat current_best).  Sizes are checked before any device work: d <= 64,
 * K <= 4096, num_gamma <= 255 and C(K, d) < 2^62, else 5; a level whose subset lists would
 * exceed 2^36 entries, else 6. */
int qsfb_enumerate_plan(int n, int stride, int K, int d, int num_gamma, const uint64_t* gamma,
                        int kcheck, const uint64_t* check, int current_best, int* out_best,
                        unsigned long long* out_counts, int* out_g, unsigned long long* out_rank);

/* Host reduction only (no device): the BZ subproblem and its information sets exactly as
 * the reference's bz_distance sees them (cpp/distfind/bz.cpp:95-115).  kind: 0 classical(H=A),
 * 1 css Z (Hx=A,Hz=B), 2 css X, 3 subsystem Z (Gx=A,Gz=B), 4 subsystem X, 5 non-CSS
 * stabilizer S=A after the (a|b)->(a|b|a^b) isometry.  meta = {n, K, num_gamma, kcheck, even,
 * count_all, seed_upper, stride}; gamma (num_gamma*K*stride words) and check
 * (kcheck*stride words) are written when they fit.  Returns 0, 1 (null), 7 (buffer small). */
int qsfb_prepare_problem(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br,
                         int bc, int* meta, int* ranks, int max_gamma, uint64_t* gamma,
                         long long max_words, uint64_t* check, long long max_check);

/* qsfb_prepare_problem with the information sets built where the engine builds them (no
 * reference counterpart; it exposes the device construction that replaces the reference's
 * host eliminations, cpp/distfind/css.cpp:177-203, 336-366 and cpp/qsf/gf2.cpp:42-58).
 * on_device = 1: the GPU kernel (one warp per subproblem, K and n <= 128; larger ones and
 * more than 16 sets are built on the host); 0: the host construction.  meta holds 12 ints:
 * qsfb_prepare_problem's 8, then W32 = ceil(n/32), SWP = max(1, ceil(kcheck/32)), 1 when
 * the device built the sets, and 1 when it built them from matroid-partition classes.  red (num_gamma*K*W32 u32, when not NULL): each set's rows over
 * its non-pivot columns in ascending order, zero padded; syn (num_gamma*K*SWP u32): bit c of
 * row r = parity(check_c & row r) -- the two tables the pair sweeps read.
 * Returns 0, 1 (null), 2 (shape), 4 (device), 7 (buffer small). */
int qsfb_prepare_sides(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br,
                       int bc, int on_device, int* meta, int* ranks, int max_gamma,
                       uint64_t* gamma, long long max_words, uint64_t* check, long long max_check,
                       uint32_t* red, long long max_red, uint32_t* syn, long long max_syn);

/* Report / witness / per-level counts of the last distance call on this thread. */
int qsfb_last_report(QsfbReport* out);
/* Witness codeword as 0/1 bytes (problem columns: n for CSS/classical, 3q after the
 * symplectic isometry); returns its length or -1. */
int qsfb_last_witness(uint8_t* out, int cap);
/* Level records: side[i], w[i], g[i], count[i] for every (level, active set); returns the
 * number of records (written up to cap). */
int qsfb_last_counts(int* side, int* w, int* g, unsigned long long* count, int cap);

/* ---- batched engine: many queries certified together (no reference counterpart; the
 * reference loops its per-code entry points).  Every query's levels of one round run in
 * one list-generation launch plus one pair-sweep launch per kernel variant; host setup is
 * spread over host_threads (0 = all cores).  Results equal the per-query entry points'. */
typedef struct {
    int kind;               /* 0 classical (A = H); 1 CSS distance (A = Hx, B = Hz);
                               2 CSS operator weight (A = Gx, B = Gz, z_op, x_op) */
    char which;             /* kind 1: 'Z', 'X' or 'M' (interleaved min) */
    const uint8_t* A;
    int a_rows, a_cols;
    const uint8_t* B;
    int b_rows, b_cols;
    const uint8_t* z_op;    /* kind 2: length a_cols */
    const uint8_t* x_op;
} QsfbQuery;

typedef struct {
    int distance;           /* kinds 0/1: distance (-1 undefined); kind 2: max(z, x) */
    int z_weight, x_weight; /* kind 2 */
    int lower_bound;
    int proven;
    int levels;
    int witness_ok;         /* 1: every certificate's witness verified on the host */
} QsfbAnswer;

typedef struct {
    double seconds;              /* wall time of the call */
    double prepare_seconds;      /* wall time of the prepare phase */
    double host_setup_seconds;   /* problem reduction + information sets + seed orders */
    double device_seed_seconds;  /* seed eliminations on the device (copy + kernel) */
    double device_ms;            /* list generation + pair sweeps (sum of kernel time) */
    double device_span_ms;       /* CUDA-event span of all rounds, host gaps included */
    double pair_ms;              /* pair-sweep kernel time alone */
    unsigned long long codewords;
    unsigned long long popc_issued;     /* POPC issued by the pair kernels */
    unsigned long long zero_codewords;  /* codewords swept by the popcount-free zero test */
    int rounds;
    int kernel_launches;
    int certificates;            /* BZ runs executed (a CSS 'M' query is one) */
    long long device_bytes;      /* device memory held by the batch (rows, seeds, lists) */
    double gen_ms;               /* list-generation kernel time */
    double host_plan_seconds;    /* host planning of the rounds (before their launches) */
    double host_apply_seconds;   /* host schedule updates after the rounds */
    unsigned long long tc_codewords;    /* codewords swept by the tensor-core kernel */
    double tc_ms;                /* tensor-core sweep launches alone (CUDA events) */
    double device_sets_seconds;  /* information sets + packed rows on the device (copies,
                                    kernels, read-back, host partition step) */
    unsigned long long tc_operand_bytes;  /* +-1 row bytes the tensor-core launches must read
                                             at least once (per round, the union of the row
                                             ranges of each list) */
    unsigned long long list_bytes_written;  /* bytes the list generation must write (probe
                                               words, pivot counts, +-1 rows) */
} QsfbBatchStats;

/* One-shot: prepare + execute + free.  Batches of 256 queries or more are pipelined in
 * chunks (the count of the library's tuning table, QSFB_BATCH_CHUNKS to change): the
 * first, small chunk's rounds start at once as three job groups, and each later chunk,
 * prepared meanwhile on all host cores but four, joins those groups at their next round
 * boundary.  The queries go to the chunks in the order of their shape's Gilbert-Varshamov
 * distance, largest first (later chunks join later, and a code needs one round per level;
 * QSFB_BATCH_ORDER=index keeps the caller's order).  out[i] answers queries[i] either way,
 * and the answers are those of one batch; the stats give the merged rounds and sum the
 * chunks' preparation phases (device_bytes: all chunks together).  QSFB_BATCH_TRACE prints
 * each chunk's phase times to stderr. */
int qsfb_batch(const QsfbQuery* queries, int nq, int host_threads, QsfbAnswer* out,
               QsfbBatchStats* stats);

/* Two-phase form: prepare does the host reduction, information sets and seed bounds of
 * every query and leaves the packed rows resident on the device; execute runs (or re-runs
 * from the post-prepare state) all BZ rounds and fills out[nq]; free releases everything.
 * Execute steps the queries as interleaved groups (QSFB_EXEC_GROUPS, default 3, at least 64
 * queries per group), each with its own stream and host thread, so that one group's host
 * planning overlaps the others' kernels; the answers do not depend on the grouping, and
 * device_span_ms is the span over all groups.  A handle is used by one thread at a time. */
typedef struct QsfbBatchHandle QsfbBatchHandle;
int qsfb_batch_prepare(const QsfbQuery* queries, int nq, int host_threads,
                       QsfbBatchHandle** handle);
int qsfb_batch_execute(QsfbBatchHandle* handle, QsfbAnswer* out, QsfbBatchStats* stats);
void qsfb_batch_free(QsfbBatchHandle* handle);

/* ---- serving: continuous batching of queries that arrive over time (no reference
 * counterpart).  submit() copies the query and returns at once; intake workers reduce it,
 * run its seed eliminations and upload its rows on their own CUDA streams while the device
 * keeps enumerating; an engine thread admits ready queries at every round boundary while
 * at most max_active are in flight and their summed device footprint (rows + all subset
 * lists their levels will build) stays within mem_budget_bytes (0 = 64 GiB), runs one
 * fused round over all admitted queries' next levels, and completes each query as soon as
 * it is proven.  Answers equal qsfb_batch's for the same query, alone or in any mix.
 * intake_threads = 0: all host cores but two.  start() grows the device memory pool behind
 * the allocator by QSFB_SERVER_RESERVE_MB (default 8192, at most the budget), so that a
 * request's first list of a new size is carved from mapped memory instead of mapping it
 * while the round waits.  For steady latencies start the process with
 * CUDA_MODULE_LOADING=EAGER (with lazy loading a kernel variant loads at its first launch,
 * which a request then waits for) and warm the server up with a few queries. */
typedef struct QsfbServer QsfbServer;
typedef struct {
    double submit_s, ready_s, admit_s, done_s;   /* seconds since the server started */
    double latency_s;                             /* done - submit */
} QsfbTiming;
typedef struct {
    long long submitted, completed;
    int active, pending;
    double busy_s;                 /* wall time spent in enumeration rounds */
    unsigned long long codewords;
    int rounds;
    long long peak_footprint_bytes;
    double elapsed_s;
} QsfbServeStats;
int qsfb_server_start(int intake_threads, long long mem_budget_bytes, int max_active,
                      QsfbServer** server);
int qsfb_server_submit(QsfbServer* server, const QsfbQuery* query, long long* ticket);
/* Blocks until the ticket's answer is ready; returns its status (0 ok). */
int qsfb_server_wait(QsfbServer* server, long long ticket, QsfbAnswer* out, QsfbTiming* timing);
int qsfb_server_stats(QsfbServer* server, QsfbServeStats* out);
/* Stops the threads (call after every submitted ticket has been waited for). */
int qsfb_server_stop(QsfbServer* server);

/* No counterpart in the reference.  qsfb_enumerate_plan for callers that cannot allocate
 * device memory (a process whose own pool owns the device, or code that must not cause the
 * device-wide synchronisation of a cudaMalloc).  Inputs and outputs are DEVICE pointers
 * owned by the caller: d_gamma (num_gamma*K*stride u64), d_check (kcheck*stride u64),
 * d_out_best (1 int), d_out_counts (num_gamma, may be NULL), d_out_g / d_out_rank (may be
 * NULL).  Results equal qsfb_enumerate_plan's.  All scratch sits in one fixed 32 MiB device
 * array inside the library (held on every GPU the library runs on until exit), shared by
 * every call: calls that overlap on the GPU race, so serialise them.  The first call on a
 * device sets the array up (its address, and a binomial table copied on `stream`); make it
 * before any stream capture.  The address stays cached while the library is loaded, so
 * after a cudaDeviceReset the library must be reloaded.  Limits: K <= 128, num_gamma <= 8,
 * kcheck <= 256, stride <= 16, d <= 64, C(K, d) < 2^62, and the level's subset lists within
 * the array; beyond them it returns 8 without touching the device.  stream: a cudaStream_t
 * (NULL = default stream); returns after the level has finished on that stream. */
int qsfb_enumerate_plan_noalloc(int n, int stride, int K, int d, int num_gamma,
                                const uint64_t* d_gamma, int kcheck, const uint64_t* d_check,
                                int current_best, int* d_out_best,
                                unsigned long long* d_out_counts, int* d_out_g,
                                unsigned long long* d_out_rank, void* stream);

/* The launch shapes in effect (no reference counterpart): `key value` lines -- the
 * tensor-core sweep's tile shape and job size per level-size class, the CUDA-core loop
 * tile, the tensor/CUDA-core cost ratio, the batch pipeline's group and chunk counts --
 * and where they came from (defaults, the tuning table beside the library written by
 * `python -m qubitserf_b200.tune`, QSFB_TUNING, QSFB_TUNE_<KEY>).  Returns 0, 1, 7. */
int qsfb_tuning(char* out, int cap);

/* Measured integer-pipe peak (ops/s over the whole device): which = 0 for 32-bit POPC
 * (the XU pipe), 1 for LOP3 (the ALU pipe).  Roofline denominators of the pair kernel. */
int qsfb_microbench(int which, double* ops_per_s);

/* Operand-layout self-test of the tensor-core pair sweep (no reference counterpart):
 * D = A * B^T over the first 32 * ksteps columns, with A 256 x 64 and B 128 x 64 int8
 * (row-major; the sweep stores +1 / -1 / 0) and D 256 x 128 int32 (row-major), computed
 * by the sweep's own copy, tcgen05 MMA and TMEM read-back path.  ksteps in 1..2.
 * packed = 1 reads the accumulators back as the sweep does (16-bit halves, two columns per
 * register; exact for |D| < 32768), 0 as 32-bit columns.  ksteps = -1 runs the timeout
 * drill: the operands are never copied, the kernel's bounded waits run out after 50 ms and
 * the call returns 4 with the device still usable.
 * Returns 0, 1 (null), 2 (ksteps), 4 (device or a wait that ran out) or 6 (memory). */
int qsfb_tc_selftest(int ksteps, int packed, const int8_t* A, const int8_t* B, int32_t* D);

/* Overwrite a 256 MiB device buffer (more than the 126 MB L2) and wait; benchmarks call it
 * between timed steps.  Returns 0, or 4 without a device. */
int qsfb_flush_l2(void);

/* Name of the device in use ("" without one) and its SM count. */
const char* qsfb_device_name(void);
int qsfb_device_sms(void);

/* Allocation calls that reached the CUDA driver since the device was opened (cache misses of
 * the device allocator; growth of sessions' pinned staging, which frees the old buffer
 * with a device-wide synchronisation), with their wall time in nanoseconds:
 * out[0] device allocations, out[1] their ns, out[2] pinned allocations, out[3] their ns.
 * Returns 0, 1 (null) or 4 (no device). */
int qsfb_alloc_counters(long long* out);

/* ---------------------------------------------------------------- Part 3: codeaut collector
 * The Brouwer-Zimmermann low-weight collector of the reference's codeaut engine, with the
 * handle ABI of cpp/codeaut/capi.h:51-72 that its Python (python/qubitserf/codeaut/
 * lowweight.py:53-78) binds with ctypes.  Every sw-subset (sw = 1..min(p, m)) of the rows
 * of the m x n 0/1 matrix G is XORed on the GPU; the distinct results of weight 1..keep
 * come back sorted by their packed 64-bit words, word 0 first (bit j of word w is column
 * 64 w + j), as the reference's handle holds them.  backend 0 ("cpu") is not run here: the
 * handle comes back with ok = 0; 1 and 2 run on the GPU.  threads is ignored.  Sizes beyond
 * n <= 1024, m <= 4096 and min(p, m) <= 64, or subset lists beyond device memory, also give
 * ok = 0.  The Leon automorphism engine (qaut_leon_*) of the same header is not part of this
 * library. */

/* Replaces codeaut_bz_collect, cpp/codeaut/capi.h:57-59.  Never NULL unless host memory
 * runs out; release with codeaut_bz_free. */
void* codeaut_bz_collect(const uint8_t* G, int32_t m, int32_t n, int32_t p,
                         int32_t keep_weight, int32_t backend, int32_t threads);
/* Replace codeaut_bz_ok / _count / _combos / _copy_rows / _backend / _free,
 * cpp/codeaut/capi.h:60-65. */
int32_t codeaut_bz_ok(void* h);
int64_t codeaut_bz_count(void* h);
int64_t codeaut_bz_combos(void* h);
void codeaut_bz_copy_rows(void* h, uint8_t* buf);
const char* codeaut_bz_backend(void* h);
void codeaut_bz_free(void* h);
/* Replaces codeaut_backend_available, cpp/codeaut/capi.h:68: "gpu"/"cuda"/"auto" -> 1 when
 * an sm_100 device is usable, anything else 0. */
int32_t codeaut_backend_available(const char* name);
/* Replaces codeaut_version, cpp/codeaut/capi.h:69. */
const char* codeaut_version(void);

/* No counterpart in the reference: what a collect handle's run did.  combos as
 * codeaut_bz_combos; hits = appended codewords before deduplication; passes = pairs whose
 * lower bound sent them to the exact evaluation; device times of the list generation and
 * of the pair sweeps (the last pass when an overflow made the sweep run twice). */
typedef struct {
    int64_t combos;
    int64_t hits;
    int64_t passes;
    int32_t probe_words;   /* 32-bit probe words per subset (1, 2, 4 or 8) */
    int32_t filter;        /* lower bound on their popcount: 0 exact sum, 2 / 4 popc of the
                              OR of 2 / 4 words, 6 carry-save over four words */
    int32_t pivots;        /* rows that own a private column */
    int32_t launches;
    int32_t reruns;        /* sweeps repeated after the output buffer overflowed */
    double gen_ms;
    double pairs_ms;
    double seconds;        /* wall time of codeaut_bz_collect */
    int32_t status;        /* 0, or the code of parts 1-2 that made ok = 0 */
} QsfbCollectStats;
int qsfb_collect_stats(void* h, QsfbCollectStats* out);

#ifdef __cplusplus
}
#endif

#endif /* QSF_B200_H */
