// extern "C" boundary of libqsfb200.so.  The distfind_* functions keep the reference's
// signatures, result structs, dispatch and return codes (cpp/distfind/capi.cpp:16-301);
// every accepted call runs on the GPU (method "bz": the BZ enumeration; "mitm": the
// meet-in-the-middle join of mitm.cu) and there is no CPU path.
#include "../../include/qsf_b200.h"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "bz.hpp"
#include "infoset_types.hpp"
#include "tuning.hpp"
#include "engine.hpp"
#include "mitm.hpp"
#include "problem.hpp"

using namespace qsfb;

namespace qsfb {
cudaError_t launch_tc_selftest(const int8_t* A, const int8_t* Bm, int ksteps, int packed,
                               int32_t* out, int* err, cudaStream_t st);
int tc_selftest_rows();
int tc_selftest_cols();
cudaError_t microbench_peak(int which, int num_sms, uint32_t* d_out, cudaStream_t st,
                            double* ops_per_s);
}

namespace {

struct LastCall {
    QsfbReport rep{};
    std::vector<u8> witness;
    std::vector<int> side, w, g;
    std::vector<unsigned long long> count;
};
thread_local LastCall g_last;

void record(const BzResult& r, int n_bits) {
    LastCall& L = g_last;
    std::memset(&L.rep, 0, sizeof(L.rep));
    L.rep.distance = r.distance;
    L.rep.lower_bound = r.lower_bound;
    L.rep.proven = r.proven ? 1 : 0;
    L.rep.levels = r.levels;
    L.rep.witness_ok = r.witness_ok ? 1 : 0;
    L.rep.witness_side = r.witness_side;
    L.rep.kernel_launches = r.stats.launches;
    L.rep.seconds = r.seconds;
    L.rep.device_ms = r.stats.ms_gen + r.stats.ms_pairs;
    L.rep.codewords = r.stats.codewords;
    L.witness.clear();
    if (!r.witness.empty()) {
        L.witness.resize(n_bits);
        for (int j = 0; j < n_bits; ++j)
            L.witness[j] = (u8)((r.witness[j >> 6] >> (j & 63)) & 1u);
    }
    L.rep.witness_bits = (int)L.witness.size();
    L.side.clear(); L.w.clear(); L.g.clear(); L.count.clear();
    for (const LevelRecord& lr : r.trace)
        for (size_t gi = 0; gi < lr.counts.size(); ++gi) {
            L.side.push_back(lr.side);
            L.w.push_back(lr.w);
            L.g.push_back((int)gi);
            L.count.push_back(lr.counts[gi]);
        }
}

void fill(DistfindResult* out, const BzResult& r) {
    out->distance = r.distance;
    out->lower_bound = r.lower_bound;
    out->proven = r.proven ? 1 : 0;
    out->levels = r.levels;
    out->seconds = r.seconds;
    std::strncpy(out->backend, "cuda", sizeof(out->backend) - 1);
    out->backend[sizeof(out->backend) - 1] = '\0';
}

// Method "mitm" runs the meet-in-the-middle join and any other name BZ, as in the
// reference's dispatch (cpp/distfind/capi.cpp:53-60, 79); "cc" (connected cluster) is not
// run here: callers that the reference sends to its cc solver get rc 5, the others map it
// before this check.  Only accelerator backends run.
int check_dispatch(const char* method, const char* backend) {
    const std::string m = method ? method : "bz";
    const std::string b = backend ? backend : "auto";
    if (m == "cc") return kErrUnsupported;
    if (b != "auto" && b != "gpu" && b != "cuda") return kErrUnsupported;
    return kOk;
}

Device* device_or(int* rc) {
    Device* d = Device::get(rc);
    if (!d) *rc = kErrDevice;
    return d;
}

BzOptions options(int verbose) {
    BzOptions o;
    o.verbose = verbose != 0;
    return o;
}

bool is_mitm(const char* method) { return method && std::strcmp(method, "mitm") == 0; }

// One subproblem by the requested method (cpp/distfind/capi.cpp:53-56, 79, 139-142).
int solve_one(Device* dev, const Problem& p, bool mitm, int verbose, BzResult& r) {
    return mitm ? mitm_distance(dev, p, r) : bz_distance(dev, p, options(verbose), r);
}

// Merge for the (non-interleaved) subsystem min, cpp/distfind/capi.cpp:147-156.
BzResult min_of(const BzResult& z, const BzResult& x) {
    auto v = [](int d) { return d < 0 ? (1 << 30) : d; };
    BzResult r = (v(x.distance) < v(z.distance)) ? x : z;
    r.distance = std::min(v(z.distance), v(x.distance));
    if (r.distance >= (1 << 30)) r.distance = -1;
    r.lower_bound = std::min(z.lower_bound, x.lower_bound);
    r.seconds = z.seconds + x.seconds;
    r.proven = z.proven && x.proven;
    r.levels = (v(x.distance) < v(z.distance)) ? x.levels : z.levels;
    r.stats.ms_gen = z.stats.ms_gen + x.stats.ms_gen;
    r.stats.ms_pairs = z.stats.ms_pairs + x.stats.ms_pairs;
    r.stats.codewords = z.stats.codewords + x.stats.codewords;
    r.stats.launches = z.stats.launches + x.stats.launches;
    r.trace = z.trace;
    for (LevelRecord lr : x.trace) { lr.side = 1; r.trace.push_back(lr); }
    return r;
}

// CSS routing shared by distfind_css_distance and the symplectic CSS fast path.
int css_like(Device* dev, const Mat& A, const Mat& B, bool subsystem, char which, bool mitm,
             int verbose, DistfindResult* out) {
    auto prob = [&](char w) {
        return subsystem ? subsystem_problem(A, B, w) : css_problem(A, B, w);
    };
    BzResult r;
    int rc;
    int nbits;
    if (which == 'Z' || which == 'X') {
        Problem p = prob(which);
        nbits = p.n;
        rc = solve_one(dev, p, mitm, verbose, r);
    } else if (subsystem) {
        Problem pz = prob('Z'), px = prob('X');
        nbits = pz.n;
        BzResult rz, rx;
        rc = solve_one(dev, pz, mitm, verbose, rz);
        if (rc == kOk) rc = solve_one(dev, px, mitm, verbose, rx);
        if (rc == kOk) r = min_of(rz, rx);
    } else {
        auto pr = css_problem_pair(A, B);
        nbits = pr.first.n;
        rc = mitm ? mitm_min_interleaved(dev, pr.first, pr.second, r)
                  : bz_min_interleaved(dev, pr.first, pr.second, options(verbose), r);
    }
    if (rc != kOk) return rc;
    fill(out, r);
    record(r, nbits);
    return kOk;
}

int symplectic_driver(const Mat& gauge, bool subsystem, const char* method, char which,
                      const char* backend, int verbose, DistfindResult* out) {
    if (gauge.cols % 2 != 0) return kErrShape;
    const std::string m = method ? method : "bz";
    const bool css = is_css_symplectic(gauge);
    if (m == "cc" && !css) return kErrMethod;
    int rc = check_dispatch(method, backend);
    if (rc != kOk) return rc;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    if (css) {
        auto hxhz = split_css(gauge);
        return css_like(dev, hxhz.first, hxhz.second, subsystem, which, is_mitm(method), verbose,
                        out);
    }
    Mat Snorm = subsystem ? symplectic_center(gauge) : gauge;
    Problem sp = symplectic_problem(Snorm, gauge);
    BzResult r;
    // mitm enumerates symplectic parts directly; bz goes through the isometry
    rc = is_mitm(method) ? mitm_distance(dev, sp, r)
                         : symplectic_bz_distance(dev, sp, options(verbose), r);
    if (rc != kOk) return rc;
    fill(out, r);
    record(r, 3 * sp.qubits);
    return kOk;
}

}  // namespace

struct QsfbBatchHandle {
    Device* dev = nullptr;
    std::vector<int> kinds;
    struct Map { int job0 = -1, job1 = -1; int zw = -1, xw = -1; };
    std::vector<Map> map;
    std::vector<std::unique_ptr<BzJob>> jobs;
    std::vector<BzJob*> ptrs;
    // declared after the jobs so that the arena outlives nothing that points into it
    std::unique_ptr<Arena> arena;
    std::unique_ptr<SessionLease> lease;
    RunStats setup;
    double prepare_s = 0.0;
    bool executed = false;
    ~QsfbBatchHandle() {
        jobs.clear();
        arena.reset();
        lease.reset();
    }
};

namespace {

// Background deletion of finished batch handles whose device memory and session have
// already been returned (only host memory is left).  One thread, started on first use and
// never joined; its queue and lock are never destroyed, so exit cannot race them.
void reap_later(QsfbBatchHandle* h) {
    struct Reaper {
        std::mutex mu;
        std::condition_variable cv;
        std::vector<QsfbBatchHandle*> q;
        Reaper() {
            std::thread([this]() {
                for (;;) {
                    std::vector<QsfbBatchHandle*> take;
                    {
                        std::unique_lock<std::mutex> lk(mu);
                        cv.wait(lk, [this]() { return !q.empty(); });
                        take.swap(q);
                    }
                    for (QsfbBatchHandle* x : take) delete x;
                }
            }).detach();
        }
    };
    static Reaper* r = new Reaper();
    {
        std::lock_guard<std::mutex> lk(r->mu);
        r->q.push_back(h);
    }
    r->cv.notify_one();
}

// Chunks of a one-shot batch prepared while the first chunk's rounds run: a helper thread
// publishes each prepared handle in order (nullptr if its preparation failed), and every
// job group takes its round-robin share of each published chunk at its next round boundary,
// so the chunks' rounds merge into one execution with one tail.
struct ChunkFeed {
    std::mutex mu;
    std::condition_variable cv;
    std::vector<QsfbBatchHandle*> ready;   // published chunks, in order
    size_t total = 0;                      // chunks that will be published
    void publish(QsfbBatchHandle* h) {
        {
            std::lock_guard<std::mutex> lk(mu);
            ready.push_back(h);
        }
        cv.notify_all();
    }
    // Group g of G: append its share of every chunk published since its last call
    // (`taken` chunks so far).  Idle: wait until a chunk gives it a job or all are published.
    bool take(std::vector<BzJob*>& jobs, size_t& taken, int g, int G, bool idle) {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            bool added = false;
            for (; taken < ready.size(); ++taken) {
                const QsfbBatchHandle* h = ready[taken];
                if (!h) continue;
                for (size_t j = (size_t)g; j < h->ptrs.size(); j += (size_t)G) {
                    jobs.push_back(h->ptrs[j]);
                    added = true;
                }
            }
            if (added || !idle || ready.size() >= total) return added;
            cv.wait(lk);
        }
    }
};

// The rounds of a prepared batch.  The jobs are independent, so they run as `groups`
// interleaved job groups (QSFB_EXEC_GROUPS, default 3; jobs dealt round robin), each
// stepping its own rounds on its own session and host thread: while one group's kernels
// run, the others plan and apply on the host, which hides the host share of each round.
// The span is the union over the groups, from one start event that every group's stream
// waits on to the last group's end event.
// With a feed, every group also takes its round-robin share of each chunk published
// during the rounds (`total_jobs`, all chunks' jobs, sets the group count).
int execute_groups(QsfbBatchHandle* H, RunStats* rs, int* rounds, double* span_ms,
                   int max_groups, ChunkFeed* F = nullptr, size_t total_jobs = 0) {
    const char* ge = std::getenv("QSFB_EXEC_GROUPS");   // read per call (benchmarks switch it)
    const int groups_env = std::max(1, std::min(ge ? std::atoi(ge) : tuning().exec_groups, 8));
    const size_t njobs = std::max(H->ptrs.size(), total_jobs);
    const int G = std::max(1, std::min({groups_env, max_groups, (int)(njobs / 64)}));
    std::vector<size_t> taken(G, 0);
    std::vector<JobFeed> feeds;
    for (int g = 0; g < G && F; ++g)
        feeds.emplace_back([F, &taken, g, G](std::vector<BzJob*>& jobs, bool idle) {
            return F->take(jobs, taken[g], g, G, idle);
        });
    std::vector<std::vector<BzJob*>> part(G);
    for (size_t j = 0; j < H->ptrs.size(); ++j) part[j % G].push_back(H->ptrs[j]);
    if (G == 1)
        return run_rounds(H->lease->s, part[0], rs, rounds, span_ms, F ? &feeds[0] : nullptr);
    std::vector<std::unique_ptr<SessionLease>> extra;
    std::vector<Session*> sess{H->lease->s};
    for (int g = 1; g < G; ++g) {
        extra.emplace_back(new SessionLease(H->dev));
        if (!extra.back()->s) return kErrDevice;
        sess.push_back(extra.back()->s);
    }
    cudaEvent_t start = nullptr;
    std::vector<cudaEvent_t> end(G, nullptr);
    bool ev_ok = cudaEventCreate(&start) == cudaSuccess;
    for (int g = 0; g < G && ev_ok; ++g) ev_ok = cudaEventCreate(&end[g]) == cudaSuccess;
    ev_ok = ev_ok && cudaEventRecord(start, sess[0]->stream) == cudaSuccess;
    for (int g = 1; g < G && ev_ok; ++g)
        ev_ok = cudaStreamWaitEvent(sess[g]->stream, start, 0) == cudaSuccess;
    if (!ev_ok) {
        cudaGetLastError();
        if (start) cudaEventDestroy(start);
        for (cudaEvent_t e : end) if (e) cudaEventDestroy(e);
        return kErrDevice;
    }
    std::vector<RunStats> st(G);
    std::vector<int> rr(G, 0), rcs(G, kOk);
    std::vector<std::thread> th;
    for (int g = 0; g < G; ++g)
        th.emplace_back([&, g]() {
            rcs[g] = run_rounds(sess[g], part[g], &st[g], &rr[g], nullptr,
                                F ? &feeds[g] : nullptr);
            if (cudaEventRecord(end[g], sess[g]->stream) != cudaSuccess) rcs[g] = kErrDevice;
        });
    for (std::thread& t : th) t.join();
    int rc = kOk;
    float span = 0.f;
    for (int g = 0; g < G; ++g) {
        if (rcs[g] != kOk && rc == kOk) rc = rcs[g];
        float ms = 0.f;
        if (cudaEventSynchronize(end[g]) == cudaSuccess &&
            cudaEventElapsedTime(&ms, start, end[g]) == cudaSuccess)
            span = std::max(span, ms);
        else if (rc == kOk)
            rc = kErrDevice;
        rs->host_plan_s += st[g].host_plan_s;
        rs->host_apply_s += st[g].host_apply_s;
        rs->ms_gen += st[g].ms_gen;
        rs->ms_pairs += st[g].ms_pairs;
        rs->ms_tc += st[g].ms_tc;
        rs->jobs += st[g].jobs;
        rs->codewords += st[g].codewords;
        rs->popc_issued += st[g].popc_issued;
        rs->zero_codewords += st[g].zero_codewords;
        rs->tc_codewords += st[g].tc_codewords;
        rs->tc_operand_bytes += st[g].tc_operand_bytes;
        rs->list_bytes_written += st[g].list_bytes_written;
        rs->launches += st[g].launches;
        *rounds = std::max(*rounds, rr[g]);
    }
    cudaGetLastError();
    cudaEventDestroy(start);
    for (cudaEvent_t e : end) cudaEventDestroy(e);
    if (span_ms) *span_ms = span;
    return rc;
}

// Witness rebuild, host verification and the per-query answers of an executed handle.
// Results (witness rebuild + host verification) of every job of the handles, independent
// per job: one pool over the host cores for all of them.
// Each job's final result (kept by the job; the rounds compute most of them as jobs
// finish, the rest -- trivially zero operator weights, say -- are computed here in parallel).
std::vector<std::vector<const BzResult*>> results_of(const std::vector<QsfbBatchHandle*>& Hs) {
    std::vector<std::vector<const BzResult*>> res(Hs.size());
    std::vector<std::pair<size_t, size_t>> work;
    for (size_t h = 0; h < Hs.size(); ++h) {
        res[h].resize(Hs[h]->jobs.size());
        for (size_t k = 0; k < Hs[h]->jobs.size(); ++k) work.emplace_back(h, k);
    }
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (size_t w; (w = next.fetch_add(1)) < work.size();)
            res[work[w].first][work[w].second] =
                &Hs[work[w].first]->jobs[work[w].second]->final_result();
    };
    const int nth = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(),
                                              (int)work.size() / 8 + 1));
    std::vector<std::thread> pool;
    for (int t = 1; t < nth; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return res;
}

// The per-query answers of an executed handle from its jobs' results.
void answers_of(QsfbBatchHandle* H, const std::vector<const BzResult*>& res, QsfbAnswer* out) {
    for (size_t i = 0; i < H->map.size(); ++i) {
        QsfbAnswer& a = out[i];
        std::memset(&a, 0, sizeof(a));
        const auto& m = H->map[i];
        if (H->kinds[i] == 2) {
            int zw = m.zw, xw = m.xw, lz = 0, lx = 0;
            bool ok = true, proven = true;
            if (m.job0 >= 0) {
                const BzResult& rz = *res[m.job0];
                zw = rz.distance; lz = rz.levels;
                ok &= rz.witness_ok || zw <= 0; proven &= rz.proven;
            }
            if (m.job1 >= 0) {
                const BzResult& rx = *res[m.job1];
                xw = rx.distance; lx = rx.levels;
                ok &= rx.witness_ok || xw <= 0; proven &= rx.proven;
            }
            a.z_weight = zw;
            a.x_weight = xw;
            a.distance = std::max(zw, xw);
            a.proven = proven ? 1 : 0;
            a.witness_ok = ok ? 1 : 0;
            a.levels = std::max(lz, lx);
        } else {
            const BzResult& r = *res[m.job0];
            a.distance = r.distance;
            a.lower_bound = r.lower_bound;
            a.proven = r.proven ? 1 : 0;
            a.levels = r.levels;
            a.witness_ok = (r.witness_ok || r.distance < 0) ? 1 : 0;
            a.z_weight = a.x_weight = -1;
        }
    }
}

// Execution figures of the rounds (whatever handles their jobs came from).
void fill_exec_stats(const RunStats& rs, int rounds, double span, QsfbBatchStats* stats) {
    stats->device_ms = rs.ms_gen + rs.ms_pairs;
    stats->device_span_ms = span;
    stats->pair_ms = rs.ms_pairs;
    stats->tc_ms = rs.ms_tc;
    stats->codewords = rs.codewords;
    stats->popc_issued = rs.popc_issued;
    stats->zero_codewords = rs.zero_codewords;
    stats->tc_codewords = rs.tc_codewords;
    stats->tc_operand_bytes = rs.tc_operand_bytes;
    stats->list_bytes_written = rs.list_bytes_written;
    stats->rounds = rounds;
    stats->kernel_launches = rs.launches;
    stats->gen_ms = rs.ms_gen;
    stats->host_plan_seconds = rs.host_plan_s;
    stats->host_apply_seconds = rs.host_apply_s;
}

int batch_execute(QsfbBatchHandle* H, QsfbAnswer* out, QsfbBatchStats* stats, int max_groups) {
    if (!H || (!out && !H->map.empty())) return kErrNull;
    const double t0 = now_seconds();
    if (H->executed)
        for (BzJob* j : H->ptrs) j->reset();
    H->executed = true;
    RunStats rs;
    int rounds = 0;
    double span = 0.0;
    int rc = execute_groups(H, &rs, &rounds, &span, max_groups);
    if (rc != kOk) return rc;
    answers_of(H, results_of({H})[0], out);
    if (stats) {
        fill_exec_stats(rs, rounds, span, stats);
        stats->seconds = now_seconds() - t0;
        stats->prepare_seconds = H->prepare_s;
        stats->host_setup_seconds = H->setup.host_setup_s;
        stats->device_seed_seconds = H->setup.device_seed_s;
        stats->device_sets_seconds = H->setup.device_sets_s;
        stats->certificates = (int)H->jobs.size();
        stats->device_bytes = (long long)H->arena->bytes();
    }
    return kOk;
}

}  // namespace

extern "C" {

int distfind_css_distance(const uint8_t* Hx, int hx_rows, int hx_cols, const uint8_t* Hz,
                          int hz_rows, int hz_cols, const char* method, char which,
                          const char* backend, int threads, int verbose, DistfindResult* out) {
    (void)threads;
    if (!out || !Hx || !Hz) return kErrNull;
    int rc = check_dispatch(method, backend);
    if (rc != kOk) return rc;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    Mat A = from_dense(Hx, hx_rows, hx_cols), B = from_dense(Hz, hz_rows, hz_cols);
    return css_like(dev, A, B, false, which, is_mitm(method), verbose, out);
}

int distfind_classical_distance(const uint8_t* H, int rows, int cols, const char* method,
                                const char* backend, int threads, int verbose,
                                DistfindResult* out) {
    (void)threads;
    if (!out || !H) return kErrNull;
    // the classical path has no cc form: the reference runs BZ for it (cpp/distfind/capi.cpp:79)
    const bool mitm = is_mitm(method);
    int rc = check_dispatch(mitm ? "mitm" : "bz", backend);
    if (rc != kOk) return rc;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    Problem p = classical_problem(from_dense(H, rows, cols));
    BzResult r;
    rc = solve_one(dev, p, mitm, verbose, r);
    if (rc != kOk) return rc;
    fill(out, r);
    record(r, p.n);
    return kOk;
}

int distfind_operator_weight(const uint8_t* Gx, int gx_rows, int gx_cols, const uint8_t* Gz,
                             int gz_rows, int gz_cols, const uint8_t* z_op, const uint8_t* x_op,
                             int n, const char* method, const char* backend, int threads,
                             int verbose, DistfindOpResult* out) {
    (void)threads;
    (void)n;
    if (!out || !Gx || !Gz || !z_op || !x_op) return kErrNull;
    std::string m = method ? method : "bz";
    if (m == "cc") {
        std::fprintf(stderr,
                     "distfind: operator weight has no connected-cluster form (the coset "
                     "parity-check is dense); using BZ instead.\n");
        m = "bz";
    }
    int rc = check_dispatch(m.c_str(), backend);
    if (rc != kOk) return rc;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    Mat A = from_dense(Gx, gx_rows, gx_cols), B = from_dense(Gz, gz_rows, gz_cols);
    double secs = 0.0;
    bool proven = true;
    BzResult last;
    int nbits = A.cols;
    // cpp/distfind/op_weight.cpp:9-36: Z part modulo rowspace(Gz), X part modulo rowspace(Gx).
    auto solve = [&](const Mat& G, const uint8_t* vec, int* res) -> int {
        if (in_rowspace(G, vec)) { *res = 0; return kOk; }
        Problem p = coset_problem(G, vec);
        BzResult r;
        const int e = solve_one(dev, p, m == "mitm", verbose, r);
        if (e != kOk) return e;
        secs += r.seconds;
        proven = proven && r.proven;
        last = r;
        *res = r.distance;
        return kOk;
    };
    int zw = -1, xw = -1;
    rc = solve(B, z_op, &zw);
    if (rc != kOk) return rc;
    rc = solve(A, x_op, &xw);
    if (rc != kOk) return rc;
    out->z_weight = zw;
    out->x_weight = xw;
    out->proven = proven ? 1 : 0;
    out->seconds = secs;
    std::strncpy(out->backend, "cuda", sizeof(out->backend) - 1);
    out->backend[sizeof(out->backend) - 1] = '\0';
    record(last, nbits);
    return kOk;
}

int distfind_subsystem_distance(const uint8_t* Gx, int gx_rows, int gx_cols, const uint8_t* Gz,
                                int gz_rows, int gz_cols, const char* method, char which,
                                const char* backend, int threads, int verbose,
                                DistfindResult* out) {
    (void)threads;
    if (!out || !Gx || !Gz) return kErrNull;
    int rc = check_dispatch(method, backend);
    if (rc != kOk) return rc;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    Mat A = from_dense(Gx, gx_rows, gx_cols), B = from_dense(Gz, gz_rows, gz_cols);
    return css_like(dev, A, B, true, which, is_mitm(method), verbose, out);
}

int distfind_stabilizer_distance(const uint8_t* S, int rows, int cols, const char* method,
                                 char which, const char* backend, int threads, int verbose,
                                 DistfindResult* out) {
    (void)threads;
    if (!out || !S) return kErrNull;
    return symplectic_driver(from_dense(S, rows, cols), false, method, which, backend, verbose,
                             out);
}

int distfind_subsystem_stabilizer_distance(const uint8_t* G, int rows, int cols,
                                           const char* method, char which, const char* backend,
                                           int threads, int verbose, DistfindResult* out) {
    (void)threads;
    if (!out || !G) return kErrNull;
    return symplectic_driver(from_dense(G, rows, cols), true, method, which, backend, verbose,
                             out);
}

int distfind_stabilizer_operator_weight(const uint8_t* G, int rows, int cols, const uint8_t* op,
                                        int op_len, const char* method, const char* backend,
                                        int threads, int verbose, DistfindResult* out) {
    (void)threads;
    if (!out || !G || !op) return kErrNull;
    if (cols % 2 != 0 || op_len != cols) return kErrShape;
    std::string m = method ? method : "bz";
    if (m == "cc") {   // cpp/distfind/capi.cpp:277-282
        std::fprintf(stderr,
                     "distfind: connected-cluster has no operator-weight form; using the "
                     "symplectic meet-in-the-middle search instead.\n");
        m = "mitm";
    }
    int rc = check_dispatch(m.c_str(), backend);
    if (rc != kOk) return rc;
    Mat mG = from_dense(G, rows, cols);
    BzResult r;
    if (in_rowspace(mG, op)) {
        r.distance = 0;
        r.lower_bound = 0;
        r.proven = true;
        fill(out, r);
        record(r, 0);
        return kOk;
    }
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    Problem sp = symplectic_coset_problem(mG, op);
    rc = m == "mitm" ? mitm_distance(dev, sp, r)
                     : symplectic_bz_distance(dev, sp, options(verbose), r);
    if (rc != kOk) return rc;
    fill(out, r);
    record(r, 3 * sp.qubits);
    return kOk;
}

int distfind_backend_available(const char* name) {
    const std::string b = name ? name : "auto";
    if (b == "gpu" || b == "cuda" || b == "auto") return Device::available() ? 1 : 0;
    return 0;
}

const char* distfind_version(void) { return "0.1.0"; }

// ---------------------------------------------------------------- Part 2
int qsfb_enumerate_plan(int n, int stride, int K, int d, int num_gamma, const uint64_t* gamma,
                        int kcheck, const uint64_t* check, int current_best, int* out_best,
                        unsigned long long* out_counts, int* out_g,
                        unsigned long long* out_rank) {
    if (!gamma || !out_best || (kcheck > 0 && !check)) return kErrNull;
    if (stride != words_for(n) || K < 1 || d < 1 || d > K || num_gamma < 1) return kErrShape;
    // sizes first: a level whose lists cannot exist is rejected before any device work
    int rc = level_size_rc(K, d);
    if (rc != kOk) return rc;
    if (num_gamma > 255) return kErrUnsupported;   // the witness key holds the set in 8 bits
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    // The reference weighs every bit of the `stride` words (cpp/qsf/bits.hpp:29-33), so a
    // raw plan is enumerated over stride*64 columns.
    const int ncols = stride * 64;
    Problem p;
    p.n = ncols;
    p.count_all = kcheck == 0;
    p.code_gen = Mat(K, ncols);
    p.check = Mat(kcheck, ncols);
    if (kcheck > 0) std::copy(check, check + (size_t)kcheck * stride, p.check.w.begin());
    std::vector<InfoSet> sets(num_gamma);
    for (int g = 0; g < num_gamma; ++g) {
        sets[g].g = Mat(K, ncols);
        std::copy(gamma + (size_t)g * K * stride, gamma + (size_t)(g + 1) * K * stride,
                  sets[g].g.w.begin());
        sets[g].rank = 0;   // raw rows: no pivot structure is assumed
    }
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    SideDev S;
    rc = S.prepare(p, sets);
    if (rc == kOk) rc = S.upload(dev, lease.s);
    if (rc != kOk) return rc;
    std::vector<LevelReq> q(1);
    q[0].side = &S;
    q[0].w = d;
    q[0].active = num_gamma;
    q[0].bound = current_best >= kWeightNone ? 4094 : current_best - 1;
    std::vector<LevelOut> o;
    rc = run_levels(lease.s, q, o, nullptr);
    if (rc != kOk) return rc;
    *out_best = o[0].found ? std::min(current_best, o[0].wt) : current_best;
    if (out_counts)
        for (int g = 0; g < num_gamma; ++g) out_counts[g] = o[0].counts[g];
    if (out_g) *out_g = o[0].found ? o[0].g : -1;
    if (out_rank) *out_rank = o[0].found ? o[0].rank : ~0ull;
    return kOk;
}

namespace {
// The BZ subproblem of one query kind (the reductions qsfb_prepare_problem documents).
int kind_problem(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br, int bc,
                 Problem* p) {
    Mat mA = from_dense(A, ar, ac);
    Mat mB = (B && br > 0) ? from_dense(B, br, bc) : Mat(0, ac);
    switch (kind) {
        case 0: *p = classical_problem(mA); break;
        case 1: *p = css_problem(mA, mB, 'Z'); break;
        case 2: *p = css_problem(mA, mB, 'X'); break;
        case 3: *p = subsystem_problem(mA, mB, 'Z'); break;
        case 4: *p = subsystem_problem(mA, mB, 'X'); break;
        case 5:
            if (ac % 2) return kErrShape;
            *p = isometry_extend(symplectic_problem(mA, mA));
            break;
        default: return kErrShape;
    }
    return kOk;
}

int write_sets(const Problem& p, const std::vector<InfoSet>& sets, int* meta, int* ranks,
               int max_gamma, uint64_t* gamma, long long max_words, uint64_t* check,
               long long max_check) {
    const int K = p.code_gen.rows, stride = words_for(p.n);
    const int ng = (int)sets.size();
    const int kcheck = p.count_all ? 0 : p.check.rows;
    meta[0] = p.n; meta[1] = K; meta[2] = ng; meta[3] = kcheck;
    meta[4] = p.even ? 1 : 0; meta[5] = p.count_all ? 1 : 0; meta[6] = p.seed_upper;
    meta[7] = stride;
    if (ng > max_gamma || (long long)ng * K * stride > max_words ||
        (long long)kcheck * stride > max_check)
        return 7;
    for (int g = 0; g < ng; ++g) {
        if (ranks) ranks[g] = sets[g].rank;
        if (gamma)
            std::copy(sets[g].g.w.begin(), sets[g].g.w.end(), gamma + (size_t)g * K * stride);
    }
    if (check)
        for (int c = 0; c < kcheck; ++c)
            std::copy(p.check.row(c), p.check.row(c) + stride, check + (size_t)c * stride);
    return kOk;
}
}  // namespace

int qsfb_prepare_problem(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br,
                         int bc, int* meta, int* ranks, int max_gamma, uint64_t* gamma,
                         long long max_words, uint64_t* check, long long max_check) {
    if (!A || !meta) return kErrNull;
    Problem p;
    const int rc = kind_problem(kind, A, ar, ac, B, br, bc, &p);
    if (rc != kOk) return rc;
    std::vector<InfoSet> sets;
    if (p.code_gen.rows > 0) sets = information_sets(p.code_gen);
    return write_sets(p, sets, meta, ranks, max_gamma, gamma, max_words, check, max_check);
}

int qsfb_prepare_sides(int kind, const uint8_t* A, int ar, int ac, const uint8_t* B, int br,
                       int bc, int on_device, int* meta, int* ranks, int max_gamma,
                       uint64_t* gamma, long long max_words, uint64_t* check, long long max_check,
                       uint32_t* red, long long max_red, uint32_t* syn, long long max_syn) {
    if (!A || !meta) return kErrNull;
    Problem p;
    int rc = kind_problem(kind, A, ar, ac, B, br, bc, &p);
    if (rc != kOk) return rc;
    const int K = p.code_gen.rows;
    const int kcheck = p.count_all ? 0 : p.check.rows;
    const int W32 = (p.n + 31) / 32, SWP = std::max(1, (kcheck + 31) / 32);
    meta[8] = W32;
    meta[9] = SWP;
    meta[10] = 0;
    meta[11] = 0;
    if (K == 0) return write_sets(p, {}, meta, ranks, max_gamma, gamma, max_words, check, max_check);
    BzSide S;   // only its information sets and device image are used
    S.prob = &p;
    S.K = K;
    std::unique_ptr<Arena> arena;
    std::unique_ptr<SessionLease> lease;
    const bool dev_ok = on_device && K <= kInfosetMaxK && p.n <= kInfosetMaxN;
    if (dev_ok) {
        Device* dev = device_or(&rc);
        if (!dev) return rc;
        lease.reset(new SessionLease(dev));
        if (!lease->s) return kErrDevice;
        arena.reset(new Arena(dev, 1ull << 20));
        S.infoset_pending = true;
        rc = device_infosets(lease->s, arena.get(), {&S}, nullptr);
        if (rc != kOk) return rc;
        meta[10] = S.dev.device_rows ? 1 : 0;
        meta[11] = S.sets_from_classes ? 1 : 0;
    } else {
        rc = S.adopt_sets(information_sets(p.code_gen), nullptr, nullptr, 0, 0, nullptr, nullptr);
        if (rc != kOk) return rc;
    }
    rc = write_sets(p, S.sets, meta, ranks, max_gamma, gamma, max_words, check, max_check);
    if (rc != kOk) return rc;
    const int ng = S.ng;
    if ((red && (long long)ng * K * W32 > max_red) || (syn && (long long)ng * K * SWP > max_syn))
        return 7;
    const SideDev& D = S.dev;
    std::vector<uint32_t> hr, hs;
    if (D.device_rows) {
        hr.resize((size_t)ng * K * W32);
        hs.resize((size_t)ng * K * SWP);
        if (cudaMemcpy(hr.data(), D.d_red, hr.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(hs.data(), D.d_syn, hs.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            cudaGetLastError();
            return kErrDevice;
        }
    } else {   // host rows: re-stride to W32 = ceil(n/32) words, zero padded
        hr.assign((size_t)ng * K * W32, 0u);
        for (size_t r = 0; r < (size_t)ng * K; ++r)
            std::copy(D.h_red.begin() + r * D.W32, D.h_red.begin() + (r + 1) * D.W32,
                      hr.begin() + r * W32);
        hs = D.h_syn;
    }
    if (red) std::copy(hr.begin(), hr.end(), red);
    if (syn) std::copy(hs.begin(), hs.end(), syn);
    return kOk;
}

int qsfb_last_report(QsfbReport* out) {
    if (!out) return kErrNull;
    *out = g_last.rep;
    return kOk;
}

int qsfb_last_witness(uint8_t* out, int cap) {
    if (g_last.witness.empty()) return -1;
    const int n = (int)g_last.witness.size();
    if (out) std::copy(g_last.witness.begin(), g_last.witness.begin() + std::min(n, cap), out);
    return n;
}

int qsfb_last_counts(int* side, int* w, int* g, unsigned long long* count, int cap) {
    const int n = (int)g_last.count.size();
    for (int i = 0; i < std::min(n, cap); ++i) {
        if (side) side[i] = g_last.side[i];
        if (w) w[i] = g_last.w[i];
        if (g) g[i] = g_last.g[i];
        if (count) count[i] = g_last.count[i];
    }
    return n;
}

namespace {

// Host phase of qsfb_batch_prepare: the handle, its jobs and their host setup.
int batch_prepare_host(const QsfbQuery* queries, int nq, int host_threads,
                       QsfbBatchHandle** handle) {
    if ((!queries && nq > 0) || !handle) return kErrNull;
    *handle = nullptr;
    const double tp0 = now_seconds();
    int rc = kOk;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    auto* H = new QsfbBatchHandle();
    H->dev = dev;
    H->kinds.resize(nq);
    H->map.resize(nq);
    BzOptions opt;
    opt.parallel_seed = false;   // the batch parallelizes over codes instead
    auto& jobs = H->jobs;
    // Problems are built inside the parallel job setup (deferred builders); the query's
    // host matrices only need to live until prepare returns.
    for (int i = 0; i < nq; ++i) {
        const QsfbQuery q = queries[i];
        H->kinds[i] = q.kind;
        if (!q.A || (q.kind != 0 && !q.B) || (q.kind == 2 && (!q.z_op || !q.x_op))) {
            delete H;
            return kErrNull;
        }
        if (q.kind < 0 || q.kind > 2) { delete H; return kErrShape; }
        auto& m = H->map[i];
        if (q.kind == 0) {
            m.job0 = (int)jobs.size();
            jobs.emplace_back(new BzJob([q](Problem& p0, Problem&) {
                p0 = classical_problem(from_dense(q.A, q.a_rows, q.a_cols));
                return 0;
            }, false, opt));
        } else if (q.kind == 1) {
            m.job0 = (int)jobs.size();
            const bool single = q.which == 'Z' || q.which == 'X';
            jobs.emplace_back(new BzJob([q, single](Problem& p0, Problem& p1) {
                Mat A = from_dense(q.A, q.a_rows, q.a_cols), B = from_dense(q.B, q.b_rows, q.b_cols);
                if (single) {
                    p0 = css_problem(A, B, q.which);
                } else {
                    auto pr = css_problem_pair(A, B);
                    p0 = std::move(pr.first);
                    p1 = std::move(pr.second);
                }
                return 0;
            }, !single, opt));
        } else {
            // Z part modulo rowspace(Gz), X part modulo rowspace(Gx) (op_weight.cpp:9-36)
            m.job0 = (int)jobs.size();
            jobs.emplace_back(new BzJob([q](Problem& p0, Problem&) {
                Mat B = from_dense(q.B, q.b_rows, q.b_cols);
                if (in_rowspace(B, q.z_op)) return 1;
                p0 = coset_problem(B, q.z_op);
                return 0;
            }, false, opt));
            m.job1 = (int)jobs.size();
            jobs.emplace_back(new BzJob([q](Problem& p0, Problem&) {
                Mat A = from_dense(q.A, q.a_rows, q.a_cols);
                if (in_rowspace(A, q.x_op)) return 1;
                p0 = coset_problem(A, q.x_op);
                return 0;
            }, false, opt));
        }
    }
    for (auto& j : jobs) H->ptrs.push_back(j.get());
    H->lease.reset(new SessionLease(dev));
    if (!H->lease->s) { delete H; return kErrDevice; }
    H->arena.reset(new Arena(dev));
    rc = setup_jobs_host(H->ptrs, host_threads, &H->setup);
    if (rc != kOk) { delete H; return rc; }
    H->prepare_s = now_seconds() - tp0;
    *handle = H;
    return kOk;
}

// Device phase: seed eliminations and upload.  On failure the handle is freed and nulled.
int batch_prepare_device(QsfbBatchHandle*& H) {
    const double t0 = now_seconds();
    const int rc = setup_jobs_device(H->dev, H->lease->s, H->arena.get(), H->ptrs, &H->setup);
    if (rc != kOk) {
        delete H;
        H = nullptr;
        return rc;
    }
    H->prepare_s += now_seconds() - t0;
    return kOk;
}

}  // namespace

int qsfb_batch_prepare(const QsfbQuery* queries, int nq, int host_threads,
                       QsfbBatchHandle** handle) {
    const int rc = batch_prepare_host(queries, nq, host_threads, handle);
    if (rc != kOk) return rc;
    return batch_prepare_device(*handle);
}

int qsfb_batch_execute(QsfbBatchHandle* H, QsfbAnswer* out, QsfbBatchStats* stats) {
    return batch_execute(H, out, stats, 8);
}


void qsfb_batch_free(QsfbBatchHandle* H) { delete H; }

// One-shot batch.  A large batch is cut into chunks: the first (small, so the device
// starts early) is prepared on all host cores and its rounds start; a helper thread
// prepares the others in order (host reduction, then the seed trials and information sets
// on the device, beside the next chunk's host reduction) and publishes each to the running
// job groups, which take their share of its jobs at their next round boundary: the chunks'
// rounds merge into one execution with one tail.  Codes are independent and a job's answer
// depends only on its own levels, so the answers are those of one batch.
namespace {
// Inverse of the binary entropy on [0, 1/2], to 1/8192: a table of H2 on that grid (made
// once) and a binary search in it.
double h2_inverse(double y) {
    static const std::vector<double> H = [] {
        std::vector<double> t(4097);
        for (int i = 0; i <= 4096; ++i) {
            const double p = i / 8192.0;
            t[i] = i == 0 ? 0.0 : -p * std::log2(p) - (1.0 - p) * std::log2(1.0 - p);
        }
        return t;
    }();
    if (y >= 1.0) return 0.5;
    return (double)(std::lower_bound(H.begin(), H.end(), y) - H.begin()) / 8192.0;
}
// Distance of a random code of the query's shape (Gilbert-Varshamov): n H2^-1(r / n) for r
// independent checks; a CSS query's Z (X) logicals lie in the kernel of its X (Z) checks,
// and its certificate ends with the lighter side.
double gv_distance_estimate(const QsfbQuery& q) {
    const int n = q.a_cols;
    if (n <= 0) return 0.0;
    auto gv = [n](int rows) { return n * h2_inverse(std::min(rows, n) / (double)n); };
    if (q.kind == 0) return gv(q.a_rows);
    if (q.kind == 1 && q.which == 'Z') return gv(q.a_rows);
    if (q.kind == 1 && q.which == 'X') return gv(q.b_rows);
    return std::min(gv(q.a_rows), gv(q.b_rows));
}
}  // namespace

int qsfb_batch(const QsfbQuery* queries, int nq, int host_threads, QsfbAnswer* out,
               QsfbBatchStats* stats) {
    const double t0 = now_seconds();
    const bool trace = std::getenv("QSFB_BATCH_TRACE") != nullptr;
    long long alloc0[4] = {0, 0, 0, 0};
    int trc = kOk;
    Device* tdev = trace ? device_or(&trc) : nullptr;
    if (tdev) {
        alloc0[0] = tdev->n_device_malloc; alloc0[1] = tdev->ns_device_malloc;
        alloc0[2] = tdev->n_pinned_alloc; alloc0[3] = tdev->ns_pinned_alloc;
    }
    constexpr int kPipeMin = 256;   // below this the batch runs in one piece
    // QSFB_BATCH_CHUNKS: number of pipeline chunks (default: the tuning table's; 1 = one
    // piece), read per call.
    const char* ce = std::getenv("QSFB_BATCH_CHUNKS");
    const int chunks = std::max(1, std::min(ce ? std::atoi(ce) : tuning().batch_chunks, 64));
    std::vector<int> cut{0};
    if (nq >= kPipeMin && chunks > 1) {
        const int fp = tuning().batch_first_permille;
        const int first = std::min(nq - (chunks - 1),
                                   std::max(32, fp > 0 ? (int)((long long)nq * fp / 1000)
                                                       : nq / (2 * chunks)));
        cut.push_back(first);
        const int rest = nq - first, parts = chunks - 1;
        for (int i = 1; i <= parts; ++i) cut.push_back(first + (int)((long long)rest * i / parts));
    } else {
        cut.push_back(nq);
    }
    const int nchunks = (int)cut.size() - 1;
    // Chunk order: later chunks join the rounds later, and a code needs one round per level
    // after it joins, so the codes expected to need the most levels go first.  The estimate
    // is the Gilbert-Varshamov distance of the code's shape (a random code of its length and
    // rate); it only orders the work, and every answer is the same in any order
    // (QSFB_BATCH_ORDER=index keeps the caller's order).
    std::vector<int> order;
    std::vector<QsfbQuery> ordered;
    const char* oe = std::getenv("QSFB_BATCH_ORDER");
    if (nchunks > 1 && !(oe && std::strcmp(oe, "index") == 0)) {
        order.resize(nq);
        std::vector<double> est(nq);
        for (int i = 0; i < nq; ++i) {
            order[i] = i;
            est[i] = gv_distance_estimate(queries[i]);
        }
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return est[a] > est[b]; });
        ordered.resize(nq);
        for (int i = 0; i < nq; ++i) ordered[i] = queries[order[i]];
        queries = ordered.data();
    }
    std::vector<QsfbBatchHandle*> H(nchunks, nullptr);
    std::vector<int> prc(nchunks, kOk);
    std::vector<double> tp0(nchunks), tp1(nchunks);
    // Preparations that run beside the rounds leave four host cores to the job groups'
    // round planning (QSFB_OVERLAP_PREP_THREADS to set the count); the merged execution
    // steps QSFB_OVERLAP_GROUPS job groups (default 3).
    const char* pe = std::getenv("QSFB_OVERLAP_PREP_THREADS");
    const char* ge = std::getenv("QSFB_OVERLAP_GROUPS");
    const int all = host_threads > 0 ? host_threads
                                     : std::max(1, (int)std::thread::hardware_concurrency());
    const int overlap_threads = pe ? std::max(1, std::atoi(pe)) : std::max(1, all - 4);
    const int overlap_groups = ge ? std::max(1, std::atoi(ge)) : tuning().overlap_groups;
    auto prepare = [&](int c) {
        tp0[c] = now_seconds();
        prc[c] = qsfb_batch_prepare(queries + cut[c], cut[c + 1] - cut[c],
                                    c == 0 ? host_threads : overlap_threads, &H[c]);
        tp1[c] = now_seconds();
    };
    // the chunks' device memory and sessions go back at once; the host-side teardown of
    // their jobs (many small frees) runs on a background thread after the call returns
    auto release = [&]() {
        for (QsfbBatchHandle*& h : H) {
            if (!h) continue;
            h->arena.reset();
            h->lease.reset();
            reap_later(h);
            h = nullptr;
        }
    };
    if (nchunks == 1) {
        prepare(0);
        if (prc[0] != kOk) return prc[0];
        const int rc = batch_execute(H[0], out, stats, 8);
        release();
        if (stats) stats->seconds = now_seconds() - t0;
        return rc;
    }
    prepare(0);
    if (prc[0] != kOk) return prc[0];
    ChunkFeed F;
    F.total = (size_t)(nchunks - 1);
    // The helper prepares chunks 1.. in order, in two phases: while chunk c's seed
    // eliminations and upload run (the host mostly waiting for the device), chunk c + 1's
    // host reduction runs beside them.
    auto prepare_host = [&](int c) {
        tp0[c] = now_seconds();
        prc[c] = batch_prepare_host(queries + cut[c], cut[c + 1] - cut[c], overlap_threads,
                                    &H[c]);
    };
    std::thread helper([&]() {
        prepare_host(1);
        for (int c = 1; c < nchunks; ++c) {
            std::thread next;
            if (c + 1 < nchunks) next = std::thread(prepare_host, c + 1);
            if (prc[c] == kOk) prc[c] = batch_prepare_device(H[c]);
            tp1[c] = now_seconds();
            F.publish(prc[c] == kOk ? H[c] : nullptr);
            if (next.joinable()) next.join();
        }
    });
    RunStats rs;
    int rounds = 0;
    double span = 0.0;
    const double te0 = now_seconds();
    H[0]->executed = true;
    int rc = execute_groups(H[0], &rs, &rounds, &span, overlap_groups, &F, (size_t)nq);
    const double te1 = now_seconds();
    helper.join();
    for (int c = 0; c < nchunks && rc == kOk; ++c)
        if (prc[c] != kOk) rc = prc[c];
    if (rc == kOk && out) {
        const std::vector<std::vector<const BzResult*>> res = results_of(H);
        std::vector<QsfbAnswer> tmp(order.empty() ? 0 : nq);
        QsfbAnswer* o = order.empty() ? out : tmp.data();
        for (int c = 0; c < nchunks; ++c) answers_of(H[c], res[c], o + cut[c]);
        for (size_t i = 0; i < order.size(); ++i) out[order[i]] = tmp[i];
    }
    const double ta1 = now_seconds();
    if (tdev)
        std::fprintf(stderr, "qsfb_batch: %lld device allocations (%.2f ms), %lld pinned "
                     "staging allocations (%.2f ms)\n", tdev->n_device_malloc - alloc0[0],
                     1e-6 * (double)(tdev->ns_device_malloc - alloc0[1]),
                     tdev->n_pinned_alloc - alloc0[2],
                     1e-6 * (double)(tdev->ns_pinned_alloc - alloc0[3]));
    if (trace)   // one stderr line per chunk (ms from the call)
        for (int c = 0; c < nchunks; ++c)
            std::fprintf(stderr, "qsfb_batch chunk %d: %d codes, prepare %.2f-%.2f ms (host "
                         "reduction %.2f ms, device seeds %.2f ms of which %.2f waiting, "
                         "device sets %.2f ms); rounds %.2f-%.2f ms\n", c,
                         cut[c + 1] - cut[c], 1e3 * (tp0[c] - t0), 1e3 * (tp1[c] - t0),
                         H[c] ? 1e3 * H[c]->setup.host_setup_s : 0.0,
                         H[c] ? 1e3 * H[c]->setup.device_seed_s : 0.0,
                         H[c] ? 1e3 * H[c]->setup.device_seed_wait_s : 0.0,
                         H[c] ? 1e3 * H[c]->setup.device_sets_s : 0.0, 1e3 * (te0 - t0),
                         1e3 * (te1 - t0));
    if (stats && rc == kOk) {
        std::memset(stats, 0, sizeof(*stats));
        fill_exec_stats(rs, rounds, span, stats);
        for (QsfbBatchHandle* h : H) {
            stats->prepare_seconds += h->prepare_s;
            stats->host_setup_seconds += h->setup.host_setup_s;
            stats->device_seed_seconds += h->setup.device_seed_s;
            stats->device_sets_seconds += h->setup.device_sets_s;
            stats->certificates += (int)h->jobs.size();
            stats->device_bytes += (long long)h->arena->bytes();
        }
        stats->seconds = now_seconds() - t0;
    }
    release();
    if (trace)
        std::fprintf(stderr, "qsfb_batch: answers %.2f ms, release %.2f ms, call %.2f ms\n",
                     1e3 * (ta1 - te1), 1e3 * (now_seconds() - ta1), 1e3 * (now_seconds() - t0));
    return rc;
}

int qsfb_tuning(char* out, int cap) {
    if (!out || cap <= 0) return kErrNull;
    const Tuning& t = tuning();
    const int n = std::snprintf(
        out, (size_t)cap,
        "tc_shape %d\ntc_job_tiles.small %d\ntc_job_tiles.large %d\ntc_small_tiles %lld\n"
        "cc_jobs_per_warp %d\ntc_cost_ratio %g\ntc_edge_div %d\nexec_groups %d\nbatch_chunks %d\n"
        "overlap_groups %d\nbatch_first_permille %d\nsource %s\n",
        t.tc_shape, t.tc_job_tiles_small, t.tc_job_tiles_large, t.tc_small_tiles,
        t.cc_jobs_per_warp, t.tc_cost_ratio, t.tc_edge_div, t.exec_groups, t.batch_chunks,
        t.overlap_groups,
        t.batch_first_permille, t.source.c_str());
    return n < cap ? kOk : 7;
}

int qsfb_microbench(int which, double* ops_per_s) {
    if (!ops_per_s) return kErrNull;
    int rc = kOk;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    void* out = dev->alloc((size_t)dev->num_sms * 8 * 4);
    if (!out) return kErrMemory;
    const cudaError_t e = microbench_peak(which, dev->num_sms, (uint32_t*)out, lease.s->stream,
                                          ops_per_s);
    dev->release(out, (size_t)dev->num_sms * 8 * 4);
    return e == cudaSuccess ? kOk : kErrDevice;
}

int qsfb_tc_selftest(int ksteps, int packed, const int8_t* A, const int8_t* B, int32_t* D) {
    if (!A || !B || !D) return kErrNull;
    if (ksteps == 0 || ksteps < -1 || ksteps > kPmRowBytes / 32) return kErrShape;
    int rc = kOk;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    const int rows_a = tc_selftest_rows(), rows_b = tc_selftest_cols();
    const size_t bytes_a = (size_t)rows_a * kPmRowBytes, bytes_b = (size_t)rows_b * kPmRowBytes;
    const size_t bytes_d = (size_t)rows_a * rows_b * 4;
    // host swizzle: 16-byte chunk j of row e goes to chunk j ^ ((e >> 1) & 3)
    std::vector<int8_t> h((size_t)(rows_a + rows_b) * kPmRowBytes);
    auto put = [&](const int8_t* src, int rows, int8_t* dst) {
        for (int e = 0; e < rows; ++e)
            for (int j = 0; j < kPmRowBytes / 16; ++j)
                std::memcpy(dst + (size_t)e * kPmRowBytes + (size_t)((j ^ ((e >> 1) & 3)) * 16),
                            src + (size_t)e * kPmRowBytes + (size_t)j * 16, 16);
    };
    put(A, rows_a, h.data());
    put(B, rows_b, h.data() + bytes_a);
    const size_t total = bytes_a + bytes_b + bytes_d + 256;
    char* buf = (char*)dev->alloc(total);
    if (!buf) return kErrMemory;
    int8_t* dA = (int8_t*)buf;
    int8_t* dB = (int8_t*)(buf + bytes_a);
    int32_t* dD = (int32_t*)(buf + bytes_a + bytes_b);
    int* dErr = (int*)(buf + bytes_a + bytes_b + bytes_d);
    cudaStream_t st = lease.s->stream;
    int herr = 0;
    bool ok = cudaMemcpyAsync(buf, h.data(), bytes_a + bytes_b, cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemsetAsync(dErr, 0, sizeof(int), st) == cudaSuccess &&
              launch_tc_selftest(dA, dB, ksteps, packed, dD, dErr, st) == cudaSuccess &&
              cudaMemcpyAsync(D, dD, bytes_d, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
              cudaMemcpyAsync(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
              cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) cudaGetLastError();
    dev->release(buf, total);
    return ok && herr == 0 ? kOk : kErrDevice;
}

int qsfb_flush_l2(void) {
    int rc = kOk;
    Device* dev = device_or(&rc);
    if (!dev) return rc;
    static void* buf = nullptr;
    const size_t bytes = 256ull << 20;
    if (!buf) buf = dev->alloc(bytes);
    if (!buf) return kErrMemory;
    SessionLease lease(dev);
    if (!lease.s) return kErrDevice;
    if (cudaMemsetAsync(buf, 0x5a, bytes, lease.s->stream) != cudaSuccess ||
        cudaStreamSynchronize(lease.s->stream) != cudaSuccess) {
        cudaGetLastError();
        return kErrDevice;
    }
    return kOk;
}

const char* qsfb_device_name(void) {
    int rc = 0;
    Device* d = Device::get(&rc);
    return d ? d->name.c_str() : "";
}

int qsfb_device_sms(void) {
    int rc = 0;
    Device* d = Device::get(&rc);
    return d ? d->num_sms : 0;
}

int qsfb_alloc_counters(long long* out) {
    if (!out) return kErrNull;
    int rc = kOk;
    Device* d = device_or(&rc);
    if (!d) return rc;
    out[0] = d->n_device_malloc;
    out[1] = d->ns_device_malloc;
    out[2] = d->n_pinned_alloc;
    out[3] = d->ns_pinned_alloc;
    return kOk;
}

}  // extern "C"
