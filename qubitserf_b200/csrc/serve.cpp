// Continuous-batching server for distance / operator-weight queries on one device.
//
//  submit()  -> the query's matrices are copied, a ticket is returned at once.
//  intake    -> a pool of workers reduces each request (problem, information sets, seed
//               column orders), runs its seed eliminations and uploads its rows on the
//               worker's own CUDA stream, while the device keeps enumerating;
//  engine    -> one thread admits ready requests at every round boundary while the number
//               of active requests and the summed device footprint (rows + every subset
//               list its levels will build, computed exactly from the level plan) stay
//               within the limits, then runs ONE round over every active request's next
//               level (one list-generation launch + one pair launch per kernel variant),
//               and completes each request the moment its certificates are proven.
// A request's answer depends only on its own levels (each level's result is the minimum
// witness key over its own candidates), so it is the same alone and in any mix.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/qsf_b200.h"
#include "bz.hpp"
#include "engine.hpp"

using namespace qsfb;

namespace {

struct OwnedQuery {
    int kind = 0;
    char which = 'M';
    int ar = 0, ac = 0, br = 0, bc = 0;
    std::vector<u8> A, B, z, x;
};

struct Request {
    long long id = 0;
    OwnedQuery q;
    std::vector<std::unique_ptr<BzJob>> jobs;
    std::unique_ptr<Arena> arena;
    size_t footprint = 0;
    double t_submit = 0, t_ready = 0, t_admit = 0, t_done = 0;
    int status = kOk;
    bool done = false;
    QsfbAnswer ans{};
};

// Bytes of every subset list the levels up to the side's stopping level will build, by the
// level plan of run_levels (prefix/suffix sizes a, b; HP words per entry; pivot counts for
// rank-deficient sets).
size_t list_footprint(Device* dev, const BzSide& S) {
    if (!S.has_logicals) return 0;
    int wmax = S.K;
    for (int w = 1; w <= S.K; ++w)
        if (S.outer_at(w) >= S.inner) { wmax = w; break; }
    size_t bytes = 0;
    for (int g = 0; g < S.ng; ++g) {
        const int nred = (int)S.dev.nonpivot[g].size();
        const int wg = std::max(1, (nred + 31) / 32);
        const int HP = wg >= 3 ? 4 : wg;
        const bool full = S.ranks[g] == S.K;
        std::vector<std::pair<int, int>> seen;
        for (int w = 1; w <= wmax; ++w) {
            if ((w + 1) - (S.K - S.ranks[g]) <= 0) continue;   // set inactive at this level
            // a level the engine cannot size: charge a footprint no budget admits beside
            // others (still far from overflowing a sum over requests)
            if (level_size_rc(S.K, w) != kOk) return (size_t)1 << 50;
            const unsigned long long pairs = dev->binom(S.K, w);
            int a, b;
            level_split(pairs, w, &a, &b);
            for (auto sz : {std::make_pair(a, 0), std::make_pair(b, 1)}) {
                if (std::find(seen.begin(), seen.end(), sz) != seen.end()) continue;
                seen.push_back(sz);
                const unsigned long long c = dev->binom(S.K, sz.first);
                bytes += (size_t)c * HP * 4 + (full ? 0 : (size_t)c) + 512;
                // +-1 rows of the tensor-core sweep (full-rank sets with two or more
                // probe words; counted whether or not the planner ends up using them)
                if (full && HP >= 2 && sz.first > 0)
                    bytes += (size_t)(c + kPmPadRows) * kPmRowBytes;
            }
        }
    }
    return bytes;
}

}  // namespace

struct QsfbServer {
    Device* dev = nullptr;
    size_t budget = 0;
    int max_active = 0;
    double t0 = 0;

    std::mutex mu;
    std::condition_variable cv_intake, cv_engine, cv_done;
    std::deque<Request*> submitted;      // waiting for intake
    std::deque<Request*> ready;          // reduced + uploaded, waiting for admission
    std::vector<Request*> active;        // enumerating
    std::unordered_map<long long, std::unique_ptr<Request>> all;
    long long next_id = 1;
    bool stopping = false;
    size_t in_use = 0, peak = 0;
    long long n_submitted = 0, n_completed = 0;
    double busy = 0.0;
    unsigned long long codewords = 0;
    int rounds = 0;
    int fatal = kOk;

    std::vector<std::thread> intake;
    std::thread engine;

    double now() const { return now_seconds() - t0; }

    void build_jobs(Request* r) {
        BzOptions opt;
        opt.parallel_seed = false;
        const OwnedQuery* q = &r->q;
        if (q->kind == 0) {
            r->jobs.emplace_back(new BzJob([q](Problem& p0, Problem&) {
                p0 = classical_problem(from_dense(q->A.data(), q->ar, q->ac));
                return 0;
            }, false, opt));
        } else if (q->kind == 1) {
            const bool single = q->which == 'Z' || q->which == 'X';
            r->jobs.emplace_back(new BzJob([q, single](Problem& p0, Problem& p1) {
                Mat A = from_dense(q->A.data(), q->ar, q->ac), B = from_dense(q->B.data(), q->br, q->bc);
                if (single) {
                    p0 = css_problem(A, B, q->which);
                } else {
                    auto pr = css_problem_pair(A, B);
                    p0 = std::move(pr.first);
                    p1 = std::move(pr.second);
                }
                return 0;
            }, !single, opt));
        } else {
            r->jobs.emplace_back(new BzJob([q](Problem& p0, Problem&) {
                Mat B = from_dense(q->B.data(), q->br, q->bc);
                if (in_rowspace(B, q->z.data())) return 1;
                p0 = coset_problem(B, q->z.data());
                return 0;
            }, false, opt));
            r->jobs.emplace_back(new BzJob([q](Problem& p0, Problem&) {
                Mat A = from_dense(q->A.data(), q->ar, q->ac);
                if (in_rowspace(A, q->x.data())) return 1;
                p0 = coset_problem(A, q->x.data());
                return 0;
            }, false, opt));
        }
    }

    void intake_loop() {
        SessionLease lease(dev);
        // staging reserved up front: growing pinned host memory later (cudaFreeHost +
        // cudaMallocHost) would synchronise the device under the engine's rounds
        if (lease.s) lease.s->ensure(1u << 20, 4u << 20);
        for (;;) {
            Request* r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_intake.wait(lk, [&] { return stopping || !submitted.empty(); });
                if (stopping) return;
                r = submitted.front();
                submitted.pop_front();
            }
            build_jobs(r);
            std::vector<BzJob*> ptrs;
            for (auto& j : r->jobs) ptrs.push_back(j.get());
            // 1 MiB chunks: a request's rows, seeds and lists are small, and its footprint
            // (which the admission budget counts) is the chunks it holds
            r->arena.reset(new Arena(dev, 1ull << 20));
            int rc = lease.s ? setup_jobs(dev, lease.s, r->arena.get(), ptrs, 1, nullptr) : kErrDevice;
            size_t fp = r->arena->bytes();
            for (BzJob* j : ptrs)
                for (int i = 0; i < (j->pair ? 2 : 1); ++i)
                    if (!j->zero) fp += list_footprint(dev, j->s[i]);
            std::lock_guard<std::mutex> lk(mu);
            r->footprint = fp;
            r->status = rc;
            r->t_ready = now();
            ready.push_back(r);
            cv_engine.notify_one();
        }
    }

    void finish(Request* r) {   // mu held
        r->t_done = now();
        r->done = true;
        ++n_completed;
        in_use -= std::min(in_use, r->footprint);
        cv_done.notify_all();
    }

    void fill_answer(Request* r) {
        QsfbAnswer& a = r->ans;
        std::memset(&a, 0, sizeof(a));
        if (r->q.kind == 2) {
            BzResult rz = r->jobs[0]->result(), rx = r->jobs[1]->result();
            a.z_weight = rz.distance;
            a.x_weight = rx.distance;
            a.distance = std::max(rz.distance, rx.distance);
            a.proven = (rz.proven && rx.proven) ? 1 : 0;
            a.levels = std::max(rz.levels, rx.levels);
            a.witness_ok = ((rz.witness_ok || rz.distance <= 0) && (rx.witness_ok || rx.distance <= 0)) ? 1 : 0;
        } else {
            BzResult b = r->jobs[0]->result();
            a.distance = b.distance;
            a.lower_bound = b.lower_bound;
            a.proven = b.proven ? 1 : 0;
            a.levels = b.levels;
            a.witness_ok = (b.witness_ok || b.distance < 0) ? 1 : 0;
            a.z_weight = a.x_weight = -1;
        }
    }

    void release(Request* r) {   // device memory back to the cache, host data dropped
        r->jobs.clear();
        r->arena.reset();
    }

    void engine_loop() {
        SessionLease lease(dev);
        if (lease.s) lease.s->ensure(32u << 20, 32u << 20);   // see intake_loop
        std::vector<LevelReq> q;
        std::vector<int> side, owner;
        std::vector<LevelOut> outs;
        for (;;) {
            std::vector<Request*> act;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_engine.wait(lk, [&] { return stopping || !ready.empty() || !active.empty(); });
                if (stopping && active.empty()) return;
                // admission at the round boundary: FIFO, slots and device-memory budget
                while (!ready.empty() && (int)active.size() < max_active) {
                    Request* r = ready.front();
                    if (r->status != kOk) {
                        ready.pop_front();
                        release(r);
                        finish(r);
                        continue;
                    }
                    if (!active.empty() && in_use + r->footprint > budget) break;
                    ready.pop_front();
                    r->t_admit = now();
                    in_use += r->footprint;
                    peak = std::max(peak, in_use);
                    active.push_back(r);
                }
                act = active;
            }
            // one round over every active request's next level
            q.clear(); side.clear(); owner.clear();
            std::vector<BzJob*> jobs;
            for (Request* r : act)
                for (auto& j : r->jobs)
                    if (!j->done()) jobs.push_back(j.get());
            for (size_t k = 0; k < jobs.size(); ++k) {
                const size_t before = q.size();
                jobs[k]->requests(q, side);
                for (size_t i = before; i < q.size(); ++i) owner.push_back((int)k);
            }
            RunStats rs;
            outs.clear();
            int rc = kOk;
            const double tr = now_seconds();
            if (!q.empty()) rc = run_levels(lease.s, q, outs, &rs);
            const double dt = now_seconds() - tr;
            size_t i = 0;
            for (size_t k = 0; k < jobs.size(); ++k) {
                std::vector<const LevelOut*> o;
                std::vector<int> sd;
                while (i < q.size() && owner[i] == (int)k) {
                    if (rc == kOk) { o.push_back(&outs[i]); sd.push_back(side[i]); }
                    ++i;
                }
                if (rc == kOk) jobs[k]->apply(o, sd);
            }
            std::lock_guard<std::mutex> lk(mu);
            busy += dt;
            codewords += rs.codewords;
            ++rounds;
            std::vector<Request*> still;
            for (Request* r : active) {
                bool fin = true;
                for (auto& j : r->jobs) fin = fin && j->done();
                if (rc != kOk) { r->status = rc; fin = true; fatal = rc; }
                if (fin) {
                    if (r->status == kOk) fill_answer(r);
                    release(r);
                    finish(r);
                } else {
                    still.push_back(r);
                }
            }
            active.swap(still);
        }
    }
};

extern "C" {

int qsfb_server_start(int intake_threads, long long mem_budget_bytes, int max_active,
                      QsfbServer** out) {
    if (!out) return kErrNull;
    *out = nullptr;
    int rc = kOk;
    Device* dev = Device::get(&rc);
    if (!dev) return kErrDevice;
    auto* S = new QsfbServer();
    S->dev = dev;
    S->budget = mem_budget_bytes > 0 ? (size_t)mem_budget_bytes : (size_t)64 << 30;
    // Mapped memory for the device allocator's first allocations of each size, so that a
    // heavy request's first large list does not map memory on the engine thread (measured:
    // one first 1 GiB-class allocation held a round, and the intake behind it, ~50 ms).
    // QSFB_SERVER_RESERVE_MB (default 8192, at most the budget; 0 = none).
    const char* re = std::getenv("QSFB_SERVER_RESERVE_MB");
    const size_t reserve = std::min(S->budget, (size_t)(re ? std::max(0, std::atoi(re)) : 8192)
                                                   << 20);
    dev->reserve(reserve);
    S->max_active = max_active > 0 ? max_active : 4096;
    S->t0 = now_seconds();
    // default: all cores but two (the engine thread and the caller's submitting thread
    // must not wait for a core behind the intake work)
    int nt = intake_threads > 0 ? intake_threads
                                : (int)std::thread::hardware_concurrency() - 2;
    nt = std::max(1, nt);
    for (int t = 0; t < nt; ++t) S->intake.emplace_back(&QsfbServer::intake_loop, S);
    S->engine = std::thread(&QsfbServer::engine_loop, S);
    *out = S;
    return kOk;
}

int qsfb_server_submit(QsfbServer* S, const QsfbQuery* q, long long* ticket) {
    if (!S || !q || !ticket || !q->A) return kErrNull;
    if (q->kind < 0 || q->kind > 2) return kErrShape;
    if (q->kind != 0 && !q->B) return kErrNull;
    if (q->kind == 2 && (!q->z_op || !q->x_op)) return kErrNull;
    std::unique_ptr<Request> r(new Request());
    OwnedQuery& o = r->q;
    o.kind = q->kind;
    o.which = q->which;
    o.ar = q->a_rows; o.ac = q->a_cols;
    o.A.assign(q->A, q->A + (size_t)q->a_rows * q->a_cols);
    if (q->kind != 0) {
        o.br = q->b_rows; o.bc = q->b_cols;
        o.B.assign(q->B, q->B + (size_t)q->b_rows * q->b_cols);
    }
    if (q->kind == 2) {
        o.z.assign(q->z_op, q->z_op + q->a_cols);
        o.x.assign(q->x_op, q->x_op + q->a_cols);
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return kErrDevice;
    r->id = S->next_id++;
    r->t_submit = S->now();
    *ticket = r->id;
    S->submitted.push_back(r.get());
    S->all[r->id] = std::move(r);
    ++S->n_submitted;
    S->cv_intake.notify_one();
    return kOk;
}

int qsfb_server_wait(QsfbServer* S, long long ticket, QsfbAnswer* out, QsfbTiming* t) {
    if (!S || !out) return kErrNull;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(ticket);
    if (it == S->all.end()) return kErrShape;
    Request* r = it->second.get();
    S->cv_done.wait(lk, [&] { return r->done; });
    *out = r->ans;
    if (t) {
        t->submit_s = r->t_submit;
        t->ready_s = r->t_ready;
        t->admit_s = r->t_admit;
        t->done_s = r->t_done;
        t->latency_s = r->t_done - r->t_submit;
    }
    const int st = r->status;
    S->all.erase(it);
    return st;
}

int qsfb_server_stats(QsfbServer* S, QsfbServeStats* out) {
    if (!S || !out) return kErrNull;
    std::lock_guard<std::mutex> lk(S->mu);
    out->submitted = S->n_submitted;
    out->completed = S->n_completed;
    out->active = (int)S->active.size();
    out->pending = (int)(S->submitted.size() + S->ready.size());
    out->busy_s = S->busy;
    out->codewords = S->codewords;
    out->rounds = S->rounds;
    out->peak_footprint_bytes = (long long)S->peak;
    out->elapsed_s = S->now();
    return kOk;
}

int qsfb_server_stop(QsfbServer* S) {
    if (!S) return kErrNull;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_intake.notify_all();
    S->cv_engine.notify_all();
    for (auto& t : S->intake) t.join();
    S->engine.join();
    // requests never admitted: drop their device data
    for (Request* r : S->ready) S->release(r);
    const int rc = S->fatal;
    delete S;
    return rc;
}

}  // extern "C"
