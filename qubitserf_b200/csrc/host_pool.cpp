// Process-wide pool of host threads for the per-code host steps of a preparation (staging
// fills, information-set descriptions, the matroid-partition search): those run once per
// chunk of a batch, a few times per call, and starting fresh threads each time costs tens
// of microseconds per thread on the critical path before the rounds.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.hpp"

namespace qsfb {

namespace {

class HostPool {
public:
    explicit HostPool(int workers) {
        for (int i = 0; i < workers; ++i) th_.emplace_back([this]() { loop(); });
    }
    int workers() const { return (int)th_.size(); }

    // f(0..n-1) on the caller and up to `helpers` workers; false (nothing run) when the pool
    // is serving another caller
    bool run(size_t n, const std::function<void(size_t)>& f, int helpers) {
        std::unique_lock<std::mutex> busy(run_mu_, std::try_to_lock);
        if (!busy.owns_lock()) return false;
        {
            std::lock_guard<std::mutex> lk(mu_);
            f_ = &f;
            n_ = n;
            next_.store(0);
            slots_ = std::max(0, std::min(helpers, workers()));
            open_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (size_t k; (k = next_.fetch_add(1)) < n;) f(k);
        std::unique_lock<std::mutex> lk(mu_);
        open_ = false;   // workers that wake from here on skip this job
        done_.wait(lk, [&]() { return active_ == 0; });
        f_ = nullptr;
        return true;
    }

private:
    void loop() {
        unsigned long long seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&]() { return gen_ != seen; });
            seen = gen_;
            if (!open_ || slots_ == 0) continue;
            --slots_;
            ++active_;
            const std::function<void(size_t)>* f = f_;
            const size_t n = n_;
            lk.unlock();
            for (size_t k; (k = next_.fetch_add(1)) < n;) (*f)(k);
            lk.lock();
            if (--active_ == 0) done_.notify_all();
        }
    }

    std::vector<std::thread> th_;
    std::mutex run_mu_;   // one job at a time
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(size_t)>* f_ = nullptr;
    size_t n_ = 0;
    std::atomic<size_t> next_{0};
    unsigned long long gen_ = 0;
    int slots_ = 0, active_ = 0;
    bool open_ = false;
};

HostPool& pool() {
    // started on first use and never destroyed (its threads park on a condition variable;
    // joining them during static destruction would race the process's other teardown)
    static HostPool* p =
        new HostPool(std::min((int)std::max(1u, std::thread::hardware_concurrency()), 16) - 1);
    return *p;
}

}  // namespace

void host_parallel_for(size_t n, const std::function<void(size_t)>& f, int max_threads) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int want = (int)std::min<size_t>({n, (size_t)std::max(1, max_threads), (size_t)hw});
    if (want <= 1) {
        for (size_t k = 0; k < n; ++k) f(k);
        return;
    }
    if (pool().run(n, f, want - 1)) return;
    // the pool is busy with another caller's job: threads of this call's own
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    for (int t = 1; t < want; ++t)
        th.emplace_back([&]() {
            for (size_t k; (k = next.fetch_add(1)) < n;) f(k);
        });
    for (size_t k; (k = next.fetch_add(1)) < n;) f(k);
    for (std::thread& t : th) t.join();
}

}  // namespace qsfb
