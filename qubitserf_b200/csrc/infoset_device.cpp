// Host half of the device information-set construction (kernel: infoset_kernels.cu).
//
// Pass 1 runs the greedy peel of every pending side (one warp each) and reads back the
// sets' generators, ranks and pivot masks.  The reference replaces the peel by an Edmonds
// matroid partition when that packs more full-rank sets (cpp/distfind/css.cpp:341-365);
// that decision and the partition's augmenting-path search are sequential and stay on the
// host (in parallel over the sides that need them), and pass 2 eliminates each chosen
// class on the device.  The packed rows (non-pivot columns) and the per-row detector
// syndromes are written by the kernel straight into the arena where the pair sweeps read
// them; nothing of them crosses to the host.  A side the kernel cannot hold (more than
// kInfosetMaxSets sets) is built on the host instead and uploaded with the others.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "bz.hpp"
#include "infoset_types.hpp"

namespace qsfb {

cudaError_t launch_infosets(int W, const InfosetDesc* d_descs, int ndesc,
                            unsigned long long* d_heap, unsigned long long* d_heap_ctr,
                            cudaStream_t st);

namespace {

size_t al256(size_t x) { return (x + 255) / 256 * 256; }

enum ItemState { kPending = 0, kDone = 1, kHost = 2, kClasses = 3 };

struct Item {
    BzSide* side = nullptr;
    const Problem* p = nullptr;
    int K = 0, n = 0, W = 0, kcheck = 0, W32 = 0, SWP = 0;
    uint32_t* red = nullptr;   // kInfosetMaxSets x K x W32 (arena)
    uint32_t* syn = nullptr;   // kInfosetMaxSets x K x SWP (arena)
    std::vector<std::vector<int>> lists;   // classes of the matroid partition (pass 2)
    std::vector<int> class_ranks;
    std::vector<InfoSet> sets;
    int state = kPending;
};

// One launch pass (greedy peel, or the explicit class lists) over `items`.
// tm[0..3] += seconds spent filling the staging, waiting for the kernels and the meta
// read-back, reading the generator heap back, and building the host descriptions
int run_pass(Session* s, Arena* arena, std::vector<Item*>& items, bool classes, double* tm) {
    if (items.empty()) return kOk;
    const double ta = now_seconds();
    std::stable_sort(items.begin(), items.end(),
                     [](const Item* a, const Item* b) { return a->W < b->W; });
    const size_t n = items.size();
    size_t off = 0;
    const size_t off_desc = off;
    off = al256(off + n * sizeof(InfosetDesc));
    const size_t off_meta = off;
    off += n * sizeof(InfosetMeta);
    const size_t off_ctr = off;
    off += 256;
    std::vector<size_t> og(n), oc(n), ol(n);
    unsigned long long cap = 0;   // heap words: every set's K x W generator
    for (size_t i = 0; i < n; ++i) {
        const Item& it = *items[i];
        og[i] = off; off = al256(off + (size_t)it.K * it.W * 8);
        oc[i] = off; off = al256(off + (size_t)std::max(1, it.kcheck) * it.W * 8);
        if (classes) {
            size_t len = 0;
            for (const auto& l : it.lists) len += l.size();
            ol[i] = off; off = al256(off + std::max<size_t>(len, 1));
        }
        const int nsets = classes ? (int)it.lists.size() : kInfosetMaxSets;
        cap += (unsigned long long)nsets * it.K * it.W;
    }
    const size_t staged = off;
    const size_t off_heap = off;
    off = al256(off + cap * 8);
    if (cap >= (1ull << 31)) return kErrUnsupported;   // heap offsets are 32-bit
    char* d = (char*)arena->alloc(off);
    if (!d) return kErrMemory;
    // pinned staging for what crosses before the kernels and the meta read-back only: the
    // heap comes back into pageable memory, so the staging does not grow with it (growing
    // pinned memory costs tens of ms and synchronises the device)
    int rc = s->ensure(0, staged);
    if (rc != kOk) return rc;
    char* h = (char*)s->h_stage.h;
    InfosetDesc* hd = (InfosetDesc*)(h + off_desc);
    std::memset(h + off_meta, 0, off_heap - off_meta);
    size_t nw1 = 0;
    for (size_t i = 0; i < n; ++i) nw1 += items[i]->W == 1;
    host_parallel_for(n, [&](size_t i) {
        const Item& it = *items[i];
        const Problem& p = *it.p;
        u64* g = (u64*)(h + og[i]);
        for (int r = 0; r < it.K; ++r) std::memcpy(g + (size_t)r * it.W, p.code_gen.row(r), it.W * 8);
        u64* c = (u64*)(h + oc[i]);
        for (int r = 0; r < it.kcheck; ++r) std::memcpy(c + (size_t)r * it.W, p.check.row(r), it.W * 8);
        InfosetDesc D;
        std::memset(&D, 0, sizeof(D));
        D.gen = (const unsigned long long*)(d + og[i]);
        D.check = (const unsigned long long*)(d + oc[i]);
        D.lists = nullptr;
        if (classes) {
            uint8_t* l = (uint8_t*)(h + ol[i]);
            size_t pos = 0;
            for (size_t k = 0; k < it.lists.size(); ++k) {
                for (int col : it.lists[k]) l[pos++] = (uint8_t)col;
                D.list_len[k] = (int)it.lists[k].size();
            }
            D.lists = (const uint8_t*)(d + ol[i]);
            D.nlists = (int)it.lists.size();
        }
        D.meta = (InfosetMeta*)(d + off_meta) + i;
        D.red = it.red;
        D.syn = it.syn;
        D.K = it.K;
        D.n = it.n;
        D.kcheck = it.kcheck;
        D.W32 = it.W32;
        D.SWP = it.SWP;
        hd[i] = D;
    });
    unsigned long long* d_heap = (unsigned long long*)(d + off_heap);
    unsigned long long* d_ctr = (unsigned long long*)(d + off_ctr);
    cudaStream_t st = s->urgent;   // the seed trials run beside it on `urgent2`
    const double tb = now_seconds();
    if (cudaMemcpyAsync(d, h, staged, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        launch_infosets(1, (const InfosetDesc*)(d + off_desc), (int)nw1, d_heap, d_ctr, st) !=
            cudaSuccess ||
        launch_infosets(2, (const InfosetDesc*)(d + off_desc) + nw1, (int)(n - nw1), d_heap, d_ctr,
                        st) != cudaSuccess ||
        cudaMemcpyAsync(h + off_meta, d + off_meta, off_ctr + 8 - off_meta, cudaMemcpyDeviceToHost,
                        st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return kErrDevice;
    }
    const double tc = now_seconds();
    const unsigned long long used = *(const unsigned long long*)(h + off_ctr);
    if (used > cap) return kErrDevice;
    thread_local std::vector<u64> heap_host;
    if (heap_host.size() < used) heap_host.resize(used);
    if (used > 0 && cudaMemcpy(heap_host.data(), d_heap, used * 8, cudaMemcpyDeviceToHost) !=
                        cudaSuccess) {
        cudaGetLastError();
        return kErrDevice;
    }
    const u64* heap = heap_host.data();
    const double td = now_seconds();
    host_parallel_for(n, [&](size_t i) {
        Item& it = *items[i];
        const InfosetMeta& M = *((const InfosetMeta*)(h + off_meta) + i);
        const int nsets = M.sets;
        if (nsets < 1 || nsets > kInfosetMaxSets || (classes && nsets != (int)it.lists.size())) {
            it.state = kHost;
            return;
        }
        it.sets.assign(nsets, InfoSet());
        bool ok = true;
        for (int g = 0; g < nsets && ok; ++g) {
            InfoSet& S = it.sets[g];
            S.g = Mat(it.K, it.n);
            const unsigned long long go = (unsigned long long)(unsigned)M.g_off[g];
            if (go + (unsigned long long)it.K * it.W > used) { ok = false; break; }
            std::memcpy(S.g.w.data(), heap + go, (size_t)it.K * it.W * 8);
            S.rank = M.rank[g];
            const unsigned long long pm[2] = {M.piv[g][0], M.piv[g][1]};
            auto is_piv = [&](int c) { return ((pm[c >> 6] >> (c & 63)) & 1u) != 0; };
            if (classes) {   // pivot i: the i-th column of the class (in list order) that took one
                for (int c : it.lists[g]) if (is_piv(c)) S.pivots.push_back(c);
                ok = S.rank == it.class_ranks[g];
            } else {         // greedy: active columns are eliminated in ascending order
                for (int c = 0; c < it.n; ++c) if (is_piv(c)) S.pivots.push_back(c);
            }
            ok = ok && (int)S.pivots.size() == S.rank;
        }
        it.state = ok ? kDone : kHost;
    });
    tm[0] += tb - ta;
    tm[1] += tc - tb;
    tm[2] += td - tc;
    tm[3] += now_seconds() - td;
    return kOk;
}

}  // namespace

int device_infosets(Session* s, Arena* arena, const std::vector<BzSide*>& sides,
                    RunStats* stats) {
    if (sides.empty()) return kOk;
    static const bool trace = std::getenv("QSFB_BATCH_TRACE") != nullptr;
    const double t0 = now_seconds();
    std::vector<Item> items(sides.size());
    size_t rows_bytes = 0;
    for (size_t i = 0; i < sides.size(); ++i) {
        Item& it = items[i];
        it.side = sides[i];
        it.p = sides[i]->prob;
        it.K = it.p->code_gen.rows;
        it.n = it.p->n;
        it.W = words_for(it.n);
        it.kcheck = it.p->count_all ? 0 : it.p->check.rows;
        it.W32 = (it.n + 31) / 32;
        it.SWP = std::max(1, (it.kcheck + 31) / 32);
        rows_bytes += al256((size_t)kInfosetMaxSets * it.K * it.W32 * 4) +
                      al256((size_t)kInfosetMaxSets * it.K * it.SWP * 4);
    }
    char* rows = (char*)arena->alloc(rows_bytes);
    if (!rows) return kErrMemory;
    size_t off = 0;
    for (Item& it : items) {
        it.red = (uint32_t*)(rows + off);
        off += al256((size_t)kInfosetMaxSets * it.K * it.W32 * 4);
        it.syn = (uint32_t*)(rows + off);
        off += al256((size_t)kInfosetMaxSets * it.K * it.SWP * 4);
    }
    std::vector<Item*> pass;
    for (Item& it : items) pass.push_back(&it);
    double tm[4] = {0, 0, 0, 0};
    int rc = run_pass(s, arena, pass, false, tm);
    if (rc != kOk) return rc;
    const double t1 = now_seconds();

    // the matroid-partition step, on the host, for the sides whose greedy peel may be beaten
    std::vector<Item*> cand;
    for (Item& it : items) {
        if (it.state != kDone || it.n > 200) continue;
        std::vector<u64> any(it.p->code_gen.stride, 0ull);
        for (int r = 0; r < it.K; ++r) vec_or(any.data(), it.p->code_gen.row(r), it.p->code_gen.stride);
        int nnz = 0;
        for (u64 x : any) nnz += popc64(x);
        if (full_sets(it.sets, it.K) < nnz / it.K) cand.push_back(&it);
    }
    auto decide = [](Item* it) {
        if (matroid_sets(it->p->code_gen, full_sets(it->sets, it->K), &it->lists, &it->class_ranks))
            it->state = (int)it->lists.size() <= kInfosetMaxSets ? kClasses : kHost;
    };
    host_parallel_for(cand.size(), [&](size_t k) { decide(cand[k]); });
    pass.clear();
    for (Item* it : cand)
        if (it->state == kClasses) pass.push_back(it);
    const double t2 = now_seconds();
    const size_t nclasses = pass.size();
    rc = run_pass(s, arena, pass, true, tm);
    if (rc != kOk) return rc;
    const double t3 = now_seconds();
    int nhost = 0;

    std::atomic<int> arc{kOk};
    host_parallel_for(items.size(), [&](size_t k) {   // host descriptions of the sets, per side
        Item& it = items[k];
        BzSide& S = *it.side;
        S.sets_from_classes = it.state == kDone && !it.lists.empty();
        const int r = it.state == kDone
                          ? S.adopt_sets(std::move(it.sets), it.red, it.syn, it.W32, it.SWP,
                                         s->dev, arena)
                          : S.adopt_sets(information_sets(it.p->code_gen), nullptr, nullptr, 0,
                                         0, s->dev, arena);
        if (r != kOk) arc.store(r);
    });
    for (const Item& it : items) nhost += it.state != kDone;
    rc = arc.load();
    if (rc != kOk) return rc;
    if (trace)
        std::fprintf(stderr, "qsfb device sets: %zu sides: greedy pass %.2f ms, partition "
                     "search %.2f ms (%zu candidates, %zu replaced), class pass %.2f ms, "
                     "adopt %.2f ms (%d built on the host); passes: staging %.2f, device %.2f, "
                     "heap read-back %.2f, host sets %.2f ms\n", items.size(), 1e3 * (t1 - t0),
                     1e3 * (t2 - t1), cand.size(), nclasses, 1e3 * (t3 - t2),
                     1e3 * (now_seconds() - t3), nhost, 1e3 * tm[0], 1e3 * tm[1], 1e3 * tm[2],
                     1e3 * tm[3]);
    if (stats) {
        stats->device_sets_s += now_seconds() - t0;
        stats->launches += 2;
    }
    return kOk;
}

}  // namespace qsfb
