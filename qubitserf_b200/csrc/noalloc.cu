// qsfb_enumerate_plan_noalloc: one BZ enumeration level for callers that cannot allocate
// device memory -- for instance a host process whose own memory pool owns the whole
// device, or code that must not trigger the device-wide synchronisation a cudaMalloc can
// cause.  The caller passes device buffers for the inputs and outputs; every byte of
// scratch the level needs (binomial table, descriptors, detector syndromes, subset lists,
// the witness key and counters) lives in one file-scope __device__ array of fixed size,
// so this entry point calls no cudaMalloc, cudaFree, cudaMallocHost or allocating library
// routine, and builds its host-side descriptors in fixed thread-local arrays.
//
// Limits (anything larger is rejected with rc 8 before touching the device):
//   K <= 128 rows, num_gamma <= 8 sets, kcheck <= 256 detector rows, stride <= 16 words,
//   and the subset lists of the level must fit in the 32 MiB scratch array.
// Every loaded copy of the library keeps that 32 MiB on every GPU it runs on until the
// process exits.  The array is shared by all calls and keeps the previous call's
// contents; each call rewrites everything it reads, and calls that overlap on the GPU
// (two host threads, or two streams) race on it -- callers must serialise them.
// The first call on a device looks up the array's device address (cudaGetSymbolAddress)
// and fills the binomial table; make that first call before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <mutex>

#include "../../include/qsf_b200.h"
#include "engine_types.hpp"
#include "filter_plan.hpp"

namespace qsfb {
cudaError_t launch_gen_lists(const GenDesc* d_descs, int ndesc, unsigned long long total,
                             const unsigned long long* d_binom, int num_sms, cudaStream_t st);
cudaError_t launch_pairs(int filt, int HP, int mode, const LevelDesc* d, int nd,
                         unsigned long long jobs, unsigned long long* ctr,
                         const unsigned long long* B, int num_sms, cudaStream_t st);
void level_split(unsigned long long pairs, int w, int* a, int* b);
}  // namespace qsfb

namespace {

using namespace qsfb;

constexpr size_t kScratchBytes = 32ull << 20;
constexpr int kMaxK = 128;
constexpr int kMaxSets = 8;
constexpr int kMaxCheck = 256;
constexpr int kMaxStride = 16;
constexpr int kLd = kBinomMaxK + 1;
constexpr int kErrScratch = 8;

// Region offsets inside the scratch array.
constexpr size_t kOffBinom = 0;                                   // (kMaxK+1) x kLd u64
constexpr size_t kBinomBytes = (size_t)(kMaxK + 1) * kLd * 8;
constexpr size_t kOffDesc = 128 << 10;                            // descriptors, tables, key
constexpr size_t kDescBytes = 64 << 10;
constexpr size_t kOffSyn = kOffDesc + kDescBytes;                 // detector syndromes
constexpr size_t kSynBytes = (size_t)kMaxSets * kMaxK * (kMaxCheck / 32) * 4;
constexpr size_t kOffLists = kOffSyn + ((kSynBytes + 255) / 256) * 256;

static_assert(kBinomBytes <= kOffDesc, "binomial region");

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Per-device address of g_scratch (looked up once per device).
struct DevSlot {
    unsigned char* ptr = nullptr;
    int sms = 0;
};
std::mutex g_mu;
DevSlot g_slots[64];

// Host staging of one call's descriptors (no heap allocation).
struct Staging {
    GenDesc gen[2 * kMaxSets];
    LevelDesc lvl[kMaxSets];
    unsigned long long terms[kMaxSets][kMaxK + 2];
    unsigned long long key;
    unsigned long long counts[kMaxSets];
    unsigned long long ctr[8];
};
static_assert(sizeof(Staging) <= kDescBytes, "descriptor region");
thread_local Staging t_stage;

// syn[g][r] = (parity(check_c & row_r(g)))_c, SW words per row.
__global__ void syndromes_kernel(const uint64_t* __restrict__ gamma, int ng, int K, int stride,
                                 const uint64_t* __restrict__ check, int kcheck, int SW,
                                 uint32_t* __restrict__ syn) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ng * K) return;
    const uint64_t* row = gamma + (size_t)t * stride;
    uint32_t* o = syn + (size_t)t * SW;
    for (int h = 0; h < SW; ++h) o[h] = 0u;
    for (int c = 0; c < kcheck; ++c) {
        uint64_t acc = 0;
        for (int w = 0; w < stride; ++w) acc ^= row[w] & check[(size_t)c * stride + w];
        if (__popcll(acc) & 1) o[c >> 5] |= 1u << (c & 31);
    }
}

// Key + counters -> the caller's outputs.
__global__ void finalize_kernel(const unsigned long long* __restrict__ key, unsigned long long key0,
                                const unsigned long long* __restrict__ counts, int ng,
                                int current_best, int* out_best, unsigned long long* out_counts,
                                int* out_g, unsigned long long* out_rank) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const unsigned long long k = *key;
    const bool found = k < key0;
    const int wt = (int)(k >> kKeyWtShift) - 1;
    *out_best = found ? (wt < current_best ? wt : current_best) : current_best;
    if (out_g) *out_g = found ? (int)((k >> kKeyGShift) & 0xff) : -1;
    if (out_rank) *out_rank = found ? (k & kKeyRankMask) : ~0ull;
    if (out_counts)
        for (int g = 0; g < ng; ++g) out_counts[g] = counts[g];
}

struct BinomTable {
    unsigned long long v[(kMaxK + 1) * kLd];
    BinomTable() {
        std::memset(v, 0, sizeof(v));
        for (int a = 0; a <= kMaxK; ++a) {
            v[(size_t)a * kLd] = 1ull;
            for (int b = 1; b <= std::min(a, kBinomMaxK); ++b) {
                const unsigned long long x = v[(size_t)(a - 1) * kLd + b - 1];
                const unsigned long long y = b <= a - 1 ? v[(size_t)(a - 1) * kLd + b] : 0ull;
                v[(size_t)a * kLd + b] = (x > ~0ull - y) ? ~0ull : x + y;
            }
        }
    }
};
const BinomTable& binom_table() {
    static const BinomTable t;   // built once, thread-safe static initialisation
    return t;
}
unsigned long long host_binom(int n, int k) {
    if (k < 0 || n < 0 || k > n) return 0ull;
    if (n > kMaxK || k > kBinomMaxK) return ~0ull;
    return binom_table().v[(size_t)n * kLd + k];
}

// Set-up once per device (device current): look up the scratch address, fill the table.
// The table goes up on the caller's stream, followed by a wait on that stream only, so the
// set-up does not synchronise the whole device.  The address is cached for the life of the
// loaded library: after a cudaDeviceReset the library must be reloaded.
int device_slot(cudaStream_t st, DevSlot** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 4;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    DevSlot& s = g_slots[dev];
    if (!s.ptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return 4;
        }
        const BinomTable& table = binom_table();   // static storage: outlives the async copy
        if (cudaMemcpyAsync((unsigned char*)p + kOffBinom, table.v, sizeof(table.v),
                            cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess ||
            cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            return 4;
        }
        s.ptr = (unsigned char*)p;
    }
    *out = &s;
    return 0;
}

}  // namespace

extern "C" int qsfb_enumerate_plan_noalloc(int n, int stride, int K, int d, int num_gamma,
                                           const uint64_t* d_gamma, int kcheck,
                                           const uint64_t* d_check, int current_best,
                                           int* d_out_best, unsigned long long* d_out_counts,
                                           int* d_out_g, unsigned long long* d_out_rank,
                                           void* stream) {
    if (!d_gamma || !d_out_best || (kcheck > 0 && !d_check)) return 1;
    if (stride != (n + 63) / 64 || K < 1 || d < 1 || d > K || num_gamma < 1) return 2;
    if (K > kMaxK || num_gamma > kMaxSets || kcheck > kMaxCheck || stride > kMaxStride ||
        d > kBinomMaxK)
        return kErrScratch;
    cudaStream_t st = (cudaStream_t)stream;

    // ---- plan (the rules of the allocating path: prefix/suffix split, probe filter)
    // Every size below is bounded before it is multiplied: a saturated binomial (C >= 2^64
    // reads as ~0ull) or a list count beyond the scratch array is rejected first, so no
    // product or sum can wrap.
    const unsigned long long pairs = host_binom(K, d);
    if (pairs == ~0ull || pairs >= (1ull << 62)) return kErrScratch;
    int a, b;
    level_split(pairs, d, &a, &b);
    const int W32 = 2 * stride;              // a u64 row is 2*stride little-endian u32 words
    const int HP = W32 >= 3 ? 4 : W32;
    const int bound = current_best >= kWeightNone ? 4094 : current_best - 1;
    const int T = std::max(0, std::min(bound + 1, 4095));
    const int filt = choose_filter(HP, 32 * W32, T - 1, false).filt;
    const int SW = (kcheck + 31) / 32;
    const unsigned long long na = host_binom(K, a), nb = host_binom(K, b);
    constexpr size_t kListRoom = kScratchBytes - kOffLists;
    const unsigned long long entry_bytes = (unsigned long long)HP * 4 + 1;   // probe words + pivot count
    if (na > kListRoom / entry_bytes || nb > kListRoom / entry_bytes) return kErrScratch;
    const size_t list_a = (size_t)na * HP * 4, list_b = (size_t)nb * HP * 4;
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t per_set = up(list_a) + up(na) + up(list_b) + up(nb);   // < 4 x (32 MiB + 256)
    if (per_set > kListRoom / (size_t)num_gamma) return kErrScratch;

    DevSlot* slot = nullptr;
    if (device_slot(st, &slot) != 0) return 4;
    unsigned char* base = slot->ptr;

    // ---- descriptors (host, fixed arrays) -> one copy into the scratch descriptor region
    Staging& S = t_stage;
    std::memset(&S, 0, sizeof(S));
    unsigned char* dd = base + kOffDesc;
    const size_t off_gen = offsetof(Staging, gen), off_lvl = offsetof(Staging, lvl);
    const size_t off_terms = offsetof(Staging, terms), off_key = offsetof(Staging, key);
    const size_t off_counts = offsetof(Staging, counts), off_ctr = offsetof(Staging, ctr);
    const unsigned long long* d_binom = (const unsigned long long*)(base + kOffBinom);
    uint32_t* d_syn = (uint32_t*)(base + kOffSyn);

    const unsigned long long want_jobs = (unsigned long long)slot->sms * 16 * 4;
    unsigned long long lt = (pairs * num_gamma) / ((unsigned long long)kRegTile * want_jobs);
    lt = std::max<unsigned long long>(32, std::min<unsigned long long>(1024, lt));
    const int loop_tile = (int)((lt + 31) / 32 * 32);

    unsigned long long gen_total = 0, job_total = 0;
    int ngen = 0;
    const int p_lo = a - 1, nterms = K - b - a + 1;
    for (int g = 0; g < num_gamma; ++g) {
        unsigned char* lb = base + kOffLists + per_set * g;
        uint32_t* la = (uint32_t*)lb;
        uint8_t* pca = (uint8_t*)(lb + up(list_a));
        uint32_t* rb = (uint32_t*)(lb + up(list_a) + up(na));
        uint8_t* pcb = (uint8_t*)(lb + up(list_a) + up(na) + up(list_b));
        const uint32_t* red = (const uint32_t*)(d_gamma + (size_t)g * K * stride);
        for (int side = 0; side < 2; ++side) {
            GenDesc& G = S.gen[ngen++];
            G.red = red;
            G.out = side == 0 ? la : rb;
            G.pc = side == 0 ? pca : pcb;
            G.entry_base = gen_total;   // in runs of kGenRun entries
            G.count = side == 0 ? na : nb;
            G.K = K;
            G.size = side == 0 ? a : b;
            G.W32 = W32;
            G.HP = HP;
            G.rank = 0;          // raw rows: no pivot structure
            G.reflect = side;
            gen_total += (G.count + kGenRun - 1) / kGenRun;
        }
        unsigned long long acc = 0;
        for (int t = 0; t < nterms; ++t) {
            const int p = p_lo + t;
            const unsigned long long nx = host_binom(p, a - 1), ny = host_binom(K - 1 - p, b);
            const unsigned long long rn = std::max(nx, ny), ln = std::min(nx, ny);
            S.terms[g][t] = acc;
            acc += ((rn + kRegTile - 1) / kRegTile) * ((ln + loop_tile - 1) / loop_tile);
        }
        S.terms[g][nterms] = acc;
        LevelDesc& D = S.lvl[g];
        D.red = red;
        D.syn = d_syn + (size_t)g * K * std::max(SW, 1);
        D.la = la; D.pca = pca; D.rb = rb; D.pcb = pcb;
        D.term_jobs = (const uint64_t*)(dd + off_terms + (size_t)g * (kMaxK + 2) * 8);
        D.key = (unsigned long long*)(dd + off_key);
        D.count = (unsigned long long*)(dd + off_counts) + g;
        D.job_base = job_total;
        D.K = K; D.w = d; D.a = a; D.b = b;
        D.W32 = W32; D.SW = SW; D.HP = HP;
        D.rank = 0;
        D.g = g;
        D.p_lo = p_lo;
        D.nterms = nterms;
        D.loop_tile = loop_tile;
        int bits = 0;
        while (bits < 64 && (pairs - 1) >> bits) ++bits;
        D.rank_shift = std::max(0, bits - kKeyGShift);
        D.count_all = kcheck == 0 ? 1 : 0;
        job_total += acc;
    }
    const unsigned long long key0 = ((unsigned long long)T << kKeyWtShift) | ((1ull << kKeyWtShift) - 1);
    S.key = key0;     // counters and counts start at zero (memset above)

    if (cudaMemcpyAsync(dd, &S, sizeof(S), cudaMemcpyHostToDevice, st) != cudaSuccess) {
        cudaGetLastError();
        return 4;
    }
    if (kcheck > 0) {
        const int threads = 128, rows = num_gamma * K;
        syndromes_kernel<<<(rows + threads - 1) / threads, threads, 0, st>>>(
            d_gamma, num_gamma, K, stride, d_check, kcheck, SW, d_syn);
    }
    if (cudaGetLastError() != cudaSuccess ||
        launch_gen_lists((const GenDesc*)(dd + off_gen), ngen, gen_total, d_binom, slot->sms, st) != cudaSuccess ||
        launch_pairs(filt, HP, 0, (const LevelDesc*)(dd + off_lvl), num_gamma, job_total,
                     (unsigned long long*)(dd + off_ctr), d_binom, slot->sms, st) != cudaSuccess) {
        cudaGetLastError();
        return 4;
    }
    finalize_kernel<<<1, 32, 0, st>>>((const unsigned long long*)(dd + off_key), key0,
                                      (const unsigned long long*)(dd + off_counts), num_gamma,
                                      current_best, d_out_best, d_out_counts, d_out_g, d_out_rank);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return 4;
    }
    return 0;
}
