// Tensor-core pair sweep (sm_100a tcgen05) for full-rank information sets.
//
// For a full-rank set every pair (P, Q) of a level weighs w + popc(red(P) ^ red(Q)); the
// CUDA-core sweep bounds the popcount from below with a few POPCs per pair.  Here the
// bound is an exact Hamming distance over the first 64 non-pivot columns, taken as an
// integer matrix product: with bits written as +-1 int8 values,
//     <x, y> = n_live - 2 * hamming(x, y)
// over the n_live live columns (dead columns are 0 on both sides), so a 128 x 128 block
// of pairs is two `tcgen05.mma.kind::i8` steps (K = 32 each) into a 32-bit TMEM
// accumulator.  A pair can beat the bound T only if
//     hamming <= T - 1 - w   <=>   <x, y> >= n_live - 2 (T - 1 - w),
// so the read-back takes a running maximum over each 64-column slice of the accumulator
// and hands the rare slices that reach the threshold to the exact survivor evaluation
// shared with the CUDA-core sweep (same key, same tie-breaking, same counts).
//
// Every suffix row fetched into shared memory serves 256 prefix rows, which keeps the
// operand traffic far below L2 and DRAM bandwidth: a job holds a 256-row prefix tile (two
// M = 128 halves, 16 KB) and streams 128-row suffix tiles (8 KB) through an 8-deep ring;
// each suffix tile feeds two accumulators, one per half.  Rows are 64 bytes, pre-swizzled
// in global memory (16-byte chunk c of row e at c ^ ((e >> 1) & 3)), so a plain bulk copy
// of 8-row-aligned rows lands in the 64-byte-swizzled K-major operand layout.
//
// CTA = 20 warps: warps 0 and 18 issue the bulk copies, warp 1 owns the TMEM allocation
// (four 128-column accumulators = all 512 columns: two halves x double buffer), warps 1
// and 19 issue the MMAs (one thread each, by suffix-tile parity), warps 2-17 read back in
// two groups of eight, one per accumulator buffer (even / odd suffix tiles), each with one
// warp per TMEM lane quarter and half and one packed `tcgen05.ld` of 128 columns per tile.
// The sweep is bound by TMEM capacity over the accumulator round trip: the 512 columns hold
// 64k accumulators, and each goes MMA -> commit -> read-back -> release (~1,400 cycles)
// before its columns take the next tile, about 47 pairs per clock per SM against the
// ~120 that the dense int8 peak allows at 64 MACs a pair.
//
// Every wait is bounded (about two seconds of %globaltimer); a wait that runs out sets the
// launch's error word (1 copy warp, 2 MMA warp, 3 read-back warps: the first role that
// gave up) and the CTA winds down without touching the device further.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdlib>

#include "engine_types.hpp"
#include "enum_device.cuh"
#include "tuning.hpp"

namespace qsfb {
namespace dev {

constexpr int kTcM = 128;                  // rows per MMA (UMMA M)
constexpr int kTcHalves = 2;               // MMA row blocks per prefix tile
constexpr int kTcRows = kTcM * kTcHalves;  // prefix rows per tile
constexpr int kTcN = 128;                  // suffix rows per tile (UMMA N)
constexpr int kTcK = 2;                    // K = 32 steps (64 columns)
constexpr int kTcBStages = 8;              // suffix tiles in flight
constexpr int kTcSlice = 64;               // accumulator columns per rescan slice
constexpr int kTcEpiGroups = 2;            // read-back groups: one per accumulator buffer
constexpr int kTcEpiWarps = 8 * kTcEpiGroups;   // x 2 halves x 4 lane quarters
constexpr int kTcThreads = 32 * (4 + kTcEpiWarps);   // + two copy and two MMA warps
constexpr uint32_t kTcHalfBytes = kTcM * kPmRowBytes;      // 8 KB
constexpr uint32_t kTcABytes = kTcRows * kPmRowBytes;      // 16 KB
constexpr uint32_t kTcBBytes = kTcN * kPmRowBytes;         // 8 KB
constexpr uint32_t kTcOffA = 0;                            // two prefix tiles
constexpr uint32_t kTcOffB = 2 * kTcABytes;                // kTcBStages suffix tiles
constexpr uint32_t kTcOffBar = kTcOffB + kTcBStages * kTcBBytes;
constexpr uint32_t kTcSmem = kTcOffBar + 512 + 1024;       // + barriers, TMEM slot, alignment
constexpr uint32_t kTcTmemCols = 2 * kTcHalves * kTcN;     // 512: buffers x halves x N
constexpr unsigned long long kTcWaitNs = 2000000000ull;
static_assert(kTcTmemCols <= 512, "TMEM holds 512 columns");
static_assert(kPmRowBytes == 64, "operand rows are 64 bytes (64 int8 columns)");

// instruction descriptor: D s32 (bits 4-5 = 2), A and B signed int8 (bits 7-9, 10-12 = 1),
// both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t kTcIdesc = (2u << 4) | (1u << 7) | (1u << 10) |
                              ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);

// A sweep shape: ROWS prefix rows per job (ROWS / 128 MMA row blocks) against suffix tiles of
// N rows, the MMA's N.  Both shapes fill the same two 256-column accumulator buffers, and
// each buffer is read back by eight warps (two per TMEM lane quarter: the two prefix halves
// of a 256 x 128 tile, or the two 128-column halves of a 128 x 256 one).  The wide shape
// issues half as many MMAs for the same pairs: each tcgen05.mma occupies its issuing thread
// ~80-130 cycles, four of them plus the commit were a third of a buffer's round trip.
template <int ROWS, int N>
struct TcShape {
    static constexpr int kRows = ROWS, kN = N;
    static constexpr int kHalves = ROWS / kTcM;           // MMA row blocks per prefix tile
    static constexpr int kChunks = N / 128;               // 128-column read-back chunks per half
    static constexpr uint32_t kABytes = ROWS * kPmRowBytes;
    static constexpr uint32_t kBBytes = N * kPmRowBytes;
    static constexpr uint32_t kOffB = 2 * kABytes;        // after the two prefix slots
    static constexpr uint32_t kOffBar = kOffB + kTcBStages * kBBytes;
    static constexpr uint32_t kSmem = kOffBar + 512 + 1024;   // + barriers, TMEM slot, alignment
    static constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) |
                                       ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
    static_assert(kHalves * N == 256, "a buffer is 256 accumulator columns");
    static_assert(kHalves * kChunks == 2, "two read-back warps per lane quarter and buffer");
    static_assert(kSmem <= 227 * 1024, "shared memory");
};
using TcHalvesShape = TcShape<256, 128>;
using TcWideShape = TcShape<128, 256>;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

// Non-suspending probe of a barrier phase: the pollers here are single threads on the
// critical path, so they spin instead of sleeping through the phase change.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of `bar` with the given parity; false after `limit_ns` (error path,
// ~2 s by default).  The timer is only consulted after a few thousand probes: normal
// waits are far shorter, and a %globaltimer read on every wait would sit on the critical
// path.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          unsigned long long limit_ns = kTcWaitNs) {
    for (int i = 0; i < 4096; ++i)
        if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 1024; ++i)
            if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared, completion counted on `bar` (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

// K-major operand, 64-byte swizzle: rows of 64 B, 8-row groups 512 B apart (SBO),
// LBO unused (1), descriptor version 1, layout type 4.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate, uint32_t idesc = kTcIdesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 64 consecutive 32-bit accumulator columns of this thread's TMEM lane; the wait for the
// load sits in the same statement, so no use of v can be scheduled before it.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, int32_t (&v)[64]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {"
        "%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]),
          "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]),
          "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]),
          "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]),
          "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]),
          "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
        : "r"(taddr)
        : "memory");
}

// 128 consecutive 32-bit accumulator columns of this thread's TMEM lane (load and wait in
// one statement, as above).
__device__ __forceinline__ void tmem_ld128(uint32_t taddr, int32_t (&v)[128]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x128.b32 {"
        "%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63,"
        "%64,%65,%66,%67,%68,%69,%70,%71,%72,%73,%74,%75,%76,%77,%78,%79,"
        "%80,%81,%82,%83,%84,%85,%86,%87,%88,%89,%90,%91,%92,%93,%94,%95,"
        "%96,%97,%98,%99,%100,%101,%102,%103,%104,%105,%106,%107,%108,%109,%110,%111,"
        "%112,%113,%114,%115,%116,%117,%118,%119,%120,%121,%122,%123,%124,%125,%126,%127}, [%128];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]),
          "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]),
          "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]),
          "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]),
          "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]),
          "=r"(v[61]), "=r"(v[62]), "=r"(v[63]), "=r"(v[64]), "=r"(v[65]), "=r"(v[66]),
          "=r"(v[67]), "=r"(v[68]), "=r"(v[69]), "=r"(v[70]), "=r"(v[71]), "=r"(v[72]),
          "=r"(v[73]), "=r"(v[74]), "=r"(v[75]), "=r"(v[76]), "=r"(v[77]), "=r"(v[78]),
          "=r"(v[79]), "=r"(v[80]), "=r"(v[81]), "=r"(v[82]), "=r"(v[83]), "=r"(v[84]),
          "=r"(v[85]), "=r"(v[86]), "=r"(v[87]), "=r"(v[88]), "=r"(v[89]), "=r"(v[90]),
          "=r"(v[91]), "=r"(v[92]), "=r"(v[93]), "=r"(v[94]), "=r"(v[95]), "=r"(v[96]),
          "=r"(v[97]), "=r"(v[98]), "=r"(v[99]), "=r"(v[100]), "=r"(v[101]), "=r"(v[102]),
          "=r"(v[103]), "=r"(v[104]), "=r"(v[105]), "=r"(v[106]), "=r"(v[107]), "=r"(v[108]),
          "=r"(v[109]), "=r"(v[110]), "=r"(v[111]), "=r"(v[112]), "=r"(v[113]), "=r"(v[114]),
          "=r"(v[115]), "=r"(v[116]), "=r"(v[117]), "=r"(v[118]), "=r"(v[119]), "=r"(v[120]),
          "=r"(v[121]), "=r"(v[122]), "=r"(v[123]), "=r"(v[124]), "=r"(v[125]), "=r"(v[126]),
          "=r"(v[127])
        : "r"(taddr)
        : "memory");
}

// 128 consecutive accumulator columns of this thread's TMEM lane, read as 16-bit values:
// register i holds the low halves of columns 2i and 2i + 1 (the accumulators here are
// integers in [-64, 64], exact in 16 bits).  Load and wait in one statement.
__device__ __forceinline__ void tmem_ld128_p16(uint32_t taddr, uint32_t (&v)[64]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.pack::16b.b32 {"
        "%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]),
          "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]),
          "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]),
          "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]),
          "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]),
          "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
        : "r"(taddr)
        : "memory");
}

// An empty statement that reads and writes all 64 loaded registers: arithmetic on them
// cannot be scheduled before it, so a buffer's release (issued just before) is not delayed
// by the slice maxima that only need the registers.
__device__ __forceinline__ void after_release(uint32_t (&v)[64]) {
    asm volatile("" : "+r"(v[0]),"+r"(v[1]),"+r"(v[2]),"+r"(v[3]),"+r"(v[4]),"+r"(v[5]),"+r"(v[6]),"+r"(v[7]),"+r"(v[8]),"+r"(v[9]),"+r"(v[10]),"+r"(v[11]),"+r"(v[12]),"+r"(v[13]),"+r"(v[14]),"+r"(v[15]),"+r"(v[16]),"+r"(v[17]),"+r"(v[18]),"+r"(v[19]),"+r"(v[20]),"+r"(v[21]),"+r"(v[22]),"+r"(v[23]),"+r"(v[24]),"+r"(v[25]),"+r"(v[26]),"+r"(v[27]),"+r"(v[28]),"+r"(v[29]),"+r"(v[30]),"+r"(v[31]),"+r"(v[32]),"+r"(v[33]),"+r"(v[34]),"+r"(v[35]),"+r"(v[36]),"+r"(v[37]),"+r"(v[38]),"+r"(v[39]),"+r"(v[40]),"+r"(v[41]),"+r"(v[42]),"+r"(v[43]),"+r"(v[44]),"+r"(v[45]),"+r"(v[46]),"+r"(v[47]),"+r"(v[48]),"+r"(v[49]),"+r"(v[50]),"+r"(v[51]),"+r"(v[52]),"+r"(v[53]),"+r"(v[54]),"+r"(v[55]),"+r"(v[56]),"+r"(v[57]),"+r"(v[58]),"+r"(v[59]),"+r"(v[60]),"+r"(v[61]),"+r"(v[62]),"+r"(v[63]));
}

// Shared setup of both tensor-core kernels: barriers by thread 0, TMEM by warp 1.
__device__ __forceinline__ uint32_t tc_setup(uint32_t bar0, int nbar, const uint32_t* counts,
                                             uint32_t* tmem_slot) {
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        for (int i = 0; i < nbar; ++i) mbar_init(bar0 + 8u * i, counts[i]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *reinterpret_cast<volatile uint32_t*>(tmem_slot);
}

__device__ __forceinline__ void tc_teardown(uint32_t tmem) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTcTmemCols));
}

// One job: prefix tile rows [r0, r0 + 256) (from the 8-aligned start of the term's block)
// against suffix tiles [b0, b1) of the term's prefix of the suffix list.  A small kernel
// decodes every job of the launch into one 64-byte record (binary searches over the
// descriptors and terms, one thread per job) that carries everything the steady state
// needs: the two operand lists, the witness key, the bound as it stood at decode time and
// the threshold constants.  The sweep's roles read their next record one job ahead, so a
// job costs them no dependent global loads.  Row and entry indices fit 32 bits: a +-1 list
// of 2^32 rows would need 256 GB.
struct TcJobRec {
    const int8_t* xpm;
    const int8_t* ypm;
    unsigned long long* key;
    unsigned int r0, xoff, nx, ny;
    unsigned int d, b0, b1;
    // bound field (bits 0-11) | n_live << 12 | w << 20; for a rank-deficient set the w field
    // holds the fewest pivot rows a suffix entry can have, and bit 31 says that each prefix
    // row adds its own pivot-row count
    unsigned int tnw;
    unsigned long long pad;
};
static_assert(sizeof(TcJobRec) == 64, "job record layout");

template <class SH>
__global__ void __launch_bounds__(256) tc_jobs_kernel(const LevelDesc* __restrict__ descs,
                                                      int ndesc, unsigned long long total,
                                                      const unsigned long long* __restrict__ B,
                                                      TcJobRec* __restrict__ recs) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long job = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         job < total; job += stride) {
        int lo = 0, hi = ndesc - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (descs[mid].job_base <= job) lo = mid; else hi = mid - 1;
        }
        const LevelDesc& D = descs[lo];
        const unsigned long long local = job - D.job_base;
        int tl = 0, th = D.nterms - 1;
        while (tl < th) {
            const int mid = (tl + th + 1) >> 1;
            if (__ldg(D.term_jobs + mid) <= local) tl = mid; else th = mid - 1;
        }
        const unsigned long long idx = local - __ldg(D.term_jobs + tl);
        const int p = D.p_lo + tl;
        const unsigned long long nx = binom(B, p, D.a - 1);
        const unsigned long long ny = binom(B, D.K - 1 - p, D.b);
        const unsigned long long xoff = binom(B, p, D.a);
        const unsigned long long nbt = (ny + SH::kN - 1) / SH::kN;
        const unsigned long long jb = (unsigned long long)D.tc_job_tiles;
        const unsigned long long nbc = (nbt + jb - 1) / jb;
        const unsigned long long ia = idx / nbc, jc = idx - ia * nbc;
        TcJobRec R;
        R.xpm = D.xpm;
        R.ypm = D.ypm;
        R.key = D.key;
        R.r0 = (unsigned int)((xoff & ~7ull) + ia * SH::kRows);
        R.xoff = (unsigned int)xoff;
        R.nx = (unsigned int)nx;
        R.ny = (unsigned int)ny;
        R.d = (unsigned int)lo;
        R.b0 = (unsigned int)(jc * jb);
        R.b1 = (unsigned int)(jc * jb + jb < nbt ? jc * jb + jb : nbt);
        const unsigned int T0 = (unsigned int)(*((volatile unsigned long long*)D.key) >> kKeyWtShift);
        // rank-deficient set: a suffix entry holds at least b - (K - rank) pivot rows
        const unsigned int wf =
            D.pca ? ((unsigned int)max(0, D.b - (D.K - D.rank)) | 0x800u) : (unsigned int)D.w;
        R.tnw = (T0 & 0xFFFu) | ((unsigned int)D.n_live << 12) | (wf << 20);
        R.pad = 0;
        recs[job] = R;
    }
}

__device__ __forceinline__ TcJobRec tc_rec(const TcJobRec* __restrict__ recs,
                                           unsigned long long job, unsigned long long total) {
    TcJobRec R;
    if (job < total) {
        const uint4* q = reinterpret_cast<const uint4*>(recs + job);
        const uint4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
        R.xpm = (const int8_t*)((unsigned long long)a.x | ((unsigned long long)a.y << 32));
        R.ypm = (const int8_t*)((unsigned long long)a.z | ((unsigned long long)a.w << 32));
        R.key = (unsigned long long*)((unsigned long long)b.x | ((unsigned long long)b.y << 32));
        R.r0 = b.z; R.xoff = b.w;
        R.nx = c.x; R.ny = c.y; R.d = c.z; R.b0 = c.w;
        R.b1 = d.x; R.tnw = d.y; R.pad = 0;
    } else {
        R.xpm = R.ypm = nullptr;
        R.key = nullptr;
        R.r0 = R.xoff = R.nx = R.ny = R.d = R.b0 = R.b1 = R.tnw = 0;
        R.pad = 0;
    }
    return R;
}

template <class SH>
__global__ void __launch_bounds__(kTcThreads, 1)
pairs_tc_kernel(const LevelDesc* __restrict__ descs, const TcJobRec* __restrict__ recs,
                unsigned long long total_jobs, const unsigned long long* __restrict__ B,
                int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte alignment of the operand tiles (covers the 512-byte swizzle atom)
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t s0 = smem_u32(smem);
    const uint32_t bar = s0 + SH::kOffBar;
    // barrier slots (8 bytes each): a_full 0-1, a_empty 2-3, b_full 4-11, tile_done 12-19,
    // acc_empty 20-21.  One MMA commit per suffix tile signals both that its stage may be
    // refilled and that its accumulator is ready: the copier and the read-back warps wait
    // on the same tile_done barrier (tile i: stage i % kTcBStages, accumulator i & 1).
    auto a_full = [&](uint32_t i) { return bar + 8u * i; };
    auto a_empty = [&](uint32_t i) { return bar + 8u * (2 + i); };
    auto b_full = [&](uint32_t i) { return bar + 8u * (4 + i); };
    auto tile_done = [&](uint32_t i) { return bar + 8u * (4 + kTcBStages + i); };
    auto acc_empty = [&](uint32_t i) { return bar + 8u * (4 + 2 * kTcBStages + i); };
    constexpr int kNBar = 6 + 2 * kTcBStages;
    uint32_t counts[kNBar];
    for (int i = 0; i < kNBar; ++i) counts[i] = 1;
    counts[2] = counts[3] = 2;   // a prefix slot is released by both MMA threads
    // one arrival per read-back warp of the buffer's group
    counts[4 + 2 * kTcBStages] = counts[5 + 2 * kTcBStages] = kTcEpiWarps / kTcEpiGroups;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + SH::kOffBar + 256);
    const uint32_t tmem = tc_setup(bar, kNBar, counts, tmem_slot);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long j0 = blockIdx.x, js = gridDim.x;
    // Copies and MMA issue are split by suffix-tile parity over two threads each (warps 0
    // and 10 copy, warps 1 and 11 issue): every role is a chain of dependent barrier
    // operations, and two chains per role keep the tensor pipe fed.  The thread of parity p
    // owns the suffix stages of parity p and accumulator buffer p; the prefix tile is loaded
    // by the parity-0 copier and released when both MMA threads have committed.
    constexpr int kWarpCopy1 = 2 + kTcEpiWarps, kWarpMma1 = 3 + kTcEpiWarps;
    const bool is_copy = warp == 0 || warp == kWarpCopy1;
    const bool is_mma = warp == 1 || warp == kWarpMma1;
    const uint32_t par = warp >= kWarpCopy1 ? 1u : 0u;
    if (is_copy) {
        // ------------------------------------------------------------ tile copies
        if (lane == 0) {
            uint32_t it_a = 0, it_b = 0;
            bool ok = true;
            TcJobRec R = tc_rec(recs, j0, total_jobs);
            for (unsigned long long job = j0; ok && job < total_jobs; job += js) {
                const TcJobRec N = tc_rec(recs, job + js, total_jobs);   // next, in flight
                const int8_t* ypm = R.ypm;
                const uint32_t sa = it_a & 1u;
                if (par == 0) {
                    if (!(ok = mbar_wait(a_empty(sa), ((it_a >> 1) & 1u) ^ 1u))) break;
                    mbar_expect_tx(a_full(sa), SH::kABytes);
                    bulk_g2s(s0 + kTcOffA + sa * SH::kABytes, R.xpm + R.r0 * kPmRowBytes,
                             SH::kABytes, a_full(sa));
                }
                ++it_a;
                for (unsigned long long bt = R.b0; bt < R.b1; ++bt, ++it_b) {
                    if ((it_b & 1u) != par) continue;
                    const uint32_t sb = it_b % kTcBStages;
                    if (!(ok = mbar_wait(tile_done(sb), ((it_b / kTcBStages) & 1u) ^ 1u))) break;
                    mbar_expect_tx(b_full(sb), SH::kBBytes);
                    bulk_g2s(s0 + SH::kOffB + sb * SH::kBBytes, ypm + bt * SH::kN * kPmRowBytes,
                             SH::kBBytes, b_full(sb));
                }
                R = N;
            }
            if (!ok) atomicCAS(err, 0, 1);
        }
    } else if (is_mma) {
        // ------------------------------------------------------------ MMA issue
        if (lane == 0) {
            uint32_t it_a = 0, it_b = 0;
            bool ok = true;
            TcJobRec R = tc_rec(recs, j0, total_jobs);
            for (unsigned long long job = j0; ok && job < total_jobs; job += js) {
                const TcJobRec N = tc_rec(recs, job + js, total_jobs);
                const unsigned int tb0 = R.b0, tb1 = R.b1;
                R = N;
                const uint32_t sa = it_a & 1u;
                // both threads wait for the prefix tile before releasing it (keeps the
                // two arrivals of every release phase from different jobs apart)
                if (!(ok = mbar_wait(a_full(sa), (it_a >> 1) & 1u))) break;
                tc_fence_after();
                const uint32_t a_addr = s0 + kTcOffA + sa * SH::kABytes;
                for (unsigned int bt = tb0; bt < tb1; ++bt, ++it_b) {
                    if ((it_b & 1u) != par) continue;
                    const uint32_t sb = it_b % kTcBStages, ac = par;   // buffer = tile parity
                    if (!(ok = mbar_wait(b_full(sb), (it_b / kTcBStages) & 1u))) break;
                    if (!(ok = mbar_wait(acc_empty(ac), ((it_b >> 1) & 1u) ^ 1u))) break;
                    tc_fence_after();
                    const uint32_t b_addr = s0 + SH::kOffB + sb * SH::kBBytes;
#pragma unroll
                    for (int h = 0; h < SH::kHalves; ++h)
#pragma unroll
                        for (int k = 0; k < kTcK; ++k)   // K = 32 int8 columns = 32 bytes
                            mma_i8(tmem + ac * 256u + h * SH::kN,
                                   smem_desc(a_addr + h * kTcHalfBytes + 32u * k),
                                   smem_desc(b_addr + 32u * k), k > 0 ? 1u : 0u, SH::kIdesc);
                    mma_commit(tile_done(sb));
                }
                if (!ok) break;
                mma_commit(a_empty(sa));
                ++it_a;
            }
            if (!ok) atomicCAS(err, 0, 2);
        }
    } else {
        // ------------------------------------------------------------ read-back
        const int e = warp - 2;
        const int quarter = warp & 3;            // TMEM lanes [32*quarter, 32*quarter+32)
        const int sub = (e >> 2) & 1;            // which of the two warps of this quarter
        const int half = SH::kHalves == 2 ? sub : 0;    // prefix half (256 x 128 tiles)
        const int chunk = SH::kHalves == 2 ? 0 : sub;   // 128-column chunk (128 x 256 tiles)
        const uint32_t group = (uint32_t)(e >> 3);   // reads the tiles of this parity
        const int row = half * kTcM + quarter * 32 + lane;   // prefix-tile row
        const uint32_t col0 = (uint32_t)(half * SH::kN + chunk * 128);   // within a buffer
        uint32_t it_c = 0;
        bool ok = true;
        TcJobRec R = tc_rec(recs, j0, total_jobs);
        const unsigned long long* kptr = nullptr;   // key of the previous job
        int tkey = 0;                                // its value, loaded during that job
        for (unsigned long long job = j0; ok && job < total_jobs; job += js) {
            const TcJobRec C = R;
            R = tc_rec(recs, job + js, total_jobs);   // next, in flight
            const LevelDesc& D = descs[C.d];         // read only on the rare rescan path
            const unsigned long long r0 = C.r0, b0 = C.b0, b1 = C.b1;
            const unsigned long long r = r0 + row;
            const bool valid = r >= C.xoff && r < C.xoff + C.nx;
            // Bound: the level's bound at decode time, tightened by the key value read
            // during the previous job of the same level (a larger bound is always safe:
            // it only flags more slices).  This job's read is consumed by the next one.
            int T = (int)(C.tnw & 0xFFFu);
            if (C.key == kptr) T = min(T, tkey);
            const unsigned long long kv = *((volatile unsigned long long*)C.key);
            const int n_live = (int)((C.tnw >> 12) & 0xFFu);
            const bool rd = ((C.tnw >> 20) & 0x800u) != 0u;   // rank-deficient set
            const int w = (int)((C.tnw >> 20) & 0x7FFu);
            // pivot rows of this lane's prefix entry (its own count on a rank-deficient set,
            // else part of w); the bound below holds for every suffix entry of the set
            const int pcx = rd && valid ? (int)__ldg(D.pca + r) : 0;
            for (unsigned long long bt = b0; bt < b1; ++bt, ++it_c) {
                const uint32_t ac = it_c & 1u;
                if (ac != group) continue;               // the other group's tile
                // one lane polls the barrier, the warp follows (256 pollers would contend)
                if (lane == 0)
                    ok = mbar_wait(tile_done(it_c % kTcBStages), (it_c / kTcBStages) & 1u);
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) break;
                tc_fence_after();
                __syncwarp();   // the TMEM load below is warp-collective
                const int thr = n_live - 2 * (T - 1 - w - pcx);
                // the accumulators are in [-64, 64]: read them as packed 16-bit halves
                uint32_t v[64];
                tmem_ld128_p16(tmem + ((uint32_t)(quarter * 32) << 16) + ac * 256u + col0, v);
                // tcgen05.wait::ld (inside the load) has completed the reads of these columns,
                // so the release below needs no further tcgen05 fence
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty(ac));   // one arrival per warp
                after_release(v);
                // per 64-column slice (32 registers), four chains of 16-bit x2 3-input maxima
                uint32_t fbits = 0;
#pragma unroll
                for (int sl = 0; sl < 2; ++sl) {
                    uint32_t m[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int o = 32 * sl + 8 * c;
                        m[c] = v[o];
#pragma unroll
                        for (int i = o + 1; i + 1 < o + 8; i += 2) m[c] = __vimax3_s16x2(v[i], v[i + 1], m[c]);
                        m[c] = __vmaxs2(m[c], v[o + 7]);
                    }
                    const uint32_t mm = __vmaxs2(__vmaxs2(m[0], m[1]), __vmaxs2(m[2], m[3]));
                    const int mx = max((int)(int16_t)(mm & 0xFFFFu), (int)(int16_t)(mm >> 16));
                    if (mx >= thr) fbits |= 1u << sl;
                }
                const uint32_t flags = valid ? fbits : 0u;
                // Flagged slices are rescanned by the whole warp: the 32 lanes screen the
                // slice's 64 pairs on every stored probe word at once (an exact lower bound
                // on the weight), and only pairs still under the bound are rebuilt.
                uint32_t need = __ballot_sync(0xffffffffu, flags != 0u);
                while (need) {
                    const int src = __ffs(need) - 1;
                    need &= need - 1u;
                    const unsigned long long rr = __shfl_sync(0xffffffffu, r, src);
                    const uint32_t fl = __shfl_sync(0xffffffffu, flags, src);
                    const int pcr = __shfl_sync(0xffffffffu, pcx, src);
                    const int HP = D.HP;
                    uint32_t xr[4] = {0u, 0u, 0u, 0u};
                    for (int h = 0; h < HP; ++h) xr[h] = __ldg(D.la + rr * HP + h);
                    for (int sl = 0; sl < 128 / kTcSlice; ++sl) {
                        if (!(fl >> sl & 1u)) continue;
                        for (int part = 0; part < kTcSlice / 32; ++part) {
                            const unsigned long long c =
                                bt * SH::kN + chunk * 128 +
                                (unsigned long long)(sl * kTcSlice + part * 32 + lane);
                            bool cand = false;
                            if (c < C.ny) {
                                int lb = rd ? pcr + (int)__ldg(D.pcb + c) : D.a + D.b;
                                for (int h = 0; h < HP; ++h)
                                    lb += __popc(xr[h] ^ __ldg(D.rb + c * HP + h));
                                cand = lb < T;
                            }
                            uint32_t cm = __ballot_sync(0xffffffffu, cand);
                            while (cm) {
                                const int s2 = __ffs(cm) - 1;
                                cm &= cm - 1u;
                                const unsigned long long cc = __shfl_sync(0xffffffffu, c, s2);
                                int Tn = T;
                                if (lane == 0)
                                    Tn = survivor_scan(D, B, 1, C.xoff, rr - C.xoff, rd ? pcr : D.a,
                                                       cc, 1, T);
                                T = __shfl_sync(0xffffffffu, Tn, 0);
                            }
                        }
                    }
                }
            }
            if (!ok) break;
            kptr = C.key;
            tkey = min(T, (int)(kv >> kKeyWtShift));
            if (warp == 2 && lane == 0) {
                const unsigned long long lo = r0 > C.xoff ? r0 : C.xoff;
                const unsigned long long hi =
                    r0 + SH::kRows < C.xoff + C.nx ? r0 + SH::kRows : C.xoff + C.nx;
                const unsigned long long c_lo = b0 * SH::kN;
                const unsigned long long c_hi = b1 * SH::kN < C.ny ? b1 * SH::kN : C.ny;
                if (hi > lo && c_hi > c_lo) atomicAdd(D.count, (hi - lo) * (c_hi - c_lo));
            }
        }
        if (!ok && lane == 0) atomicCAS(err, 0, 3);
    }
    tc_teardown(tmem);
}

// +-1 expansion of packed probe words, one thread per row: the first two probe words (64
// columns) become 64 int8 values, written as four swizzled 16-byte chunks.
__global__ void __launch_bounds__(256) expand_pm_kernel(const ExpandDesc* __restrict__ descs,
                                                        int ndesc, unsigned long long total) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long ge = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         ge < total; ge += stride) {
        int lo = 0, hi = ndesc - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (descs[mid].row_base <= ge) lo = mid; else hi = mid - 1;
        }
        const ExpandDesc& E = descs[lo];
        const unsigned long long e = E.row_lo + (ge - E.row_base);
        uint32_t w0 = 0u, w1 = 0u;
        if (e < E.count) {
            w0 = __ldg(E.words + e * E.HP);
            if (E.HP > 1) w1 = __ldg(E.words + e * E.HP + 1);
        }
        write_pm_row(E.out, e, w0, w1, e < E.count ? E.n_enc : 0);   // padding rows: zeros
    }
}

// Self-test of the operand layout: D = A (256 x 64) * B (128 x 64)^T through the same
// copy / MMA / TMEM path (both halves), written out as 256 x 128 s32.  A and B are rows
// in the pre-swizzled layout.  ksteps < 0 is the timeout drill: no copy is issued, so the
// operand and accumulator waits run out after 50 ms and the error word is set, as a
// broken pipeline would; the launch still ends normally and frees its TMEM.
__global__ void __launch_bounds__(kTcThreads, 1)
tc_selftest_kernel(const int8_t* __restrict__ A, const int8_t* __restrict__ Bm, int ksteps,
                   int packed, int32_t* __restrict__ out, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t s0 = smem_u32(smem);
    const uint32_t bar = s0 + kTcOffBar;   // 0: operands landed, 1: accumulators ready
    const uint32_t counts[2] = {1, 1};
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTcOffBar + 256);
    const uint32_t tmem = tc_setup(bar, 2, counts, tmem_slot);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    bool ok = true;
    const bool drill = ksteps < 0;
    const unsigned long long limit = drill ? 50000000ull : kTcWaitNs;
    if (warp == 0 && lane == 0 && !drill) {
        mbar_expect_tx(bar, kTcABytes + kTcBBytes);
        bulk_g2s(s0 + kTcOffA, A, kTcABytes, bar);
        bulk_g2s(s0 + kTcOffB, Bm, kTcBBytes, bar);
    }
    if (warp == 1 && lane == 0) {
        ok = mbar_wait(bar, 0, limit);
        if (ok) {
            tc_fence_after();
            for (int h = 0; h < kTcHalves; ++h)
                for (int k = 0; k < ksteps; ++k)
                    mma_i8(tmem + h * kTcN, smem_desc(s0 + kTcOffA + h * kTcHalfBytes + 32u * k),
                           smem_desc(s0 + kTcOffB + 32u * k), k > 0 ? 1u : 0u);
            mma_commit(bar + 8);
        } else {
            atomicCAS(err, 0, 2);
        }
    }
    if (warp >= 2 && warp < 10) {   // one warp per (half, lane quarter)
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        ok = mbar_wait(bar + 8, 0, limit);
        ok = __all_sync(0xffffffffu, ok);
        if (ok) {
            tc_fence_after();
            __syncwarp();
            int32_t* o = out + (size_t)(half * kTcM + quarter * 32 + lane) * kTcN;
            if (packed) {   // the sweep's read-back: 16-bit halves, sign-extended here
                uint32_t v[64];
                tmem_ld128_p16(tmem + ((uint32_t)(quarter * 32) << 16) + half * kTcN, v);
                for (int i = 0; i < 64; ++i) {
                    o[2 * i] = (int32_t)(int16_t)(v[i] & 0xFFFFu);
                    o[2 * i + 1] = (int32_t)(int16_t)(v[i] >> 16);
                }
            } else {
                for (int cs = 0; cs < kTcN / kTcSlice; ++cs) {
                    int32_t v[64];
                    tmem_ld64(tmem + ((uint32_t)(quarter * 32) << 16) + half * kTcN + cs * kTcSlice, v);
                    for (int i = 0; i < 64; ++i) o[cs * kTcSlice + i] = v[i];
                }
            }
        } else if (lane == 0) {
            atomicCAS(err, 0, 3);
        }
    }
    tc_teardown(tmem);
}

}  // namespace dev

// ---------------------------------------------------------------- host launchers
// The sweep's tile shape, read once: 0 for 256 x 128 tiles (two prefix halves per suffix
// tile), 1 for 128 x 256 tiles (one MMA row block, N = 256); the tuning table's tc_shape,
// or QSFB_TC_SHAPE.  Both give the same answers and counts; the planner and the job decoder
// follow the active shape.
int tc_shape() {
    static const int shape = []() {
        const char* e = std::getenv("QSFB_TC_SHAPE");
        if (e) return std::atoi(e) == 0 ? 0 : 1;
        return tuning().tc_shape;
    }();
    return shape;
}
int tc_tile_rows() { return tc_shape() == 0 ? dev::TcHalvesShape::kRows : dev::TcWideShape::kRows; }
int tc_tile_cols() { return tc_shape() == 0 ? dev::TcHalvesShape::kN : dev::TcWideShape::kN; }
// the operand-layout self-test runs the 256 x 128 tile (its A and B are that size)
int tc_selftest_rows() { return dev::kTcRows; }
int tc_selftest_cols() { return dev::kTcN; }

cudaError_t launch_expand_pm(const ExpandDesc* d, int nd, unsigned long long total_rows,
                             int num_sms, cudaStream_t st) {
    if (total_rows == 0) return cudaSuccess;
    unsigned long long blocks = (total_rows + 255) / 256;
    const unsigned long long cap = (unsigned long long)num_sms * 16;
    if (blocks > cap) blocks = cap;
    dev::expand_pm_kernel<<<(unsigned)blocks, 256, 0, st>>>(d, nd, total_rows);
    return cudaGetLastError();
}

size_t tc_job_record_bytes() { return sizeof(dev::TcJobRec); }

template <class SH>
static cudaError_t launch_pairs_tc_t(const LevelDesc* d, int nd, unsigned long long jobs,
                                     const unsigned long long* B, dev::TcJobRec* recs, int* err,
                                     int num_sms, cudaStream_t st) {
    {
        unsigned long long blocks = (jobs + 255) / 256;
        const unsigned long long cap = (unsigned long long)num_sms * 8;
        if (blocks > cap) blocks = cap;
        dev::tc_jobs_kernel<SH><<<(unsigned)blocks, 256, 0, st>>>(d, nd, jobs, B, recs);
    }
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(dev::pairs_tc_kernel<SH>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SH::kSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    unsigned long long blocks = (unsigned long long)num_sms;
    if (jobs < blocks) blocks = jobs;
    dev::pairs_tc_kernel<SH><<<(unsigned)blocks, dev::kTcThreads, SH::kSmem, st>>>(d, recs, jobs,
                                                                                   B, err);
    return cudaGetLastError();
}

cudaError_t launch_pairs_tc(const LevelDesc* d, int nd, unsigned long long jobs,
                            const unsigned long long* B, void* job_recs, int* err, int num_sms,
                            cudaStream_t st) {
    if (jobs == 0) return cudaSuccess;
    dev::TcJobRec* recs = (dev::TcJobRec*)job_recs;
    return tc_shape() == 0
               ? launch_pairs_tc_t<dev::TcHalvesShape>(d, nd, jobs, B, recs, err, num_sms, st)
               : launch_pairs_tc_t<dev::TcWideShape>(d, nd, jobs, B, recs, err, num_sms, st);
}

cudaError_t launch_tc_selftest(const int8_t* A, const int8_t* Bm, int ksteps, int packed,
                               int32_t* out, int* err, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(dev::tc_selftest_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)dev::kTcSmem);
    if (e != cudaSuccess) return e;
    dev::tc_selftest_kernel<<<1, dev::kTcThreads, dev::kTcSmem, st>>>(A, Bm, ksteps, packed, out,
                                                                     err);
    return cudaGetLastError();
}

}  // namespace qsfb
