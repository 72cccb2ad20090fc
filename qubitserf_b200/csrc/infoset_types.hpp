// Descriptor of one side's information-set construction on the device (one warp per side).
#pragma once
#include <cstdint>

namespace qsfb {

constexpr int kInfosetMaxK = 128;    // rows held in registers (4 slots x 32 lanes)
constexpr int kInfosetMaxN = 128;    // columns (two 64-bit words per row)
constexpr int kInfosetMaxSets = 16;  // sets per side on the device; more -> host construction

// Per-side results the host reads back (one 512-byte block per side).
struct InfosetMeta {
    int sets;                                     // number of sets; -1: more than kInfosetMaxSets
    int rank[kInfosetMaxSets];                    // pivots of each set
    int g_off[kInfosetMaxSets];                   // each set's generator: offset (u64 words) in the heap
    int pad_[31];
    unsigned long long piv[kInfosetMaxSets][2];   // pivot columns of each set (bit mask)
};
static_assert(sizeof(InfosetMeta) == 512, "meta block");

struct InfosetDesc {
    const unsigned long long* gen;    // K x W rows of the code generator
    const unsigned long long* check;  // kcheck x W detector rows
    const uint8_t* lists;             // explicit sets: column lists, concatenated (nullptr: greedy peel)
    InfosetMeta* meta;
    uint32_t* red;                    // kInfosetMaxSets x K x W32 non-pivot bits, ascending columns
    uint32_t* syn;                    // kInfosetMaxSets x K x SWP detector syndrome bits
    int K, n, kcheck, W32, SWP;
    int nlists;                       // explicit sets: number of lists (<= kInfosetMaxSets)
    int list_len[kInfosetMaxSets];    // explicit sets: length of each list
};

}  // namespace qsfb
