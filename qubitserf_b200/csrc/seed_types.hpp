// Descriptor of one side's random-information-set trials on the device.
#pragma once
#include <cstdint>

namespace qsfb {

constexpr int kSeedMaxK = 128;   // rows held in registers (4 slots x 32 lanes)
constexpr int kSeedMaxN = 256;   // columns (up to four 64-bit words per row)

struct SeedDesc {
    const unsigned long long* gen;    // K x W code generator rows
    const unsigned long long* check;  // kcheck x W detector rows
    const uint8_t* perm;              // trials x n column orders (n <= 256)
    unsigned* key;                    // (weight:17 | trial:8 | row:7), atomicMin
    int trial_base;                   // first global trial of this side
    int K, n, kcheck, count_all, init_best, pad_;
};

}  // namespace qsfb
