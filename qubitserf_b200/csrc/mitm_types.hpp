// Plain-old-data shared by the host driver of the meet-in-the-middle distance (mitm.cpp)
// and its kernels (mitm.cu).
//
// The reference's method "mitm" (cpp/distfind/mitm.cpp:1-21): with H = nullspace(code_gen)
// a parity check of the searched code, split the coordinates into Left = [0, nL) and
// Right = [nL, ncoord); a vector of weight d = wL + wR with left part SL and right part SR
// is a codeword iff syn(SL) = syn(SR) (syn = XOR of H's columns), and a logical iff
// count_all or log(SL) != log(SR) (log = XOR of the detector's columns).  Level d is a hit
// when some (wL, d - wL) split matches.  Symplectic problems count qubits: a part picks w
// qubits and one of Z, X, Y on each (3^w parts per qubit set).
//
// Device join: the parts of one left weight go into an open-addressing table keyed by
// their syndrome (a 64-bit tag of it claims a slot with one CAS; the full syndrome and the
// first logical fingerprint sit beside it), built once and probed by the right parts of
// every level that needs that weight.
#pragma once
#include <cstdint>

namespace qsfb {

constexpr int kMitmMaxSynWords = 16;   // 32-bit words of a syndrome: n - K <= 512
constexpr int kMitmMaxLogWords = 8;    // 32-bit words of a logical fingerprint: kcheck <= 256
constexpr int kMitmMaxWeight = 32;     // part weight (combination size)

// status words of a table / probe launch
enum MitmStatus : int {
    kMitmFound = 0,       // some right part matched a left part as a logical
    kMitmCollision = 1,   // two different syndromes share a 64-bit tag: rebuild, new seed
    kMitmOverrun = 2,     // a probe walked the whole table (cannot happen below load 1)
};

struct MitmTable {
    unsigned long long* tag;    // cap: 0 = empty, else hash | 1
    uint32_t* key;              // cap x (SW + LW): syndrome then first logical fingerprint
    uint32_t* flags;            // cap: bit 0 = the bucket holds two different fingerprints
    unsigned long long mask;    // cap - 1 (cap a power of two)
    unsigned long long seed;
    unsigned long long tag_mask;  // hash bits kept in a tag (all but in the collision drill)
};

struct MitmShared {
    const uint32_t* syn_cols;   // ncols x SW: column j of H, bit i = H[i][j]
    const uint32_t* log_cols;   // ncols x LW: column j of the detector (LW = 0: count_all)
    int SW, LW;
    int sym;                    // symplectic parts (qubits, Z/X/Y) instead of bits
    int qubits;                 // symplectic: x column of qubit j is qubits + j
    int* status;                // MitmStatus words
};

}  // namespace qsfb
