// Meet-in-the-middle distance (method "mitm") on the device: same problems, results and
// level semantics as the reference's mitm_distance / mitm_min_interleaved
// (cpp/distfind/mitm.cpp:318-537).  No witness is produced (the reference returns none).
#pragma once
#include "bz.hpp"

namespace qsfb {

// One subproblem (bit or symplectic weight by p.symplectic).
int mitm_distance(Device* dev, const Problem& p, BzResult& r);
// CSS which='min': Z and X stepped one level at a time, a side capped once it cannot lower
// the running minimum.
int mitm_min_interleaved(Device* dev, const Problem& pz, const Problem& px, BzResult& r);

}  // namespace qsfb
