// Launch shapes of the engine that are chosen by measurement rather than fixed.
//
// Defaults are the hand-set values.  A table of `key value` lines overrides them: the file
// `tuning.txt` next to the library (written by `python -m qubitserf_b200.tune`, which
// measures every candidate on the GPU it runs on and keeps the fastest), or the file named
// by QSFB_TUNING; QSFB_TUNE_<KEY> (dots as underscores, upper case) overrides one entry.
// Every choice gives the same answers and counts; only the time differs.
#pragma once
#include <string>

namespace qsfb {

struct Tuning {
    int tc_shape = 1;                  // tensor-core sweep tile: 0 = 256 x 128, 1 = 128 x 256
    int tc_job_tiles_small = 16;       // suffix tiles per tensor-core job, small levels
    int tc_job_tiles_large = 16;       // ... large levels
    long long tc_small_tiles = 4096;   // level-size class boundary: tiles of its tensor plan
    int cc_jobs_per_warp = 16;         // CUDA-core sweep: jobs per resident warp (loop tile)
    double tc_cost_ratio = 0.6;        // tensor plan when its cost < ratio x CUDA-core cost
    // terms join a level's tensor-core range while their prefix rows reach tile rows / div
    // and their suffix columns tile columns / div (the rest go to the CUDA cores)
    int tc_edge_div = 2;
    int exec_groups = 3;               // interleaved job groups of qsfb_batch_execute
    int batch_chunks = 4;              // pipeline chunks of the one-shot qsfb_batch
    // the first chunk's share of the batch in 1/1000 (0: half a chunk, nq / (2 chunks));
    // it is prepared before any round starts
    int batch_first_permille = 0;
    int overlap_groups = 3;            // job groups of the one-shot qsfb_batch
    std::string source = "defaults";   // where the values came from
};

// The process-wide tuning, read once.
const Tuning& tuning();

// Suffix tiles per tensor-core job for a level whose tensor plan covers `tiles` tiles.
int tc_job_tiles_for(unsigned long long tiles);

}  // namespace qsfb
