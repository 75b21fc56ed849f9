// Launch-schedule autotuner: picks one of a kernel's launch variants (tile shape, warps per CTA,
// CTAs per SM, ...) for a given device and problem shape by timing every variant on the caller's
// stream the first time that key is seen in the process, and caches the choice.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace vbcore {

// Returns the chosen variant for `key` (one of 0 .. n_variants - 1).  On a cache miss each variant
// runs once untimed and then `reps` times between CUDA events (best time kept); `reset` (may be
// empty) runs before every variant launch to restore what a launch consumes (counters, lists).
// Every variant must produce the same results, so the outputs of the last run stand.  Runs the
// chosen variant itself only when the key was cached (on a miss the timing runs have produced the
// outputs).  The environment variable VBCORE_AUTOTUNE=0 turns timing off: variant 0 (the default
// schedule) is used.  *status receives the first launch error.
int autotune_run(const std::string& key, int n_variants, cudaStream_t stream,
                 const std::function<cudaError_t(int)>& launch, const std::function<cudaError_t()>& reset,
                 cudaError_t* status, int reps = 2);

// One line per cached key: "key -> variant (ms of each variant)".
std::string autotune_report();
void autotune_clear();

}  // namespace vbcore
