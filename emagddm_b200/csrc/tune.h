// tune.h -- the library's own launch-configuration autotuner.
//
// For a kernel family and a problem key (the shape that decides the best
// configuration), pick() times every candidate value on the device -- one
// untimed launch, then kReps launches between CUDA events on the given
// stream, median -- and keeps the fastest in a process-wide table, so the
// measurement runs once per (family, key).  The first candidate is the
// built-in default: with EMG_TUNE=0 in the environment (or tuning switched
// off through emg_tune_enable) it is used without timing.  EMG_TUNE_CACHE
// names a text file that carries the table between processes (read at the
// first pick, appended to after every new decision).  report() lists the
// decisions with every candidate's median time, as JSON.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace emg {
namespace tune {

// launch(value, stream) must enqueue one run of the tuned work with the
// candidate value and nothing else; it may be called up to 1 + kReps times
// per candidate.  Returns the chosen value (the default when tuning is off or
// a launch fails).
int pick(const std::string& family, const std::string& key, const std::vector<int>& candidates,
         const std::function<void(int, cudaStream_t)>& launch, cudaStream_t st);

bool enabled();
void set_enabled(bool on);
std::string report();

}  // namespace tune
}  // namespace emg
