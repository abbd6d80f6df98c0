// Launch-shape autotuner: for a launch whose shape (threads, resident blocks per SM, ring
// stages) can change without changing its arithmetic, the candidates are timed once
// on the real problem with CUDA events and the fastest is remembered, per (kernel,
// problem shape, device), in a text file that later processes read again.
//
// Cache file: $ETCU_TUNE_CACHE, else $HOME/.cache/ettention_b200/launch_shapes.txt; one
// "key value" line per choice (the last line of a key wins).  The choice never changes a
// result: every candidate computes the same values in the same order.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace etcu_tune {

// The cached choice of `key`, or -1.
int lookup(const std::string& key);
// Remembers `value` for `key` (in memory and appended to the cache file).
void store(const std::string& key, int value);
// "<device name>|sm<major><minor>|<multiprocessors>".
std::string device_tag(int device);
// Runs run(c) once untimed and `reps` times timed (CUDA events on `st`) for every
// candidate c; returns the fastest candidate, or -1 when every run failed.  `log`
// receives one "c=ms" entry per candidate.
int search(cudaStream_t st, const std::vector<int>& candidates, const std::function<bool(int)>& run, int reps,
           std::string* log);

}  // namespace etcu_tune
