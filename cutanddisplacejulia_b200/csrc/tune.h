// The library's autotuner (csrc/tune.cu): launch shapes chosen by timing the
// candidates on the device the first time a (kernel, size class, precision)
// key is met, remembered in a per-context table and in a cache file that
// later processes read.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <vector>

namespace cad {

enum { TUNE_OFF = 0, TUNE_ON = 1, TUNE_CACHED = 2 };

struct Tuner {
    int mode = TUNE_OFF;          // TUNE_ON: time missing keys; TUNE_CACHED: use stored keys only
    std::string path;             // cache file ("" = none)
    std::map<std::string, int> table;
    int64_t tuned = 0;            // keys timed in this process

    // loads `path` (lines "key value"); a missing file is an empty cache
    bool load(const std::string& p);
    bool save() const;
    // the stored choice for key, or -1
    int find(const std::string& key) const;
};

// Size class of a dimension: the power of two at or above it.
int64_t tune_class(int64_t n);

// Runs each candidate's launch sequence `run(candidate)` twice on stream st
// (the first run warms up), times the second with CUDA events and returns the
// fastest candidate, or `fallback` if a launch fails.  Every run must leave
// the same results behind (the tuned kernels' outputs do not depend on the
// launch shape).
int tune_pick(cudaStream_t st, const std::vector<int>& candidates, int fallback,
              const std::function<cudaError_t(int)>& run);

// The choice for key: the stored one; else, in TUNE_ON mode, the fastest
// candidate (timed, stored, and written to the cache file); else fallback.
int tune_choice(Tuner& t, const std::string& key, cudaStream_t st, const std::vector<int>& candidates, int fallback,
                const std::function<cudaError_t(int)>& run);

}  // namespace cad
