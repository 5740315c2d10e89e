// Autotuner: candidate launch shapes timed with CUDA events on the caller's
// stream, the fastest remembered per (kernel, size class, precision) key.
#include "tune.h"

#include <cstdio>
#include <fstream>
#include <sstream>

namespace cad {

bool Tuner::load(const std::string& p)
{
    path = p;
    table.clear();
    if (p.empty()) return true;
    std::ifstream in(p);
    if (!in) return true;   // no cache yet
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string key;
        int v = 0;
        if (ls >> key >> v && !key.empty() && key[0] != '#') table[key] = v;
    }
    return true;
}

bool Tuner::save() const
{
    if (path.empty()) return true;
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::trunc);
        if (!out) return false;
        out << "# libcad_td autotune cache: key value (launch shape chosen by timing on this device)\n";
        for (const auto& kv : table) out << kv.first << " " << kv.second << "\n";
        if (!out) return false;
    }
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

int Tuner::find(const std::string& key) const
{
    auto it = table.find(key);
    return it == table.end() ? -1 : it->second;
}

int64_t tune_class(int64_t n)
{
    int64_t c = 1;
    while (c < n) c <<= 1;
    return c;
}

int tune_pick(cudaStream_t st, const std::vector<int>& candidates, int fallback,
              const std::function<cudaError_t(int)>& run)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return fallback;
    }
    int best = fallback;
    float best_ms = 0.f;
    bool have = false;
    for (int c : candidates) {
        if (run(c) != cudaSuccess) {   // warm-up (and validity)
            have = false;
            break;
        }
        cudaEventRecord(e0, st);
        const cudaError_t e = run(c);
        cudaEventRecord(e1, st);
        if (e != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
            have = false;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (!have || ms < best_ms) {
            best = c;
            best_ms = ms;
            have = true;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return have ? best : fallback;
}

int tune_choice(Tuner& t, const std::string& key, cudaStream_t st, const std::vector<int>& candidates, int fallback,
                const std::function<cudaError_t(int)>& run)
{
    const int stored = t.find(key);
    if (stored >= 0 && t.mode != TUNE_OFF) return stored;
    if (t.mode != TUNE_ON) return fallback;
    const int best = tune_pick(st, candidates, fallback, run);
    t.table[key] = best;
    ++t.tuned;
    t.save();
    return best;
}

}  // namespace cad
