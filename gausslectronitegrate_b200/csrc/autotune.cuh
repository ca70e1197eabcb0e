// Autotuner: for a shape key, time every candidate launch configuration once
// on the real work (each run computes the full, correct result), keep the
// fastest, and reuse that choice for every later call with the same key.
#pragma once
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace gli {

class Autotuner {
public:
    // Returns the candidate with the least time_ms(candidate) for `key`; the
    // first call for a key measures every candidate (min of two runs after one
    // warm-up run), later calls return the recorded choice without measuring.
    // GLI_B200_TUNE_<NAME>=<value> in the environment (NAME = the key's first
    // word, upper-cased) forces a candidate.
    int choose(const std::string& key, const std::vector<int>& candidates,
               const std::function<double(int)>& time_ms);
    // JSON object: key -> {"best": c, "ms": {candidate: ms, ...}}
    std::string report() const;
    void clear();

private:
    struct Decision {
        int best = 0;
        std::vector<std::pair<int, double>> timings;
    };
    mutable std::mutex mu_;
    std::map<std::string, Decision> table_;
};

Autotuner& autotune();

}  // namespace gli
