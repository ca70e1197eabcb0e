// Autotuner (see autotune.cuh).  Host code only.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <limits>

#include "autotune.cuh"
#include "gli_internal.cuh"

namespace gli {

Autotuner& autotune() {
    static Autotuner t;
    return t;
}

int Autotuner::choose(const std::string& key, const std::vector<int>& candidates,
                      const std::function<double(int)>& time_ms) {
    if (candidates.empty()) fail(GLI_ERR_INTERNAL, "autotuner: no candidates for %s", key.c_str());
    std::string name = key.substr(0, key.find(' '));
    for (char& c : name) c = (char)toupper((unsigned char)c);
    if (const char* forced = getenv(("GLI_B200_TUNE_" + name).c_str())) {
        const int v = atoi(forced);
        if (std::find(candidates.begin(), candidates.end(), v) != candidates.end()) return v;
    }
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = table_.find(key);
        if (it != table_.end()) return it->second.best;
    }
    if (candidates.size() == 1) {
        std::lock_guard<std::mutex> lk(mu_);
        table_[key] = Decision{candidates[0], {}};
        return candidates[0];
    }
    Decision d;
    double best_ms = std::numeric_limits<double>::infinity();
    for (int c : candidates) {
        time_ms(c);  // warm-up: first-use costs (allocation pools, module loading)
        const double t = std::min(time_ms(c), time_ms(c));
        d.timings.push_back({c, t});
        if (t < best_ms) {
            best_ms = t;
            d.best = c;
        }
    }
    std::lock_guard<std::mutex> lk(mu_);
    table_[key] = d;
    return d.best;
}

std::string Autotuner::report() const {
    std::lock_guard<std::mutex> lk(mu_);
    std::string s = "{";
    bool first = true;
    for (const auto& kv : table_) {
        char buf[64];
        s += first ? "\"" : ", \"";
        first = false;
        s += kv.first + "\": {\"best\": " + std::to_string(kv.second.best) + ", \"ms\": {";
        for (size_t i = 0; i < kv.second.timings.size(); ++i) {
            snprintf(buf, sizeof(buf), "%s\"%d\": %.4f", i ? ", " : "", kv.second.timings[i].first,
                     kv.second.timings[i].second);
            s += buf;
        }
        s += "}}";
    }
    return s + "}";
}

void Autotuner::clear() {
    std::lock_guard<std::mutex> lk(mu_);
    table_.clear();
}

}  // namespace gli

// ---------------------------------------------------------------------------
// C entry points

// JSON of the autotuner's decisions into buf (truncated to len); returns the
// full length
extern "C" glong gli_b200_autotune_report(char* buf, glong len) {
    const std::string s = gli::autotune().report();
    if (buf && len > 0) {
        const size_t n = std::min((size_t)(len - 1), s.size());
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return (glong)s.size();
}

// Checks the autotuner's selection logic with a synthetic cost model (no
// device work): the fastest candidate wins, the choice is cached (no second
// measurement), and each candidate is measured three times.  Returns 0 on success.
extern "C" int gli_b200_autotune_selftest(void) {
    gli::Autotuner t;
    int calls = 0;
    auto cost = [&](int c) {
        ++calls;
        return 10.0 + (c - 4) * (c - 4);  // minimum at 4
    };
    const std::vector<int> cands = {1, 2, 4, 8};
    if (t.choose("selftest a", cands, cost) != 4) return 1;
    if (calls != 3 * (int)cands.size()) return 2;
    if (t.choose("selftest a", cands, cost) != 4) return 3;
    if (calls != 3 * (int)cands.size()) return 4;
    if (t.choose("selftest b", {8}, cost) != 8) return 5;
    if (t.report().find("\"selftest a\": {\"best\": 4") == std::string::npos) return 6;
    return 0;
}
