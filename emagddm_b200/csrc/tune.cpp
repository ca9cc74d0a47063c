// tune.cpp -- launch-configuration autotuner (see tune.h).
#include "tune.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

namespace emg {
namespace tune {
namespace {

constexpr int kReps = 5;

struct Entry {
  int value = 0;
  std::vector<std::pair<int, double>> ms;  // candidate value, median ms (empty when read from the cache file)
};

std::mutex g_mu;
std::map<std::string, Entry> g_table;
bool g_loaded = false;
int g_enabled = -1;  // -1: not read from the environment yet

const char* cache_path() {
  const char* p = std::getenv("EMG_TUNE_CACHE");
  return p && p[0] ? p : nullptr;
}

// Cache file lines: "<family>|<key> <value>"
void load_cache() {
  if (g_loaded) return;
  g_loaded = true;
  const char* p = cache_path();
  if (!p) return;
  std::ifstream f(p);
  std::string line;
  while (std::getline(f, line)) {
    const size_t sp = line.rfind(' ');
    if (sp == std::string::npos) continue;
    Entry e;
    e.value = std::atoi(line.c_str() + sp + 1);
    g_table[line.substr(0, sp)] = e;
  }
}

void append_cache(const std::string& id, int value) {
  const char* p = cache_path();
  if (!p) return;
  std::ofstream f(p, std::ios::app);
  f << id << ' ' << value << '\n';
}

double median(std::vector<float> v) {
  std::sort(v.begin(), v.end());
  return v.empty() ? 0.0 : v[v.size() / 2];
}

}  // namespace

bool enabled() {
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_enabled < 0) {
    const char* e = std::getenv("EMG_TUNE");
    g_enabled = (e && e[0] == '0') ? 0 : 1;
  }
  return g_enabled != 0;
}

void set_enabled(bool on) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_enabled = on ? 1 : 0;
}

int pick(const std::string& family, const std::string& key, const std::vector<int>& candidates,
         const std::function<void(int, cudaStream_t)>& launch, cudaStream_t st) {
  if (candidates.empty()) return 0;
  if (!enabled() || candidates.size() == 1) return candidates[0];
  const std::string id = family + "|" + key;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    load_cache();
    auto it = g_table.find(id);
    if (it != g_table.end() &&
        std::find(candidates.begin(), candidates.end(), it->second.value) != candidates.end())
      return it->second.value;
  }
  cudaEvent_t ev[kReps + 1];
  for (cudaEvent_t& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return candidates[0]; }
  Entry best;
  double best_ms = 0.0;
  bool ok = true;
  for (int c : candidates) {
    launch(c, st);  // warm-up
    cudaEventRecord(ev[0], st);
    for (int r = 0; r < kReps; ++r) {
      launch(c, st);
      cudaEventRecord(ev[r + 1], st);
    }
    if (cudaEventSynchronize(ev[kReps]) != cudaSuccess || cudaGetLastError() != cudaSuccess) { ok = false; break; }
    std::vector<float> t(kReps);
    for (int r = 0; r < kReps; ++r) cudaEventElapsedTime(&t[r], ev[r], ev[r + 1]);
    const double m = median(t);
    best.ms.emplace_back(c, m);
    if (best.ms.size() == 1 || m < best_ms) { best_ms = m; best.value = c; }
  }
  for (cudaEvent_t& e : ev) cudaEventDestroy(e);
  if (!ok) return candidates[0];
  std::lock_guard<std::mutex> lock(g_mu);
  g_table[id] = best;
  append_cache(id, best.value);
  return best.value;
}

std::string report() {
  std::lock_guard<std::mutex> lock(g_mu);
  std::ostringstream o;
  o << '{';
  bool first = true;
  for (const auto& kv : g_table) {
    if (!first) o << ", ";
    first = false;
    o << '"' << kv.first << "\": {\"value\": " << kv.second.value << ", \"candidates_ms\": {";
    for (size_t i = 0; i < kv.second.ms.size(); ++i) {
      char buf[64];
      std::snprintf(buf, sizeof(buf), "%s\"%d\": %.4f", i ? ", " : "", kv.second.ms[i].first, kv.second.ms[i].second);
      o << buf;
    }
    o << "}}";
  }
  o << '}';
  return o.str();
}

}  // namespace tune
}  // namespace emg
