// Autotuner (see tune.h).
#include "tune.h"

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>

namespace hb {

namespace {

struct Timing {
  std::string key;
  int index = 0;
  cudaEvent_t a = nullptr, b = nullptr;
  double units = 0;
  bool ended = false;
};

struct Entry {
  std::vector<int> cand;
  std::vector<double> ms_per_unit;   // best completed timing per candidate, < 0 while unmeasured
  int next = 0;
  int decided = -1;
};

std::mutex g_mu;
std::map<std::string, Entry> g_table;
std::map<int, Timing> g_open;
int g_token = 0;

bool env_is(const char* name, const char* value) {
  const char* v = std::getenv(name);
  return v && std::string(v) == value;
}

bool enabled() {
  static const bool on = !env_is("HALF_TUNE", "0");
  return on;
}

std::string full_key(const std::string& key) {
  int dev = 0;
  cudaGetDevice(&dev);
  return std::to_string(dev) + "|" + key;
}

void decide(const std::string& key, Entry& e) {
  if (e.decided >= 0) return;
  int best = -1;
  for (size_t i = 0; i < e.cand.size(); ++i) {
    if (e.ms_per_unit[i] < 0) return;
    if (best < 0 || e.ms_per_unit[i] < e.ms_per_unit[best]) best = int(i);
  }
  e.decided = best;
  if (env_is("HALF_TUNE_LOG", "1")) {
    std::fprintf(stderr, "HALF tune %s ->", key.c_str());
    for (size_t i = 0; i < e.cand.size(); ++i)
      std::fprintf(stderr, " %d:%.4g%s", e.cand[i], e.ms_per_unit[i], int(i) == best ? "*" : "");
    std::fprintf(stderr, " (ms per unit)\n");
  }
}

// Completed timings -> table (under g_mu).  Never waits.
void harvest() {
  for (auto it = g_open.begin(); it != g_open.end();) {
    Timing& t = it->second;
    if (!t.ended) { ++it; continue; }
    const cudaError_t q = cudaEventQuery(t.b);
    if (q == cudaErrorNotReady) { ++it; continue; }
    if (q == cudaSuccess) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess && t.units > 0) {
        Entry& e = g_table[t.key];
        if (t.index < int(e.ms_per_unit.size())) {
          const double v = double(ms) / t.units;
          double& cur = e.ms_per_unit[t.index];
          if (cur < 0 || v < cur) cur = v;
          decide(t.key, e);
        }
      } else {
        cudaGetLastError();
      }
    } else {
      cudaGetLastError();
    }
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
    it = g_open.erase(it);
  }
}

}  // namespace

int Tuner::pick(const std::string& key, const std::vector<int>& candidates) {
  if (!enabled() || candidates.size() <= 1) return 0;
  const std::string k = full_key(key);
  std::lock_guard<std::mutex> lock(g_mu);
  harvest();
  Entry& e = g_table[k];
  if (e.cand != candidates) {
    e.cand = candidates;
    e.ms_per_unit.assign(candidates.size(), -1.0);
    e.next = 0;
    e.decided = -1;
  }
  if (e.decided >= 0) return e.decided;
  const int n = int(e.cand.size());
  for (int t = 0; t < n; ++t) {
    const int i = (e.next + t) % n;
    if (e.ms_per_unit[i] < 0) {
      e.next = i + 1;
      return i;
    }
  }
  return 0;
}

int Tuner::begin(const std::string& key, int index, cudaStream_t s) {
  if (!enabled()) return 0;
  const std::string k = full_key(key);
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_table.find(k);
  if (it == g_table.end() || it->second.decided >= 0) return 0;   // nothing left to measure
  Timing t;
  t.key = k;
  t.index = index;
  if (cudaEventCreate(&t.a) != cudaSuccess || cudaEventCreate(&t.b) != cudaSuccess) {
    cudaGetLastError();
    if (t.a) cudaEventDestroy(t.a);
    return 0;
  }
  cudaEventRecord(t.a, s);
  const int token = ++g_token;
  g_open[token] = t;
  return token;
}

void Tuner::finish(int token, cudaStream_t s, double units) {
  if (token == 0) return;
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_open.find(token);
  if (it == g_open.end()) return;
  cudaEventRecord(it->second.b, s);
  it->second.units = units;
  it->second.ended = true;
}

int Tuner::decided(const std::string& key) {
  const std::string k = full_key(key);
  std::lock_guard<std::mutex> lock(g_mu);
  harvest();
  auto it = g_table.find(k);
  return it == g_table.end() ? -1 : it->second.decided;
}

}  // namespace hb
