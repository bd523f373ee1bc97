// Online launch-shape tuner (launch_tuner.hpp).
#include "launch_tuner.hpp"

#include <algorithm>
#include <sstream>

#include "common.cuh"

namespace dcaacc {

namespace {
float median(std::vector<float> v) {
  std::sort(v.begin(), v.end());
  return v[v.size() / 2];
}
}  // namespace

LaunchTuner::~LaunchTuner() {
  for (auto& p : pending_) {
    cudaEventSynchronize(p.e);
    cudaEventDestroy(p.b);
    cudaEventDestroy(p.e);
  }
  for (auto e : pool_)
    cudaEventDestroy(e);
}

cudaEvent_t LaunchTuner::event() {
  if (!pool_.empty()) {
    cudaEvent_t e = pool_.back();
    pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  DCAACC_CUDA_CHECK(cudaEventCreate(&e));
  return e;
}

// Moves the completed probes' times into their entries; with wait_key, first waits for that key's
// closed probes.
void LaunchTuner::harvest(const std::string* wait_key) {
  for (size_t i = 0; i < pending_.size();) {
    Probe& p = pending_[i];
    if (!p.closed) {
      ++i;
      continue;
    }
    if (wait_key && p.key == *wait_key)
      DCAACC_CUDA_CHECK(cudaEventSynchronize(p.e));
    const cudaError_t q = cudaEventQuery(p.e);
    if (q == cudaErrorNotReady) {
      ++i;
      continue;
    }
    DCAACC_CUDA_CHECK(q);
    float ms = 0.f;
    DCAACC_CUDA_CHECK(cudaEventElapsedTime(&ms, p.b, p.e));
    auto it = entries_.find(p.key);
    if (it != entries_.end())
      it->second.ms[p.cand].push_back(ms);
    pool_.push_back(p.b);
    pool_.push_back(p.e);
    pending_.erase(pending_.begin() + i);
  }
}

void LaunchTuner::decide(Entry& e) {
  int best = -1;
  float best_ms = 0.f;
  for (int c = 0; c < e.n; ++c) {
    if (e.ms[c].empty())
      continue;
    const float m = median(e.ms[c]);
    if (best < 0 || m < best_ms) {
      best = c;
      best_ms = m;
    }
  }
  e.chosen = best < 0 ? 0 : best;
  --exploring_;
}

LaunchTuner::Pick LaunchTuner::pick(const std::string& key, int n, cudaStream_t s) {
  if (!enabled_ || n <= 1)
    return Pick{};
  auto it = entries_.find(key);
  if (it == entries_.end()) {
    it = entries_.emplace(key, Entry{}).first;
    it->second.n = n;
    it->second.ms.assign(n, {});
    ++exploring_;
  }
  Entry& e = it->second;
  if (e.chosen >= 0)
    return Pick{e.chosen, -1};
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  DCAACC_CUDA_CHECK(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return Pick{};  // no events inside a capture (the accumulator captures only when settled)
  harvest(nullptr);
  if (e.issued >= e.n * kReps) {
    harvest(&key);
    decide(e);
    return Pick{e.chosen, -1};
  }
  Probe p{next_id_++, key, e.issued % e.n, event(), event(), false};
  ++e.issued;
  DCAACC_CUDA_CHECK(cudaEventRecord(p.b, s));
  pending_.push_back(p);
  return Pick{p.cand, p.id};
}

void LaunchTuner::end(const Pick& p, cudaStream_t s) {
  if (p.probe < 0)
    return;
  for (auto it = pending_.rbegin(); it != pending_.rend(); ++it)
    if (it->id == p.probe) {
      DCAACC_CUDA_CHECK(cudaEventRecord(it->e, s));
      it->closed = true;
      return;
    }
}

std::string LaunchTuner::report() {
  harvest(nullptr);
  std::ostringstream o;
  for (auto& [key, e] : entries_) {
    o << key << " n=" << e.n << " choice=" << e.chosen << " ms=";
    for (int c = 0; c < e.n; ++c)
      o << (c ? "," : "") << (e.ms[c].empty() ? -1.f : median(e.ms[c]));
    o << "\n";
  }
  return o.str();
}

}  // namespace dcaacc
