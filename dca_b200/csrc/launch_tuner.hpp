// Online launch-shape tuner.
//
// A tuning site is a kernel launch with several launch shapes (tile widths, threads or warps per
// block, persistent grid sizes) that give bit-identical results: every candidate computes each
// output with the same arithmetic in the same order, so only the time differs.  The site asks the
// tuner which candidate to launch for its key (the kernel family and the problem shape: bands,
// cluster size, frequencies, order bound, batch).  Candidate 0 is the built-in heuristic.  The
// first kReps x n launches of a key run every candidate in turn between two CUDA events on the
// launching stream (no extra work: each probe is a real launch of the real batch); once they have
// completed, the candidate with the smallest median time is kept for the key.  Nothing blocks
// while probes are in flight, except that a key whose last probe has been issued waits for its
// events at its next launch.  Probing never happens inside a stream capture, and the accumulator
// captures a batch shape's CUDA graph only after a batch of that shape ran without probes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace dcaacc {

class LaunchTuner {
public:
  static constexpr int kReps = 3;  // timed launches per candidate

  struct Pick {
    int choice = 0;     // candidate to launch
    long probe = -1;    // >= 0: a timed probe, close it with end()
  };

  explicit LaunchTuner(bool enabled = true) : enabled_(enabled) {}
  ~LaunchTuner();
  LaunchTuner(const LaunchTuner&) = delete;
  LaunchTuner& operator=(const LaunchTuner&) = delete;

  // The candidate for this launch of `key` among n; a probe records its start event on s.
  Pick pick(const std::string& key, int n, cudaStream_t s);
  // Records the end event of a probe (no-op for a plain pick).
  void end(const Pick& p, cudaStream_t s);
  // No key is exploring.
  bool settled() const {
    return exploring_ == 0;
  }
  // Probes issued since creation.
  uint64_t probes() const {
    return static_cast<uint64_t>(next_id_);
  }
  bool enabled() const {
    return enabled_;
  }
  void setEnabled(bool on) {
    enabled_ = on;
  }
  // One line per key: "key n=<candidates> choice=<c> ms=<median per candidate>".
  std::string report();

private:
  struct Entry {
    int n = 0;
    int chosen = -1;
    int issued = 0;                      // probes issued
    std::vector<std::vector<float>> ms;  // completed probe times per candidate
  };
  struct Probe {
    long id;
    std::string key;
    int cand;
    cudaEvent_t b, e;
    bool closed;
  };
  bool enabled_;
  int exploring_ = 0;
  long next_id_ = 0;
  std::map<std::string, Entry> entries_;
  std::vector<Probe> pending_;
  std::vector<cudaEvent_t> pool_;

  cudaEvent_t event();
  void harvest(const std::string* wait_key);
  void decide(Entry& e);
};

// Tuning key: kernel family, bands, cluster size, extended frequencies, the order bound rounded up
// to a power of two (at least 128), sectors and element size.
inline std::string tuneKey(const char* family, int nb, int nc, int nw_ext, int n_max, int n_sectors, int elem) {
  int nb2 = 128;
  while (nb2 < n_max)
    nb2 *= 2;
  return std::string(family) + "|nb" + std::to_string(nb) + "|nc" + std::to_string(nc) + "|nwe" +
         std::to_string(nw_ext) + "|n" + std::to_string(nb2) + "|sec" + std::to_string(n_sectors) + "|e" +
         std::to_string(elem);
}

// Helpers for launch sites that may run without a tuner (null: candidate 0, no probe).
inline LaunchTuner::Pick tunePick(LaunchTuner* t, const std::string& key, int n, cudaStream_t s) {
  return t ? t->pick(key, n, s) : LaunchTuner::Pick{};
}
inline void tuneEnd(LaunchTuner* t, const LaunchTuner::Pick& p, cudaStream_t s) {
  if (t)
    t->end(p, s);
}

}  // namespace dcaacc
