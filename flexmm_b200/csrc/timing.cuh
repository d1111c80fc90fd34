// Optional per-kernel CUDA-event timing (the reference's `verbose` phase
// timers, flexmm/flexmm2d/fmm.py:24-30, 55-58, 106-107, 148-149, made
// per-kernel).  Disabled by default; when enabled every timed launch records
// an event pair on its own stream, read back by fmm_timing_read().
#pragma once
#include <mutex>
#include <vector>

#include "common.cuh"

namespace fmmb {

enum Phase : int {
  PH_TREE = 0,      // whole tree build (span, includes its two host waits)
  PH_SORT_TGT = 1,  // targets into leaves: keys, binning (KIFMM) or sort (BB, Stokes), items
  PH_UPWARD = 2,    // k_upward launches (S2M + M2M + C2E)
  PH_M2L = 3,       // k_m2l launch
  PH_DOWNWARD = 4,  // k_downward launches (L2L + C2E)
  PH_EVAL = 5,      // k_evaluate launch (L2T + P2P)
  PH_DIRECT = 6,    // direct sums
  PH_TREE_SPLITS = 7,   // tree: point keys, sort, initial splits (to the first host round trip)
  PH_TREE_BALANCE = 8,  // tree: 2:1 closure and X-list (to the second)
  PH_TREE_NODES = 9,    // tree: parent-box sort, node arrays, colleagues, interaction lists
  PH_PREP = 10,         // expansions: charge gather, buffers, per-node charge sums
  N_PHASES = 12
};

struct TimingRegistry {
  std::mutex mu;
  bool enabled = false;
  struct Rec {
    int phase;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  static TimingRegistry &get() {
    static TimingRegistry r;
    return r;
  }
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
};

// RAII scope: records a start event at construction and an end event at
// destruction on `stream`, if timing is enabled.
struct PhaseTimer {
  int phase;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  PhaseTimer(int ph, cudaStream_t stream) : phase(ph), s(stream) {
    auto &R = TimingRegistry::get();
    if (!R.enabled) return;
    std::lock_guard<std::mutex> g(R.mu);
    a = R.take();
    cudaEventRecord(a, s);
  }
  ~PhaseTimer() {
    if (!a) return;
    auto &R = TimingRegistry::get();
    std::lock_guard<std::mutex> g(R.mu);
    cudaEvent_t b = R.take();
    cudaEventRecord(b, s);
    R.recs.push_back({phase, a, b});
  }
};

}  // namespace fmmb
