// Fused segment backend: generates one persistent CUDA kernel per segment
// DAG, compiles it at run time for sm_100a with NVRTC (cached by DAG text),
// and launches it.  See fused.cpp for the kernel design.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace bsz {

class FusedBackend {
 public:
  FusedBackend(Device& dev, const ExecOptions& opt);
  ~FusedBackend();
  // Computes seg.order; materializes seg.outputs into nodes[i].buf and adds
  // the popcounts of seg.pops into d_slots[slot].
  void run(std::vector<Node>& nodes, const Segment& seg, int64_t N, int64_t nw,
           unsigned long long* d_slots, double* compile_ms);

  int64_t fallbacks = 0;   // parts re-run with the plain kernels (speculation unproven)
  int64_t launches = 0;    // fused kernels launched

  struct Impl;

 private:
  std::unique_ptr<Impl> impl_;
};

}  // namespace bsz
