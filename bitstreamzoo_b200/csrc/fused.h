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
  // the popcounts of seg.pops into d_slots[slot].  Asynchronous: the kernels
  // are enqueued with one speculation flag per part, and the segment stays
  // pending (its parts, node records and buffers held) until resolve().
  void run(std::vector<Node>& nodes, const Segment& seg, int64_t N, int64_t nw,
           unsigned long long* d_slots, double* compile_ms);
  // Waits for the pending segment, reads its parts' flags and re-runs every
  // part from the first unproven one on with the exact per-op kernels (a
  // later part may have read the unproven part's outputs).  Must be called
  // before anything reads the segment's outputs or popcounts or launches
  // work that depends on them; a no-op when nothing is pending.
  void resolve();
  bool pending() const;
  // Asynchronous form of resolve(): enqueue_flags copies the pending
  // segment's flags (pending_parts() words) to pinned host memory on the
  // stream; once that copy has completed, resolve_with(flags) re-runs what
  // is unproven and returns true if it re-ran anything.
  int64_t pending_parts() const;
  void enqueue_flags(uint32_t* host);
  bool resolve_with(const uint32_t* flags);

  void set_schedule(const Schedule& s);
  // True when every kernel `run` would launch for this segment is already
  // compiled (in this process or in the on-disk kernel cache).
  bool all_compiled(const std::vector<Node>& nodes, const Segment& seg, int64_t N);

  int64_t fallbacks = 0;   // parts re-run with the plain kernels (speculation unproven)
  int64_t launches = 0;    // fused kernels launched
  // Host time (ms) in run(): before each launch returns (split, kernel
  // lookup or generation, arguments, launch) and waiting for the kernel.
  double t_prelaunch_ms = 0, t_wait_ms = 0;

  struct Impl;

 private:
  std::unique_ptr<Impl> impl_;
};

// ---------------------------------------------------------------------------
// Batches: many independent instances (stream sets of different lengths) of
// several straight-line programs, executed by ONE persistent kernel that
// holds every program's DAG as a device function and pulls (instance, word
// range) work items from an atomic counter.  The launch (with the resets of
// its counters) is captured once in a CUDA graph and replayed.

struct BatchInstance {
  int program = 0;
  int64_t bitlength = 0;
  std::vector<const uint64_t*> inputs;   // device pointers, one per scalar input
  std::vector<uint64_t*> outputs;        // device pointers, one per scalar output (null: skip)
};

class BatchRunner {
 public:
  BatchRunner(Device& dev, const std::vector<const Program*>& progs,
              std::vector<BatchInstance> instances, const Schedule& sched);
  ~BatchRunner();
  void launch();   // asynchronous on the device's stream
  void finish();   // waits; re-runs per-op if speculation was unproven; reads popcounts
  const std::vector<int64_t>& ints(int64_t instance) const;
  int64_t op_count(int64_t instance) const;
  int64_t n_items() const;
  double compile_ms = 0.0;
  int64_t fallbacks = 0;
  int64_t launches = 0;

  struct Impl;

 private:
  std::unique_ptr<Impl> impl_;
};

}  // namespace bsz
