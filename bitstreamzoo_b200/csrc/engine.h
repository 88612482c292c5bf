// Executor: walks the program on the host and lowers stream statements into
// an op DAG that runs on the GPU in segments.
//
// Replaces the reference's statement-at-a-time Interpreter<CudaBackend>
// (simulator/csim/src/interpreter.inl:93-364), which launches one or more
// kernels per DSL op and synchronizes for every popcount and condition.
// Here stream values are DAG nodes; nothing runs until a value is needed on
// the host (an if/while condition, a popcount that feeds a loop bound, shift
// amount or array index, or the end of the program).  At that point the
// pending DAG (after dead-code elimination against the live variables) is
// executed as one segment, either
//   * plain: one kernel per DSL operation, or
//   * fused: one generated persistent kernel for the whole segment.
// Popcounts are accumulated into device slots and read back once.
//
// Semantics are the normative Python ones (simulator/pythonsim/interpreter.py):
// a stream is n = ceil(N/64) stored words plus a "tail" bit that every bit past
// the stored words equals (Python's negative integers).  ~, + and << clear the
// bits at and above N; & | ^ >> do not; ONES is the N-bit mask as an operand
// but all-ones with tail 1 when copied; popcount of a value whose tail is 1 is
// an error.  Tails never depend on data, so they are tracked on the host.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "device.h"
#include "frontend.h"

namespace bsz {

struct RuntimeError : std::runtime_error { using std::runtime_error::runtime_error; };

enum class NOp : uint8_t { Buf, Zero, OnesMask, AllOnes, Not, And, Or, Xor, AndNot, Add, Shl, Shr };

struct Node {
  NOp op = NOp::Zero;
  int32_t a = -1, b = -1;
  int64_t k = 0;          // shift amount
  uint8_t tail = 0;       // bits past the stored words (0 or 1)
  uint8_t clean = 0;      // known: stored bits at/above N are zero and tail is 0
  BufRef buf;             // Buf nodes, and computed nodes once materialized
};

// Plain: one kernel per operation.  Fused: generated segment kernels
// (NVRTC).  Vm: each segment is one launch of the device interpreter
// (vm.cu).  Auto: the VM for short streams; for long ones fused kernels when
// they are cached or the segment's per-op time would exceed their compile
// time, else per-op kernels.
enum class ExecMode : int { Plain = 0, Fused = 1, Auto = 2, Vm = 3 };

// Fused-kernel schedule: the knobs the autotuner and the cost model choose.
struct Schedule {
  int warps = 4;          // warps per CTA
  int range_steps = 64;   // minimum 32-word steps per warp range (words per tile / 32)
  int ctas_per_sm = 0;    // resident CTAs per SM; 0 = as many as the kernel's occupancy allows; -1 = no cap (one minimum-length range per warp)
  int min_blocks = 4;     // __launch_bounds__ minimum blocks (caps registers per thread)
  int prefetch = 1;       // issue the next step's loads before the current step's arithmetic
  int cut_adds = 0;       // carry scheme: 0, additions inside the generated kernels (speculative
                          // carry state); 1, the same with every addition's result materialized;
                          // 2, every addition run by the plain carry-scan kernel (decoupled
                          // look-back) on materialized operands
  int layout = 0;         // 0: warp ranges, lane = word; 1: thread-sequential ranges
                          // (register chunks); 2: thread-sequential ranges through TMA boxes
  int chunk_words = 4;    // layouts 1, 2: words per thread per chunk / box (4 or 8)
  int stages = 2;         // layout 2: shared-memory stages of input boxes (2 or 3)
  int unroll = 0;         // layout 2: 1 = each chunk's word pairs unrolled
  int shift_mul = 0;      // layouts 1-2: 1 = shifts by multiply-adds (integer FMA pipe)
};

struct ExecOptions {
  ExecMode mode = ExecMode::Plain;
  bool simplify = false;        // algebraic folding + CSE (on in fused mode)
  Schedule sched;
};

// A segment handed to the plain or fused backend: nodes in topological order.
struct Segment {
  std::vector<int> order;                     // computed nodes, topological
  std::vector<int> inputs;                    // Buf / constant nodes read
  std::vector<int> outputs;                   // nodes to materialize
  std::vector<std::pair<int, int64_t>> pops;  // (node, slot index)
};

class FusedBackend;

class Executor {
 public:
  Executor(Device& dev, const Program& prog, int64_t bitlength, ExecOptions opt);
  ~Executor();

  int64_t bitlength() const { return N_; }
  int64_t n_words() const { return nw_; }

  void set_param(int name, int64_t v);
  void bind_input(int name, BufRef buf, uint8_t tail, bool clean);
  void bind_input_array(int name, int64_t idx, BufRef buf, uint8_t tail, bool clean);
  void bind_broadcast(int name, const std::vector<uint8_t>& ones);   // element i: 1 = -1

  // Walks the program and enqueues its device work.  With finish = false it
  // returns without waiting for the device (no host read-back at the end):
  // call finish() before reading results.
  void run(bool finish = true);
  // Waits for the enqueued work, re-runs any fused part whose speculation
  // was unproven, reads the popcount slots and checks the device error word.
  void finish();

  // Results (valid after run()).
  bool has_stream(int name) const;
  BufRef stream_value(int name);                 // materialized buffer
  uint8_t stream_tail(int name) const;
  std::vector<int64_t> array_indices(int name) const;   // sorted; empty if absent
  BufRef array_value(int name, int64_t idx);
  bool has_array(int name) const;
  bool int_value(int name, int64_t* v);

  int64_t op_count = 0;
  std::map<std::string, int64_t> op_mix;
  int64_t n_segments = 0;
  int64_t n_syncs = 0;
  int64_t max_live_buffers = 0;
  double compile_ms = 0.0;
  int64_t vm_launches = 0;
  bool ran_as_vm_program = false;
  bool walk_replayed = false;     // the walk came from the program's walk cache
  // Host time split of flushes (ms): building segments, choosing the form,
  // running them (launch + host work; device time overlaps), compacting.
  // Printed to stderr at destruction when $BSZ_HOST_TIMES is set.
  double t_segment_ms = 0, t_policy_ms = 0, t_run_ms = 0, t_compact_ms = 0;
  int64_t fused_launches() const;
  int64_t fused_fallbacks() const;
  void set_schedule(const Schedule& s);

  // ---- batch support ----------------------------------------------------
  // A straight-line program traced symbolically: its DAG from the declared
  // scalar inputs to the declared scalar outputs and popcounts, independent
  // of the stream length.  Integer outputs are postfix programs over the
  // popcount slots: ('k', value) constant, ('s', slot), '+', '-', '*'.
  struct Traced {
    std::vector<Node> nodes;
    std::vector<int> input_nodes;    // per scalar input of the program
    std::vector<int> output_nodes;   // per scalar output stream (-1: never assigned)
    std::vector<std::pair<int, int64_t>> pops;   // (node, slot 0..n-1)
    std::vector<std::vector<std::pair<char, int64_t>>> int_outputs;   // per output int
    int64_t op_count = 0;
  };
  // Walks the program with unbound symbolic inputs.  Throws if the program
  // needs the device during the walk (if/while on a stream, an int from a
  // popcount used as a loop bound, index or shift amount, arrays).
  Traced trace();

 private:
  struct IntV { int64_t v = 0; int32_t e = -1; };
  struct IE { char op; int32_t a, b; int64_t v; };
  struct Arr {
    bool defined = false;
    bool broadcast = false;
    std::vector<uint8_t> bcast;
    int64_t decl_size = 0;          // indices [0, decl_size) exist (zero unless written)
    std::map<int64_t, int> elems;   // index -> node
  };

  Device& dev_;
  const Program& prog_;
  int64_t N_, nw_;
  uint64_t last_mask_;
  ExecOptions opt_;

  std::vector<Node> nodes_;
  std::unordered_map<uint64_t, int> cse_;
  int zero_ = -1, ones_mask_ = -1, all_ones_ = -1;
  BufRef c_zero_, c_mask_, c_all_;

  std::vector<int> var_;          // name -> node (-1 undefined, -2 dropped as dead)
  std::vector<IntV> ints_;
  std::vector<uint8_t> int_def_;
  std::vector<std::unique_ptr<Arr>> arrs_;
  std::vector<IE> iexpr_;

  // popcount slots
  unsigned long long* d_slots_ = nullptr;
  BufRef slots_buf_;              // device buffers below come from the device's buffer
  BufRef flag_buf_;               // cache, so a run makes no cudaMalloc/cudaFree (each
  BufRef vm_mem_;                 // cudaFree would synchronize the whole device)
  int64_t slot_cap_ = 0, slot_base_ = 0, n_slots_ = 0;
  std::vector<uint64_t> slot_val_;
  std::vector<std::pair<int, int64_t>> pending_pops_;
  int64_t resolved_upto_ = 0;

  // liveness: stream names live at each if/while statement and at the end
  // (computed once per program)
  struct Liveness {
    std::unordered_map<int, std::vector<uint64_t>> at;
    std::vector<uint64_t> end;
  };
  std::shared_ptr<const Liveness> live_;

  // Walk cache.  A run of a program without if/while whose walk needed no
  // flush is a deterministic function of the program, the bit length, the
  // mode and the bindings made before run() (names, tails, cleanliness,
  // parameters: bind_sig_).  Its result, the DAG and the walk's variable
  // state, is kept with the program, and a later run with the same key
  // restores it instead of walking the statements again.  The device work
  // (every kernel of the flush) runs on every run.
  struct WalkSnap;
  struct ExecCache;
  std::string bind_sig_;
  int64_t n_flushes_ = 0;
  bool finished_ = false;         // finish() completed: no device work of this run outstanding
  // Asynchronous run: the read-backs (popcount slots, fused speculation
  // flags, device error word) enqueued behind the run's work into a pinned
  // block, and an event after them; finish() waits on that event only, not
  // on whatever other runs enqueued since.
  std::shared_ptr<void> readback_;
  cudaEvent_t done_ev_ = nullptr;
  int64_t rb_slots_ = 0, rb_flags_ = 0;
  void enqueue_readback();
  ExecCache& exec_cache() const;
  std::string walk_key() const;
  bool replay_walk(const std::string& key);
  void save_walk(const std::string& key, size_t n0);

  std::unique_ptr<FusedBackend> fused_;
  unsigned int* d_flag_ = nullptr;
  void* vm_buf_ = nullptr;        // VM instruction list, pointer table and slot file
  size_t vm_cap_ = 0;
  size_t nodes_after_flush_ = 0;  // node count after the last compaction
  bool tracing_ = false;   // symbolic walk for batches: no device work, no length-dependent folds

  // walk
  void exec_block(const std::vector<Stmt>& v);
  void exec(const Stmt& s);
  int rhs(const SExpr& e);
  int operand(const SExpr& e);
  int elem(const SExpr& e);
  int read_var(int name);
  IntV ival(const IExpr& e);
  int64_t force(const IntV& x);
  int64_t eval_ie(int32_t e);
  bool nonzero(int node, const Stmt* at);
  IntV popcount(int node);
  void count(const char* op);
  void publish_op_mix();
  int64_t op_class_[8] = {0, 0, 0, 0, 0, 0, 0, 0};

  // graph
  int mk(NOp op, int a = -1, int b = -1, int64_t k = 0);
  int mk_raw(NOp op, int a, int b, int64_t k, uint8_t tail);
  int buf_node(BufRef buf, uint8_t tail, bool clean);
  bool pending(int node) const;
  void flush(const std::vector<uint64_t>* live, int* extra);
  void compact(int* extra);
  void run_plain(const Segment& seg);
  void run_vm(const Segment& seg);
  // Whole program, control flow included, as one device-interpreter launch
  // (vmprog.cpp).  Returns false, with no state changed, when the program
  // needs the host during its run (see vmprog.cpp for the conditions).
  bool run_vm_program();
  friend struct VmCompiler;
  bool fused_pays(const Segment& seg);
  const uint64_t* const_ptr(int node);
  void ensure_slots(int64_t need);
  void resolve_slots();
  std::shared_ptr<const Liveness> compute_liveness() const;
  int64_t live_buffer_count() const;
};

}  // namespace bsz
