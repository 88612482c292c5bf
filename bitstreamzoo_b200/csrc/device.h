// Device runtime: one CUDA stream per context, a size-keyed cache of stream
// buffers (no cudaMalloc/cudaFree on the steady-state path), popcount slots,
// look-back scratch for the carry scan, and a device error word that bounded
// spin-waits write instead of hanging.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace bsz {

struct CudaError : std::runtime_error { using std::runtime_error::runtime_error; };

#define BSZ_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw ::bsz::CudaError(std::string(#call) + " failed: " + cudaGetErrorString(e_) + \
                             (e_ == cudaErrorMemoryAllocation ? " (out of memory)" : "")); \
  } while (0)

// Device error word bits (set by kernels, read by the host after a sync).
enum : uint32_t {
  kErrLookbackTimeout = 1u << 0,   // a carry look-back spin hit its limit
  kErrFusedTimeout = 1u << 1,      // a fused-kernel boundary wait hit its limit
  kErrFusedOverflow = 1u << 2,     // fused kernel: halo/state capacity exceeded
};

// Human-readable text of a nonzero device error word.
inline std::string describe_device_error(uint32_t e) {
  std::string s = "device error word " + std::to_string(e) + ":";
  if (e & kErrLookbackTimeout) s += " carry look-back timed out;";
  if (e & kErrFusedTimeout) s += " fused-kernel wait timed out;";
  if (e & kErrFusedOverflow) s += " fused-kernel state capacity exceeded;";
  s.pop_back();
  return s;
}

class Device;

// A device stream buffer of n_words uint64 words (256-byte aligned).  Freed
// back into the owning Device's cache; the memory is reused in stream order.
struct DevStream {
  uint64_t* p = nullptr;
  int64_t n_words = 0;
  size_t bytes = 0;
  Device* dev = nullptr;
  DevStream() = default;
  DevStream(const DevStream&) = delete;
  DevStream& operator=(const DevStream&) = delete;
  ~DevStream();
};
using BufRef = std::shared_ptr<DevStream>;

class Device {
 public:
  explicit Device(int ordinal);
  ~Device();
  Device(const Device&) = delete;
  Device& operator=(const Device&) = delete;

  int ordinal() const { return ordinal_; }
  cudaStream_t stream() const { return stream_; }
  int sm_count() const { return sm_count_; }

  BufRef alloc_stream(int64_t n_words);
  void release(DevStream* s);
  void trim_cache();

  // Look-back scratch: >= n_words_needed uint32 words, zeroed on the stream.
  uint32_t* scan_state(int64_t n_u32);
  uint32_t* error_word() const { return d_err_; }
  // Copies the error word to the host (synchronizes the stream) and clears it.
  uint32_t take_error();
  void sync();

  // Counters reported in the bsim_cuda JSON.
  int64_t n_launches = 0;
  int64_t n_mallocs = 0;
  int64_t bytes_live = 0;
  int64_t bytes_peak = 0;


  // Untyped device scratch (cached; grows).
  void* scratch(size_t bytes);

  // A pinned host block of at least `bytes` for asynchronous read-backs,
  // from a cache (cudaHostAlloc only when none fits); it returns to the
  // cache when the last reference goes.
  std::shared_ptr<void> pinned_block(size_t bytes);

  // Copies between pageable host memory and the device through two pinned
  // staging buffers: chunks are double-buffered (the host memcpy of one
  // chunk, split across threads, overlaps the DMA of the other), so large
  // transfers run at link speed instead of the driver's pageable path.
  // h2d returns once `src` may be reused (the last DMA may still be in
  // flight on the stream); d2h returns with `dst` filled.  Small copies go
  // straight to cudaMemcpyAsync.
  void h2d(void* dst, const void* src, size_t bytes);
  void d2h(void* dst, const void* src, size_t bytes);

  // Per-kernel CUDA-event timing on this device's stream (off by default).
  bool profiling = false;
  cudaEvent_t prof_begin();
  void prof_end(const char* name, cudaEvent_t begin);
  std::string prof_report();   // synchronizes; JSON {name: {launches, ms}}
  void prof_reset();

 private:
  int ordinal_;
  int sm_count_ = 148;
  cudaStream_t stream_ = nullptr;
  std::multimap<size_t, void*> free_;   // bytes -> cached block
  std::vector<std::pair<void*, size_t>> all_;
  uint32_t* d_scan_ = nullptr;
  int64_t scan_cap_ = 0;
  uint32_t* d_err_ = nullptr;
  void* d_scratch_ = nullptr;
  size_t scratch_cap_ = 0;
  void* pin_[2] = {nullptr, nullptr};
  std::shared_ptr<std::multimap<size_t, void*>> pinned_free_ = std::make_shared<std::multimap<size_t, void*>>();
  cudaEvent_t pin_ev_[2] = {nullptr, nullptr};
  void ensure_pinned();
  void* raw_alloc(size_t bytes);
  struct ProfRec { const char* name; cudaEvent_t a, b; };
  std::vector<ProfRec> prof_pending_;
  std::vector<cudaEvent_t> prof_pool_;
  std::map<std::string, std::pair<int64_t, double>> prof_totals_;
  cudaEvent_t prof_event();
};

// Records CUDA events around one launch when the device is profiling.
struct ProfScope {
  Device& d;
  const char* name;
  cudaEvent_t a = nullptr;
  ProfScope(Device& dev, const char* n) : d(dev), name(n) {
    if (d.profiling) a = d.prof_begin();
  }
  ~ProfScope() {
    if (a) d.prof_end(name, a);
  }
};

// ---------------------------------------------------------------------------
// Plain per-op kernels (kernels.cu).  All launch asynchronously on
// dev.stream().  ``last_mask`` clears the bits at and above the bitlength in
// the last word, as the normative semantics mask ~, + and <<.
// Pointer arguments must be 16-byte aligned for the vector path; unaligned
// pointers take a scalar path.
enum BitOp : int { kAnd = 0, kOr = 1, kXor = 2, kAndNot = 3 };

void launch_bitwise(Device& dev, int op, uint64_t* d, const uint64_t* a, const uint64_t* b,
                    int64_t n);
void launch_not(Device& dev, uint64_t* d, const uint64_t* a, int64_t n, uint64_t last_mask);
void launch_shl(Device& dev, uint64_t* d, const uint64_t* a, int64_t k, int64_t n,
                uint64_t last_mask);
void launch_shr(Device& dev, uint64_t* d, const uint64_t* a, int64_t k, int64_t n,
                uint64_t fill);
void launch_add(Device& dev, uint64_t* d, const uint64_t* a, const uint64_t* b, int64_t n,
                uint64_t last_mask);
// Same carry scan with caller-provided look-back state: ``state`` must hold
// add_state_words(n) zeroed uint32 words.
void launch_add_with_state(Device& dev, uint64_t* d, const uint64_t* a, const uint64_t* b,
                           int64_t n, uint64_t last_mask, uint32_t* state);
int64_t add_state_words(int64_t n);
// The same carry-scan kernel on a caller's stream with caller-provided
// look-back state (add_state_words(n) zeroed words) and error word.
void launch_add_on_stream(cudaStream_t stream, uint64_t* d, const uint64_t* a, const uint64_t* b,
                          int64_t n, uint64_t last_mask, uint32_t* state, uint32_t* err);
// Test hook of the add kernel's look-back: tile `silent_tile` never publishes
// its status and every wait gives up after `spin_limit` spins (<= 0: the
// default limit).  silent_tile = -1 turns the hook off.
void set_add_lookback_test_hook(int64_t silent_tile, int spin_limit);
void launch_popcount(Device& dev, const uint64_t* a, int64_t n,
                     unsigned long long* slot);
void launch_any(Device& dev, const uint64_t* a, int64_t n, unsigned int* flag);
void launch_fill(Device& dev, uint64_t* d, int64_t n, uint64_t value, uint64_t last_value);
void launch_copy(Device& dev, uint64_t* d, const uint64_t* a, int64_t n);
// Byte -> basis bits (s2p.cu): out[i] (ceil(n_bytes/64) words each) gets bit i
// of every byte.
void launch_s2p(Device& dev, const uint8_t* bytes, int64_t n_bytes, uint64_t* const* out);

inline uint64_t mask_for_bits(int64_t nbits) {
  int r = static_cast<int>(nbits & 63);
  return r ? ((uint64_t(1) << r) - 1) : ~uint64_t(0);
}

}  // namespace bsz
