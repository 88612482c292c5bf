// Stream addition that allocates no device memory.
//
// Some callers cannot allocate GPU memory at the moment they call us: a
// serving process whose memory pool has reserved nearly all of HBM up front,
// a host application (a database, a stream processor) that hands its device
// buffers in through FFI and routes every allocation through its own
// allocator, or a latency-critical loop that cannot afford the implicit
// device-wide synchronisation of cudaMalloc/cudaFree.  For them this file
// provides bsz_add_noalloc(): the same single-pass carry-scan addition as
// bsz_op_add(), but its look-back scratch (one status word per 256-word
// tile, a tile ticket and an error word) lives in a fixed-size file-scope
// __device__ array instead of memory from cudaMalloc.  Every GPU that loads
// the library's device code holds this array (about 1 MiB) until the
// process exits.  The CUDA runtime loads that code on a device lazily, at the
// first kernel launch or symbol lookup there, and that load commits the
// array: it is the one device allocation this entry point causes, and it
// happens on its first call on each device.  A caller that must not allocate
// later makes that first call at start-up (a call with n_words = 0 does only
// the set-up), while allocation is still allowed and before any stream
// capture.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/bsz.h"
#include "device.h"

namespace bsz {
void set_last_error(const std::string& msg);
}

namespace {

// Largest stream: 2^26 words = 2^32 bits (512 MiB per operand).
constexpr int64_t kMaxWords = int64_t(1) << 26;
// Look-back state for kMaxWords: one ticket word + one status word per tile
// of 256 words (checked against the kernel's own sizing at set-up).
constexpr int64_t kStateWords = 1 + kMaxWords / 256;
// The error word sits after the state, on its own 256-byte line.
constexpr int64_t kErrOffset = ((kStateWords + 63) / 64) * 64;
constexpr int64_t kScratchWords = kErrOffset + 64;

static __device__ __align__(256) uint32_t g_add_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_add_scratch on the current device.  In host code the
// symbol names a host-side shadow, not device memory, so the address must
// come from cudaGetSymbolAddress, once per device, with that device current.
uint32_t* scratch_on_current_device() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    if (bsz::add_state_words(kMaxWords) > kStateWords)
      throw std::runtime_error("bsz_add_noalloc: scratch array smaller than the kernel needs");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_add_scratch);
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
  }
  return g_scratch_ptr[dev];
}

}  // namespace

extern "C" int bsz_add_noalloc(uint64_t* dst, const uint64_t* a, const uint64_t* b, uint64_t n_words,
                               int64_t bitlength, void* stream) {
  try {
    if (n_words == 0) {
      // set-up only: load this library's device code on the current device
      // (which commits the scratch array) and look up the array's address
      scratch_on_current_device();
      return 0;
    }
    if (n_words > static_cast<uint64_t>(kMaxWords))
      throw std::invalid_argument("bsz_add_noalloc: n_words = " + std::to_string(n_words) +
                                  " exceeds the maximum of " + std::to_string(kMaxWords) +
                                  " words (2^32 bits); use bsz_op_add for longer streams");
    if (bitlength < 0 || (bitlength > 0 && static_cast<uint64_t>(bitlength) > 64 * n_words))
      throw std::invalid_argument("bsz_add_noalloc: bitlength " + std::to_string(bitlength) +
                                  " outside [0, 64 * n_words] for n_words = " + std::to_string(n_words));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* scratch = scratch_on_current_device();
    const int64_t n = static_cast<int64_t>(n_words);
    // The array keeps the previous call's contents: clear the ticket, the
    // tile status words this call uses, and the error word.
    cudaError_t e = cudaMemsetAsync(scratch, 0, static_cast<size_t>(bsz::add_state_words(n)) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch + kErrOffset, 0, 4, s);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    bsz::launch_add_on_stream(s, dst, a, b, n, bsz::mask_for_bits(bitlength), scratch,
                              scratch + kErrOffset);
    uint32_t err = 0;
    e = cudaMemcpyAsync(&err, scratch + kErrOffset, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) throw std::runtime_error(std::string("bsz_add_noalloc: ") + cudaGetErrorString(e));
    if (err) throw std::runtime_error("bsz_add_noalloc: carry look-back timed out (device error word " +
                                      std::to_string(err) + ")");
    return 0;
  } catch (const std::exception& ex) {
    bsz::set_last_error(ex.what());
  } catch (...) {
    bsz::set_last_error("unknown error");
  }
  return 1;
}
