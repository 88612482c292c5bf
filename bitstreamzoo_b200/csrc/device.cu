// Device context: stream, buffer cache, scratch, error word.
#include "device.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

namespace bsz {

DevStream::~DevStream() {
  if (dev && p) dev->release(this);
}

Device::Device(int ordinal) : ordinal_(ordinal) {
  BSZ_CUDA(cudaSetDevice(ordinal));
  cudaDeviceProp prop;
  BSZ_CUDA(cudaGetDeviceProperties(&prop, ordinal));
  if (prop.major < 10)
    throw CudaError("bitstreamzoo_b200 needs an sm_100 (Blackwell B200) device; device " +
                    std::to_string(ordinal) + " is " + prop.name);
  sm_count_ = prop.multiProcessorCount;
  BSZ_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  BSZ_CUDA(cudaMalloc(&d_err_, 256));
  ++n_mallocs;
  BSZ_CUDA(cudaMemsetAsync(d_err_, 0, 256, stream_));
}

Device::~Device() {
  cudaSetDevice(ordinal_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& kv : all_) cudaFree(kv.first);
  if (d_scan_) cudaFree(d_scan_);
  if (d_err_) cudaFree(d_err_);
  if (d_scratch_) cudaFree(d_scratch_);
  for (auto& kv : *pinned_free_) cudaFreeHost(kv.second);
  pinned_free_->clear();
  for (int k = 0; k < 2; ++k) {
    if (pin_[k]) cudaFreeHost(pin_[k]);
    if (pin_ev_[k]) cudaEventDestroy(pin_ev_[k]);
  }
  if (stream_) cudaStreamDestroy(stream_);
}

std::shared_ptr<void> Device::pinned_block(size_t bytes) {
  bytes = std::max<size_t>(4096, (bytes + 4095) / 4096 * 4096);
  void* p = nullptr;
  size_t have = bytes;
  auto it = pinned_free_->lower_bound(bytes);
  if (it != pinned_free_->end() && it->first <= 4 * bytes) {
    have = it->first;
    p = it->second;
    pinned_free_->erase(it);
  } else {
    BSZ_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocDefault));
  }
  // the cache outlives the Device only through blocks still referenced:
  // those are freed directly when the Device is gone
  std::weak_ptr<std::multimap<size_t, void*>> pool = pinned_free_;
  return std::shared_ptr<void>(p, [pool, have](void* q) {
    if (auto m = pool.lock()) m->emplace(have, q);
    else cudaFreeHost(q);
  });
}

namespace {

constexpr size_t kStageBytes = size_t(32) << 20;
constexpr size_t kDirectBytes = size_t(1) << 20;

// memcpy split across host threads for large chunks.
void parallel_memcpy(void* dst, const void* src, size_t n) {
  const size_t kMinPerThread = size_t(4) << 20;
  unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  size_t nt = std::min<size_t>({static_cast<size_t>(hw), size_t(8), n / kMinPerThread});
  if (nt <= 1) {
    std::memcpy(dst, src, n);
    return;
  }
  std::vector<std::thread> th;
  const size_t per = (n + nt - 1) / nt;
  for (size_t t = 0; t < nt; ++t) {
    const size_t off = t * per;
    if (off >= n) break;
    const size_t len = std::min(per, n - off);
    th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len); });
  }
  for (auto& t : th) t.join();
}

}  // namespace

void Device::ensure_pinned() {
  if (pin_[0]) return;
  for (int k = 0; k < 2; ++k) {
    BSZ_CUDA(cudaHostAlloc(&pin_[k], kStageBytes, cudaHostAllocDefault));
    BSZ_CUDA(cudaEventCreateWithFlags(&pin_ev_[k], cudaEventDisableTiming));
    BSZ_CUDA(cudaEventRecord(pin_ev_[k], stream_));
  }
}

void Device::h2d(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  if (bytes <= kDirectBytes) {
    BSZ_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_));
    return;
  }
  ensure_pinned();
  int k = 0;
  for (size_t off = 0; off < bytes; off += kStageBytes, k ^= 1) {
    const size_t len = std::min(kStageBytes, bytes - off);
    BSZ_CUDA(cudaEventSynchronize(pin_ev_[k]));   // its previous DMA is done
    parallel_memcpy(pin_[k], static_cast<const char*>(src) + off, len);
    BSZ_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, pin_[k], len, cudaMemcpyHostToDevice, stream_));
    BSZ_CUDA(cudaEventRecord(pin_ev_[k], stream_));
  }
}

void Device::d2h(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  if (bytes <= kDirectBytes) {
    BSZ_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_));
    BSZ_CUDA(cudaStreamSynchronize(stream_));
    return;
  }
  ensure_pinned();
  // chunk i DMAs into pin_[i & 1]; the host copies chunk i-1 out meanwhile
  size_t prev_off = 0, prev_len = 0;
  int k = 0;
  for (size_t off = 0; off < bytes; off += kStageBytes, k ^= 1) {
    const size_t len = std::min(kStageBytes, bytes - off);
    BSZ_CUDA(cudaEventSynchronize(pin_ev_[k]));
    BSZ_CUDA(cudaMemcpyAsync(pin_[k], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, stream_));
    BSZ_CUDA(cudaEventRecord(pin_ev_[k], stream_));
    if (prev_len) {
      BSZ_CUDA(cudaEventSynchronize(pin_ev_[k ^ 1]));
      parallel_memcpy(static_cast<char*>(dst) + prev_off, pin_[k ^ 1], prev_len);
    }
    prev_off = off;
    prev_len = len;
  }
  BSZ_CUDA(cudaEventSynchronize(pin_ev_[k ^ 1]));
  parallel_memcpy(static_cast<char*>(dst) + prev_off, pin_[k ^ 1], prev_len);
}

void* Device::raw_alloc(size_t bytes) {
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    trim_cache();
    e = cudaMalloc(&p, bytes);
  }
  if (e != cudaSuccess)
    throw CudaError(std::string("cudaMalloc(") + std::to_string(bytes) +
                    ") failed: " + cudaGetErrorString(e) +
                    (e == cudaErrorMemoryAllocation ? " (out of memory)" : ""));
  ++n_mallocs;
  all_.push_back({p, bytes});
  return p;
}

BufRef Device::alloc_stream(int64_t n_words) {
  // Round to 256 bytes so vector loops may run over whole 16-byte pairs.
  size_t bytes = (static_cast<size_t>(std::max<int64_t>(n_words, 1)) * 8 + 255) & ~size_t(255);
  void* p = nullptr;
  auto it = free_.find(bytes);
  if (it != free_.end()) {
    p = it->second;
    free_.erase(it);
  } else {
    p = raw_alloc(bytes);
  }
  auto s = std::make_shared<DevStream>();
  s->p = static_cast<uint64_t*>(p);
  s->n_words = n_words;
  s->bytes = bytes;
  s->dev = this;
  bytes_live += static_cast<int64_t>(bytes);
  bytes_peak = std::max(bytes_peak, bytes_live);
  return s;
}

void Device::release(DevStream* s) {
  free_.emplace(s->bytes, s->p);
  bytes_live -= static_cast<int64_t>(s->bytes);
  s->p = nullptr;
}

void Device::trim_cache() {
  cudaStreamSynchronize(stream_);
  for (auto& kv : free_) {
    cudaFree(kv.second);
    all_.erase(std::remove_if(all_.begin(), all_.end(),
                              [&](const std::pair<void*, size_t>& a) { return a.first == kv.second; }),
               all_.end());
  }
  free_.clear();
}

uint32_t* Device::scan_state(int64_t n_u32) {
  if (n_u32 > scan_cap_) {
    if (d_scan_) {
      BSZ_CUDA(cudaStreamSynchronize(stream_));
      BSZ_CUDA(cudaFree(d_scan_));
    }
    int64_t cap = std::max<int64_t>(n_u32, 4096);
    BSZ_CUDA(cudaMalloc(&d_scan_, static_cast<size_t>(cap) * 4));
    ++n_mallocs;
    scan_cap_ = cap;
  }
  BSZ_CUDA(cudaMemsetAsync(d_scan_, 0, static_cast<size_t>(n_u32) * 4, stream_));
  return d_scan_;
}

void* Device::scratch(size_t bytes) {
  if (bytes > scratch_cap_) {
    if (d_scratch_) {
      BSZ_CUDA(cudaStreamSynchronize(stream_));
      BSZ_CUDA(cudaFree(d_scratch_));
    }
    size_t cap = std::max<size_t>(bytes, 1 << 16);
    BSZ_CUDA(cudaMalloc(&d_scratch_, cap));
    ++n_mallocs;
    scratch_cap_ = cap;
  }
  return d_scratch_;
}

uint32_t Device::take_error() {
  uint32_t h = 0;
  BSZ_CUDA(cudaMemcpyAsync(&h, d_err_, 4, cudaMemcpyDeviceToHost, stream_));
  BSZ_CUDA(cudaStreamSynchronize(stream_));
  if (h) BSZ_CUDA(cudaMemsetAsync(d_err_, 0, 4, stream_));
  return h;
}

void Device::sync() {
  BSZ_CUDA(cudaStreamSynchronize(stream_));
  BSZ_CUDA(cudaGetLastError());
}

cudaEvent_t Device::prof_event() {
  if (!prof_pool_.empty()) {
    cudaEvent_t e = prof_pool_.back();
    prof_pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  BSZ_CUDA(cudaEventCreate(&e));
  return e;
}

cudaEvent_t Device::prof_begin() {
  cudaEvent_t e = prof_event();
  BSZ_CUDA(cudaEventRecord(e, stream_));
  return e;
}

void Device::prof_end(const char* name, cudaEvent_t begin) {
  cudaEvent_t e = prof_event();
  BSZ_CUDA(cudaEventRecord(e, stream_));
  prof_pending_.push_back({name, begin, e});
  if (prof_pending_.size() > 4096) prof_report();   // resolve in batches
}

std::string Device::prof_report() {
  BSZ_CUDA(cudaStreamSynchronize(stream_));
  for (auto& r : prof_pending_) {
    float ms = 0;
    cudaEventElapsedTime(&ms, r.a, r.b);
    auto& t = prof_totals_[r.name];
    t.first += 1;
    t.second += ms;
    prof_pool_.push_back(r.a);
    prof_pool_.push_back(r.b);
  }
  prof_pending_.clear();
  std::string js = "{";
  bool first = true;
  for (auto& kv : prof_totals_) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s\"%s\":{\"launches\":%lld,\"ms\":%.6f}", first ? "" : ",",
                  kv.first.c_str(), static_cast<long long>(kv.second.first), kv.second.second);
    js += buf;
    first = false;
  }
  return js + "}";
}

void Device::prof_reset() {
  prof_report();
  prof_totals_.clear();
}

}  // namespace bsz
