// Fused segment backend: one generated persistent kernel per segment DAG.
//
// Kernel design (sm_100a, HBM-bound integer work):
//  * The stream is split into contiguous word ranges, one per warp; a warp
//    walks its range in 32-word steps (lane = word), so every load and store
//    is a coalesced 256-byte warp access and only the segment's inputs and
//    outputs touch HBM.  Every DAG temporary lives in registers.
//  * Cross-word operators carry state from step to step inside the warp:
//      - x + y: the carries of a step are resolved with two ballots and one
//        32-bit add ((G|P) + G + carry_in); the carry out is warp-uniform;
//      - x << k of a temporary: the words below come from lane shuffles of
//        this step and the previous step's value;
//      - shifts of an input read the neighbouring words from memory.
//  * A warp's first step needs the state at the start of its range.  It is
//    obtained by speculation: the warp first processes H warm-up words before
//    its range from an all-zero state while tracking, per node, how far the
//    possibly-wrong ("dirty") prefix reaches (additions stop being dirty at
//    the first word whose sum is not all ones; shifts move the dirt by their
//    distance).  If the dirt has died out before the range starts the state
//    is exact; otherwise the warm-up is doubled (up to 8 times).  If it still
//    cannot be proven exact the kernel raises a flag and the host re-runs the
//    segment with the plain per-op kernels, which are exact by construction.
//  * Right shifts of temporaries and left shifts of temporaries by 2048 bits
//    or more need words the warp has not computed yet / no longer holds; the
//    segment is cut there: the operand is materialized by an earlier kernel.
//  * Popcounts accumulate per lane, reduce per warp, one atomic per warp.
// Kernels are compiled with NVRTC for sm_100a and cached by their source.
#include "fused.h"

#include <cuda.h>
#include <nvrtc.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <sstream>

namespace bsz {
namespace {

// Driver entry points are resolved at run time through the runtime API, so
// the library has no link-time dependency on libcuda (it loads on hosts
// without a driver, where only the front end is usable).
struct Driver {
  CUresult (*module_load_data)(CUmodule*, const void*) = nullptr;
  CUresult (*module_get_function)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*func_get_attribute)(int*, CUfunction_attribute, CUfunction) = nullptr;
  CUresult (*launch_kernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                            unsigned, CUstream, void**, void**) = nullptr;
  CUresult (*get_error_string)(CUresult, const char**) = nullptr;
};

template <class F>
void resolve(const char* name, F& fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
    throw CudaError(std::string("cannot resolve driver entry point ") + name);
  fn = reinterpret_cast<F>(p);
}

const Driver& drv() {
  static Driver d = [] {
    Driver x;
    resolve("cuModuleLoadData", x.module_load_data);
    resolve("cuModuleGetFunction", x.module_get_function);
    resolve("cuFuncGetAttribute", x.func_get_attribute);
    resolve("cuLaunchKernel", x.launch_kernel);
    resolve("cuGetErrorString", x.get_error_string);
    return x;
  }();
  return d;
}

#define BSZ_CU(call)                                                              \
  do {                                                                            \
    CUresult r_ = (call);                                                         \
    if (r_ != CUDA_SUCCESS) {                                                     \
      const char* s_ = nullptr;                                                   \
      drv().get_error_string(r_, &s_);                                            \
      throw CudaError(std::string(#call) + " failed: " + (s_ ? s_ : "?"));        \
    }                                                                             \
  } while (0)

constexpr int kMaxInputs = 1024;

struct Compiled {
  CUmodule mod = nullptr;
  CUfunction fn = nullptr;
  int n_regs = 0;
};

// Process-wide cache of compiled kernels keyed by generated source.
std::mutex g_cache_mu;
std::map<std::string, Compiled>& cache() {
  static std::map<std::string, Compiled> c;
  return c;
}

bool is_const(NOp op) { return op == NOp::Zero || op == NOp::OnesMask || op == NOp::AllOnes; }

}  // namespace

struct FusedBackend::Impl {
  Device& dev;
  ExecOptions opt;
  unsigned int* d_fail = nullptr;
  Impl(Device& d, const ExecOptions& o) : dev(d), opt(o) {
    BSZ_CUDA(cudaMalloc(&d_fail, 256));
    ++dev.n_mallocs;
  }
  ~Impl() {
    if (d_fail) cudaFree(d_fail);
  }
};

FusedBackend::FusedBackend(Device& dev, const ExecOptions& opt)
    : impl_(std::make_unique<Impl>(dev, opt)) {}
FusedBackend::~FusedBackend() = default;

namespace {

// One kernel's worth of the segment.
struct Part {
  std::vector<int> order;                     // computed nodes (topological)
  std::vector<int> inputs;                    // materialized nodes read (Buf or earlier part)
  std::vector<int> outputs;                   // nodes to store
  std::vector<std::pair<int, int64_t>> pops;  // (node, slot)
};

struct Gen {
  const std::vector<Node>& nodes;
  const Part& part;
  int64_t N;
  int warps;
  int min_blocks;
  bool masked;
  // derived
  std::map<int, int> in_idx;       // node -> input index
  std::map<int, int> out_idx;      // node -> output index
  std::set<int> in_part;           // computed in this part
  std::set<int> shl_src;           // temporaries shifted left (need previous-step value)
  std::map<int, int> shl_ws;       // max word shift per shl source temporary
  std::vector<uint8_t> dyn;        // node dirt must be tracked during warm-up
  std::map<int, int64_t> sdh;      // static dirt (words) for nodes without add ancestors
  int64_t warm = 64;               // warm-up words

  std::string v(int n) const { return "v" + std::to_string(n); }
  bool is_input(int n) const { return in_idx.count(n) != 0; }

  void analyze() {
    for (size_t i = 0; i < part.inputs.size(); ++i) in_idx[part.inputs[i]] = static_cast<int>(i);
    for (size_t i = 0; i < part.outputs.size(); ++i) out_idx[part.outputs[i]] = static_cast<int>(i);
    for (int n : part.order) in_part.insert(n);
    dyn.assign(nodes.size(), 0);
    int64_t max_static = 0;
    for (int n : part.order) {
      const Node& x = nodes[n];
      auto d = [&](int o) -> int64_t { return (o >= 0 && sdh.count(o)) ? sdh[o] : 0; };
      bool dy = false;
      for (int o : {x.a, x.b})
        if (o >= 0 && dyn[o]) dy = true;
      int64_t s = std::max(d(x.a), d(x.b));
      if (x.op == NOp::Add) dy = true;
      if (x.op == NOp::Shl && x.a >= 0 && in_part.count(x.a)) {
        int ws = static_cast<int>(x.k / 64);
        shl_src.insert(x.a);
        shl_ws[x.a] = std::max(shl_ws[x.a], ws);
        s = d(x.a) + ws + ((x.k % 64) ? 1 : 0);
      }
      dyn[n] = dy;
      if (!dy) {
        sdh[n] = s;
        max_static = std::max(max_static, s);
      }
    }
    warm = ((max_static + 64 + 31) / 32) * 32;
    if (warm > 8192) warm = 8192;
  }

  // expression for an input node value at word index expression `idx`
  std::string load(int n, const std::string& idx) const {
    const Node& x = nodes[n];
    if (x.op == NOp::Zero) return "0ull";
    if (x.op == NOp::AllOnes) return "~0ull";
    if (x.op == NOp::OnesMask)
      return "((" + idx + ") < A.nw - 1 ? ~0ull : ((" + idx + ") == A.nw - 1 ? A.last_mask : 0ull))";
    std::string fill = x.tail ? "~0ull" : "0ull";
    return "((" + idx + ") >= 0 && (" + idx + ") < A.nw ? __ldg(A.in[" + std::to_string(in_idx.at(n)) +
           "] + (" + idx + ")) : " + fill + ")";
  }

  // value of operand o in the current step (already computed or loaded)
  std::string opnd(int o) const { return v(o); }

  void emit_step(std::ostringstream& s, bool track) const {
    s << "      const long long w = base + lane;\n";
    if (masked) s << "      const u64 lm = (w == A.nw - 1) ? A.last_mask : ~0ull;\n";
    // loads of unshifted inputs
    for (auto& kv : in_idx) {
      int n = kv.first;
      s << "      const u64 " << v(n) << " = " << load(n, "w") << ";\n";
    }
    if (track) s << "      const int rel = (int)(base - p0);\n";
    for (int n : part.order) {
      const Node& x = nodes[n];
      const std::string a = x.a >= 0 ? opnd(x.a) : "", b = x.b >= 0 ? opnd(x.b) : "";
      switch (x.op) {
        case NOp::Not:
          s << "      u64 " << v(n) << " = ~" << a << ";\n";
          break;
        case NOp::And: s << "      const u64 " << v(n) << " = " << a << " & " << b << ";\n"; break;
        case NOp::Or: s << "      const u64 " << v(n) << " = " << a << " | " << b << ";\n"; break;
        case NOp::Xor: s << "      const u64 " << v(n) << " = " << a << " ^ " << b << ";\n"; break;
        case NOp::AndNot:
          s << "      u64 " << v(n) << " = " << a << " & ~" << b << ";\n";
          break;
        case NOp::Add: {
          std::string c = "c" + std::to_string(n);
          s << "      u64 " << v(n) << ";\n      {\n"
            << "        const u64 sa = " << a << " + " << b << ";\n"
            << "        const u32 G = __ballot_sync(~0u, sa < " << a << ");\n"
            << "        const u32 P = __ballot_sync(~0u, sa == ~0ull);\n";
          if (track && dyn[n]) {
            s << "        if (!res" << n << ") {\n"
              << "          const int d0 = max(" << dh(x.a) << ", " << dh(x.b) << ") - rel;\n"
              << "          if (d0 < 32) {\n"
              << "            const u32 cand = ~P & (d0 <= 0 ? ~0u : (~0u << d0));\n"
              << "            if (cand) { res" << n << " = 1; dh" << n << " = rel + __ffs(cand); }\n"
              << "          }\n"
              << "        }\n";
          }
          s << "        const unsigned long long z = (unsigned long long)(G | P) + G + " << c << ";\n"
            << "        const u32 cv = (u32)z ^ P;\n"
            << "        " << c << " = (u32)(z >> 32);\n"
            << "        " << v(n) << " = sa + ((cv >> lane) & 1u)" << (masked ? " & lm" : "") << ";\n"
            << "      }\n";
          break;
        }
        case NOp::Shl: {
          int64_t ws = x.k / 64;
          int bs = static_cast<int>(x.k % 64);
          if (is_input(x.a) || is_const(nodes[x.a].op)) {
            s << "      u64 " << v(n) << ";\n      {\n"
              << "        const u64 lo = " << load(x.a, "w - " + std::to_string(ws) + "ll") << ";\n";
            if (bs) {
              s << "        u64 hi = __shfl_up_sync(~0u, lo, 1);\n"
                << "        if (lane == 0) hi = " << load(x.a, "base - " + std::to_string(ws + 1) + "ll")
                << ";\n"
                << "        " << v(n) << " = (lo << " << bs << ") | (hi >> " << (64 - bs) << ");\n";
            } else {
              s << "        " << v(n) << " = lo;\n";
            }
            s << "      }\n";
          } else {
            // temporary: words w-ws and w-ws-1 from this step and the previous one
            const std::string cur = opnd(x.a), prev = "pv" + std::to_string(x.a);
            s << "      u64 " << v(n) << ";\n      {\n";
            // shuffles must be executed by all lanes: compute both sources unconditionally
            auto emit_word = [&](const std::string& var, int64_t off) {
              if (off == 0) { s << "        const u64 " << var << " = " << cur << ";\n"; return; }
              if (off == 32) { s << "        const u64 " << var << " = " << prev << ";\n"; return; }
              std::string o = std::to_string(off);
              s << "        const u64 " << var << "_c = __shfl_up_sync(~0u, " << cur << ", " << o << ");\n"
                << "        const u64 " << var << "_p = __shfl_down_sync(~0u, " << prev << ", "
                << (32 - off) << ");\n"
                << "        const u64 " << var << " = lane >= " << o << " ? " << var << "_c : " << var
                << "_p;\n";
            };
            emit_word("lo", ws);
            if (bs) {
              emit_word("hi", ws + 1);
              s << "        " << v(n) << " = (lo << " << bs << ") | (hi >> " << (64 - bs) << ");\n";
            } else {
              s << "        " << v(n) << " = lo;\n";
            }
            s << "      }\n";
          }
          break;
        }
        case NOp::Shr: {
          // only inputs reach here (temporaries are cut)
          int64_t ws = x.k / 64;
          int bs = static_cast<int>(x.k % 64);
          s << "      u64 " << v(n) << ";\n      {\n"
            << "        const u64 lo = " << load(x.a, "w + " + std::to_string(ws) + "ll") << ";\n";
          if (bs) {
            s << "        u64 hi = __shfl_down_sync(~0u, lo, 1);\n"
              << "        if (lane == 31) hi = " << load(x.a, "base + " + std::to_string(ws + 32) + "ll") << ";\n"
              << "        " << v(n) << " = (lo >> " << bs << ") | (hi << " << (64 - bs) << ");\n";
          } else {
            s << "        " << v(n) << " = lo;\n";
          }
          s << "      }\n";
          break;
        }
        default:
          throw RuntimeError("fused: unexpected node kind");
      }
      if (masked && (x.op == NOp::Shl || x.op == NOp::Not || x.op == NOp::AndNot))
        s << "      " << v(n) << " &= lm;\n";
      if (track && dyn[n] && x.op != NOp::Add) {
        if (x.op == NOp::Shl && in_part.count(x.a) && !is_input(x.a)) {
          int64_t ws = x.k / 64;
          int bs = static_cast<int>(x.k % 64);
          s << "      dh" << n << " = min(" << dh(x.a) << " + " << (ws + (bs ? 1 : 0)) << ", 1 << 30);\n";
        } else {
          s << "      dh" << n << " = max(" << dh(x.a) << ", " << dh(x.b) << ");\n";
        }
      }
    }
    // carry previous-step values of left-shifted temporaries
    for (int n : shl_src) s << "      pv" << n << " = " << v(n) << ";\n";
    if (!track) {
      s << "      if (w < e) {\n";
      for (auto& kv : out_idx) s << "        A.out[" << kv.second << "][w] = " << v(kv.first) << ";\n";
      for (size_t j = 0; j < part.pops.size(); ++j)
        s << "        pc" << j << " += __popcll(" << v(part.pops[j].first) << ");\n";
      s << "      }\n";
    }
  }

  // dirt expression for operand o during warm-up tracking
  std::string dh(int o) const {
    if (o < 0) return "0";
    if (!in_part.count(o)) return "0";   // inputs / constants are exact
    if (dyn[o]) return "dh" + std::to_string(o);
    auto it = sdh.find(o);
    return std::to_string(it == sdh.end() ? 0 : it->second);
  }

  std::string source() {
    analyze();
    std::ostringstream s;
    const int ni = static_cast<int>(part.inputs.size()), no = static_cast<int>(part.outputs.size());
    s << "typedef unsigned long long u64;\ntypedef unsigned int u32;\n"
      << "struct Args {\n  const u64* in[" << std::max(1, ni) << "];\n  u64* out[" << std::max(1, no)
      << "];\n  unsigned long long* slots;\n  unsigned int* fail;\n  long long nw;\n"
      << "  long long range;\n  u64 last_mask;\n};\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << warps * 32 << ", " << min_blocks
      << ")\nbsz_fused(const Args A) {\n"
      << "  const int lane = threadIdx.x & 31;\n"
      << "  const long long gw = (long long)blockIdx.x * " << warps << " + (threadIdx.x >> 5);\n"
      << "  const long long s = gw * A.range;\n"
      << "  if (s >= A.nw) return;\n"
      << "  const long long e = min(s + A.range, A.nw);\n";
    std::vector<int> adds;
    for (int n : part.order)
      if (nodes[n].op == NOp::Add) adds.push_back(n);
    for (int n : adds) s << "  u32 c" << n << " = 0;\n";
    for (int n : shl_src) s << "  u64 pv" << n << " = 0;\n";
    for (size_t j = 0; j < part.pops.size(); ++j) s << "  u32 pc" << j << " = 0;\n";
    // ---- warm-up (speculative, exactness-checked)
    const bool need_warm = !adds.empty() || !shl_src.empty();
    if (need_warm) {
      s << "  const long long H = " << warm << ";\n"
        << "  long long p0 = s - H;\n  if (p0 < 0) p0 = 0;\n"
        << "  for (int attempt = 0; p0 < s; ++attempt) {\n";
      for (int n : adds) s << "    c" << n << " = 0;\n";
      for (int n : shl_src) s << "    pv" << n << " = 0;\n";
      for (int n : adds)
        if (dyn[n]) s << "    int res" << n << " = (p0 == 0);\n    int dh" << n << " = (p0 == 0) ? 0 : (1 << 30);\n";
      for (int n : part.order)
        if (dyn[n] && nodes[n].op != NOp::Add) s << "    int dh" << n << " = 0;\n";
      s << "    for (long long base = p0; base < s; base += 32) {\n";
      emit_step(s, true);
      s << "    }\n";
      // exactness: every carry and every previous-step value at s is exact
      s << "    const int need = (int)(s - p0);\n    bool ok = true;\n";
      for (int n : adds)
        if (dyn[n]) s << "    ok = ok && res" << n << " && dh" << n << " <= need;\n";
      for (int n : shl_src) {
        if (dyn[n]) s << "    ok = ok && dh" << n << " <= need - 32;\n";
        else if (sdh.count(n) && sdh.at(n) > 0)
          s << "    ok = ok && " << sdh.at(n) << " <= need - 32;\n";
      }
      s << "    if (ok || p0 == 0) break;\n"
        << "    if (attempt >= 8) { if (lane == 0) atomicOr(A.fail, 1u); break; }\n"
        << "    p0 = s - 2 * (s - p0);\n    if (p0 < 0) p0 = 0;\n"
        << "  }\n";
    }
    // ---- owned range
    s << "  for (long long base = s; base < e; base += 32) {\n";
    emit_step(s, false);
    s << "  }\n";
    for (size_t j = 0; j < part.pops.size(); ++j) {
      s << "  {\n    unsigned long long t = pc" << j << ";\n"
        << "    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(~0u, t, o);\n"
        << "    if (lane == 0 && t) atomicAdd(A.slots + " << part.pops[j].second << ", t);\n  }\n";
    }
    s << "}\n";
    return s.str();
  }
};

Compiled compile_source(const std::string& src, double* compile_ms) {
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = cache().find(src);
    if (it != cache().end()) return it->second;
  }
  auto t0 = std::chrono::high_resolution_clock::now();
  if (const char* dir = std::getenv("BSZ_DUMP_DIR")) {
    // developer aid: keep every generated kernel source
    static int counter = 0;
    std::string path = std::string(dir) + "/fused_" + std::to_string(counter++) + ".cu";
    if (FILE* f = std::fopen(path.c_str(), "w")) {
      std::fwrite(src.data(), 1, src.size(), f);
      std::fclose(f);
    }
  }
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), "bsz_fused.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
    throw RuntimeError("nvrtcCreateProgram failed");
  // warnings 550/177: warm-up steps compute values only the owned range stores
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device",
                        "--extra-device-vectorization", "--diag-suppress=550,177"};
  nvrtcResult r = nvrtcCompileProgram(prog, 5, opts);
  if (r != NVRTC_SUCCESS) {
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    nvrtcGetProgramLog(prog, &log[0]);
    nvrtcDestroyProgram(&prog);
    throw RuntimeError("NVRTC compile failed: " + log.substr(0, 2000));
  }
  size_t cubin_size = 0;
  nvrtcGetCUBINSize(prog, &cubin_size);
  std::string cubin(cubin_size, '\0');
  nvrtcGetCUBIN(prog, &cubin[0]);
  nvrtcDestroyProgram(&prog);
  Compiled c;
  BSZ_CU(drv().module_load_data(&c.mod, cubin.data()));
  BSZ_CU(drv().module_get_function(&c.fn, c.mod, "bsz_fused"));
  drv().func_get_attribute(&c.n_regs, CU_FUNC_ATTRIBUTE_NUM_REGS, c.fn);
  if (compile_ms)
    *compile_ms += std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
  std::lock_guard<std::mutex> lk(g_cache_mu);
  cache()[src] = c;
  return c;
}

// Splits a segment into parts: a node that reads a temporary through a right
// shift, or through a left shift of 2048 bits or more, starts a later part,
// and that temporary becomes an output of its own part.
std::vector<Part> split(const std::vector<Node>& nodes, const Segment& seg) {
  std::map<int, int> level;
  std::set<int> computed(seg.order.begin(), seg.order.end());
  std::set<int> cut_src;
  for (int n : seg.order) {
    const Node& x = nodes[n];
    int lv = 0;
    for (int o : {x.a, x.b}) {
      if (o < 0 || !computed.count(o)) continue;
      int l = level[o];
      bool cut = (x.op == NOp::Shr) || (x.op == NOp::Shl && x.k / 64 >= 32);
      if (cut) {
        cut_src.insert(o);
        l += 1;
      }
      lv = std::max(lv, l);
    }
    level[n] = lv;
  }
  int max_lv = 0;
  for (auto& kv : level) max_lv = std::max(max_lv, kv.second);
  std::vector<Part> parts(max_lv + 1);
  std::set<int> seg_out(seg.outputs.begin(), seg.outputs.end());
  for (int n : seg.order) parts[level[n]].order.push_back(n);
  for (int L = 0; L <= max_lv; ++L) {
    Part& p = parts[L];
    std::set<int> in_this(p.order.begin(), p.order.end());
    std::set<int> ins;
    for (int n : p.order) {
      const Node& x = nodes[n];
      for (int o : {x.a, x.b})
        if (o >= 0 && !in_this.count(o)) ins.insert(o);
    }
    for (int n : p.order)
      if (seg_out.count(n) || cut_src.count(n)) p.outputs.push_back(n);
    // temporaries of this part read by later parts through anything
    for (int L2 = L + 1; L2 <= max_lv; ++L2)
      for (int m : parts[L2].order)
        for (int o : {nodes[m].a, nodes[m].b})
          if (o >= 0 && in_this.count(o) &&
              std::find(p.outputs.begin(), p.outputs.end(), o) == p.outputs.end())
            p.outputs.push_back(o);
    p.inputs.assign(ins.begin(), ins.end());
  }
  // pops go to the part that computes their node (or part 0 for inputs)
  for (auto& pp : seg.pops) {
    int L = computed.count(pp.first) ? level[pp.first] : 0;
    Part& p = parts[L];
    p.pops.push_back(pp);
    if (!computed.count(pp.first) &&
        std::find(p.inputs.begin(), p.inputs.end(), pp.first) == p.inputs.end())
      p.inputs.push_back(pp.first);
  }
  return parts;
}

}  // namespace

void FusedBackend::run(std::vector<Node>& nodes, const Segment& seg, int64_t N, int64_t nw,
                       unsigned long long* d_slots, double* compile_ms) {
  Device& dev = impl_->dev;
  const ExecOptions& opt = impl_->opt;
  std::vector<Part> parts = split(nodes, seg);
  for (Part& p : parts) {
    if (p.order.empty() && p.pops.empty()) continue;
    if (p.inputs.size() > kMaxInputs) throw RuntimeError("fused: too many inputs in one segment");
    Gen g{nodes, p, N, opt.fused_warps, opt.fused_ctas_per_sm, (N % 64) != 0};
    const std::string src = g.source();
    Compiled c = compile_source(src, compile_ms);
    // outputs
    for (int n : p.outputs)
      if (!nodes[n].buf) nodes[n].buf = dev.alloc_stream(nw);
    // argument block, laid out as the generated struct
    const int ni = std::max<int>(1, static_cast<int>(p.inputs.size()));
    const int no = std::max<int>(1, static_cast<int>(p.outputs.size()));
    std::vector<uint64_t> args(ni + no + 5, 0);
    for (size_t i = 0; i < p.inputs.size(); ++i) {
      const Node& x = nodes[p.inputs[i]];
      args[i] = x.buf ? reinterpret_cast<uint64_t>(x.buf->p) : 0;
    }
    for (size_t i = 0; i < p.outputs.size(); ++i) args[ni + i] = reinterpret_cast<uint64_t>(nodes[p.outputs[i]].buf->p);
    // grid: contiguous ranges of whole 32-word steps, at least 8 warm-ups long
    const int64_t steps = (nw + 31) / 32;
    int64_t max_warps = static_cast<int64_t>(dev.sm_count()) * opt.fused_ctas_per_sm * opt.fused_warps;
    int64_t min_range_steps = std::max<int64_t>(opt.fused_chunk_steps, (g.warm / 32) * 8);
    int64_t warps_needed = std::max<int64_t>(1, std::min(max_warps, (steps + min_range_steps - 1) / min_range_steps));
    int64_t range = ((steps + warps_needed - 1) / warps_needed) * 32;
    int64_t total_warps = (nw + range - 1) / range;
    int blocks = static_cast<int>((total_warps + opt.fused_warps - 1) / opt.fused_warps);
    args[ni + no + 0] = reinterpret_cast<uint64_t>(d_slots);
    args[ni + no + 1] = reinterpret_cast<uint64_t>(impl_->d_fail);
    args[ni + no + 2] = static_cast<uint64_t>(nw);
    args[ni + no + 3] = static_cast<uint64_t>(range);
    args[ni + no + 4] = mask_for_bits(N);
    BSZ_CUDA(cudaMemsetAsync(impl_->d_fail, 0, 4, dev.stream()));
    void* kparams[] = {args.data()};
    {
      ProfScope prof(dev, "fused");
      BSZ_CU(drv().launch_kernel(c.fn, blocks, 1, 1, opt.fused_warps * 32, 1, 1, 0,
                            reinterpret_cast<CUstream>(dev.stream()), kparams, nullptr));
    }
    ++dev.n_launches;
    ++launches;
    unsigned int fail = 0;
    BSZ_CUDA(cudaMemcpyAsync(&fail, impl_->d_fail, 4, cudaMemcpyDeviceToHost, dev.stream()));
    BSZ_CUDA(cudaStreamSynchronize(dev.stream()));
    if (fail) {
      // Speculation could not be proven exact: redo this part with the plain
      // per-op kernels (exact by construction).
      for (auto& pp : p.pops) BSZ_CUDA(cudaMemsetAsync(d_slots + pp.second, 0, 8, dev.stream()));
      const uint64_t lm = mask_for_bits(N);
      std::map<int, BufRef> tmp;
      auto ptr = [&](int n) -> const uint64_t* {
        if (nodes[n].buf) return nodes[n].buf->p;
        auto it = tmp.find(n);
        if (it != tmp.end()) return it->second->p;
        throw RuntimeError("fused fallback: operand without a buffer");
      };
      for (int n : p.order) {
        const Node& x = nodes[n];
        BufRef out = nodes[n].buf ? nodes[n].buf : dev.alloc_stream(nw);
        uint64_t* D = out->p;
        auto opnd = [&](int o) -> const uint64_t* {
          const Node& y = nodes[o];
          if (is_const(y.op)) {
            auto it = tmp.find(o);
            if (it == tmp.end()) {
              BufRef b = dev.alloc_stream(nw);
              uint64_t val = y.op == NOp::Zero ? 0 : ~uint64_t(0);
              uint64_t last = y.op == NOp::OnesMask ? lm : val;
              launch_fill(dev, b->p, nw, val, last);
              it = tmp.emplace(o, b).first;
            }
            return it->second->p;
          }
          return ptr(o);
        };
        switch (x.op) {
          case NOp::Not: launch_not(dev, D, opnd(x.a), nw, lm); break;
          case NOp::And: launch_bitwise(dev, kAnd, D, opnd(x.a), opnd(x.b), nw); break;
          case NOp::Or: launch_bitwise(dev, kOr, D, opnd(x.a), opnd(x.b), nw); break;
          case NOp::Xor: launch_bitwise(dev, kXor, D, opnd(x.a), opnd(x.b), nw); break;
          case NOp::AndNot: launch_bitwise(dev, kAndNot, D, opnd(x.a), opnd(x.b), nw); break;
          case NOp::Add: launch_add(dev, D, opnd(x.a), opnd(x.b), nw, lm); break;
          case NOp::Shl: launch_shl(dev, D, opnd(x.a), x.k, nw, lm); break;
          case NOp::Shr: launch_shr(dev, D, opnd(x.a), x.k, nw, nodes[x.a].tail ? ~uint64_t(0) : 0); break;
          default: throw RuntimeError("fused fallback: unexpected node");
        }
        if (!nodes[n].buf) tmp[n] = out;
      }
      for (auto& pp : p.pops) {
        const Node& y = nodes[pp.first];
        const uint64_t* src_ptr = y.buf ? y.buf->p : tmp.at(pp.first)->p;
        launch_popcount(dev, src_ptr, nw, d_slots + pp.second);
      }
      ++fallbacks;
    }
  }
}

}  // namespace bsz
