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
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <unordered_map>
#include <unordered_set>

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
  CUresult (*occupancy)(int*, CUfunction, int, size_t) = nullptr;
  CUresult (*func_set_attribute)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*tensor_map_encode_tiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                      const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill) = nullptr;
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
    resolve("cuOccupancyMaxActiveBlocksPerMultiprocessor", x.occupancy);
    resolve("cuFuncSetAttribute", x.func_set_attribute);
    resolve("cuTensorMapEncodeTiled", x.tensor_map_encode_tiled);
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
  int blocks_per_sm = 1;   // occupancy of the compiled kernel at its block size
};

// Process-wide cache of compiled kernels keyed by a 128-bit digest of the
// generated source (two independent 64-bit hashes and the length), not the
// source itself: a tuning run holds tens of thousands of kernels whose
// sources are hundreds of kilobytes each.
std::mutex g_cache_mu;
std::unordered_map<std::string, Compiled>& cache() {
  static std::unordered_map<std::string, Compiled> c;
  return c;
}

std::string src_digest(const std::string& src) {
  uint64_t h1 = 1469598103934665603ull, h2 = 0x9E3779B97F4A7C15ull;
  for (char ch : src) {
    const uint64_t c = static_cast<unsigned char>(ch);
    h1 = (h1 ^ c) * 1099511628211ull;   // FNV-1a
    h2 = (h2 + c + 1) * 0xff51afd7ed558ccdull;
    h2 ^= h2 >> 29;
  }
  char buf[64];
  std::snprintf(buf, sizeof buf, "%016llx%016llx:%zu", static_cast<unsigned long long>(h1),
                static_cast<unsigned long long>(h2), src.size());
  return buf;
}

bool is_const(NOp op) { return op == NOp::Zero || op == NOp::OnesMask || op == NOp::AllOnes; }

}  // namespace

namespace {

// One kernel's worth of the segment.
struct Part {
  std::vector<int> order;                     // computed nodes (topological)
  std::vector<int> inputs;                    // materialized nodes read (Buf or earlier part)
  std::vector<int> outputs;                   // nodes to store
  std::vector<std::pair<int, int64_t>> pops;  // (node, slot)
  bool lookback_add = false;                  // one addition of materialized operands, run by
                                              // the plain carry-scan kernel (decoupled look-back)
};

struct Gen {
  const std::vector<Node>& nodes;
  const Part& part;
  int64_t N;
  int warps;
  int min_blocks;
  bool masked;
  bool prefetch;
  bool guard_outputs = false;      // batches: an output pointer may be null (not stored)
  // batches: fixed argument positions (input node -> A.in index; (node, A.out index))
  const std::map<int, int>* in_index_override = nullptr;
  const std::vector<std::pair<int, int>>* outs_override = nullptr;
  // derived
  std::map<int, int> in_idx;       // node -> input index
  std::vector<std::pair<int, int>> outs;   // (node, output index); a node may repeat
  std::set<int> in_part;           // computed in this part
  std::set<int> shl_src;           // temporaries shifted left (need previous-step value)
  std::map<int, int> shl_ws;       // max word shift per shl source temporary
  // Shifted temporaries whose every left shift is by 1 or 2 bits: the bits
  // shifted in come from the top bits of the word below, which one ballot
  // per bit delivers to every lane; across steps only those 1-2 bits of the
  // last lane are carried (a warp-uniform u32 instead of a 64-bit
  // previous-step value per lane, and no shuffles).
  std::map<int, int> small_shl;    // source -> max bit shift (1 or 2); absent: general
  // Warp-uniform carried bits (add carries, small-shift edge bits) are packed
  // into u32 words pk0, pk1, ...: bit position per add / small-shift source.
  std::map<int, int> cbit, mbit;
  int n_pack = 0;
  // Emission order: depth-first from the part's roots, larger operand
  // subtree first, which keeps fewer values live inside a step than node-id
  // order (fewer registers, so more warps per SM).
  std::vector<int> emit_order;
  // Small-shift sources: the last shift node (in emit_order) that reads
  // them; that node also stores the carried edge bits for the next step, so
  // no ballot result stays live across the step.
  std::map<int, int> last_small_use;
  std::string pk(int bitpos) const { return "pk" + std::to_string(bitpos / 32); }
  std::vector<uint8_t> dyn;        // node dirt must be tracked during warm-up
  std::map<int, int64_t> sdh;      // static dirt (words) for nodes without add ancestors
  int64_t warm = 64;               // warm-up words
  // Global loads of one step ("load slots"): expression templates over @W@
  // (this lane's word) and @B@ (the step's first word), de-duplicated.  The
  // owned-range loop issues them one step ahead of the arithmetic.
  std::vector<std::string> slot_tmpl;
  std::map<std::string, int> slot_of;

  std::string v(int n) const { return "v" + std::to_string(n); }
  bool is_input(int n) const { return in_idx.count(n) != 0; }

  int slot(const std::string& tmpl) {
    auto it = slot_of.find(tmpl);
    if (it != slot_of.end()) return it->second;
    int id = static_cast<int>(slot_tmpl.size());
    slot_tmpl.push_back(tmpl);
    slot_of[tmpl] = id;
    return id;
  }
  static std::string subst(std::string t, const std::string& w, const std::string& b) {
    for (size_t p; (p = t.find("@W@")) != std::string::npos;) t.replace(p, 3, w);
    for (size_t p; (p = t.find("@B@")) != std::string::npos;) t.replace(p, 3, b);
    return t;
  }
  std::string slot_cur(const std::string& tmpl) const { return "cur" + std::to_string(slot_of.at(tmpl)); }
  // templates used by nodes
  std::string t_word(int n) const { return load(n, "@W@"); }
  std::string t_shl_lo(const Node& x) const { return load(x.a, "@W@ - " + std::to_string(x.k / 64) + "ll"); }
  std::string t_shl_edge(const Node& x) const {
    return "(lane == 0 ? " + load(x.a, "@B@ - " + std::to_string(x.k / 64 + 1) + "ll") + " : 0ull)";
  }
  std::string t_shr_lo(const Node& x) const { return load(x.a, "@W@ + " + std::to_string(x.k / 64) + "ll"); }
  std::string t_shr_edge(const Node& x) const {
    return "(lane == 31 ? " + load(x.a, "@B@ + " + std::to_string(x.k / 64 + 32) + "ll") + " : 0ull)";
  }
  void make_slots() {
    for (auto& kv : in_idx) slot(t_word(kv.first));
    for (int n : part.order) {
      const Node& x = nodes[n];
      if (x.op == NOp::Shl && (is_input(x.a) || is_const(nodes[x.a].op))) {
        slot(t_shl_lo(x));
        if (x.k % 64) slot(t_shl_edge(x));
      } else if (x.op == NOp::Shr) {
        slot(t_shr_lo(x));
        if (x.k % 64) slot(t_shr_edge(x));
      }
    }
  }
  // assignments of every load slot for the step starting at `b` (lane word `w`)
  void emit_loads(std::ostringstream& s, const std::string& prefix, bool declare, const std::string& w,
                  const std::string& b, const char* indent) const {
    for (size_t i = 0; i < slot_tmpl.size(); ++i)
      s << indent << (declare ? "const u64 " : "") << prefix << i << " = " << subst(slot_tmpl[i], w, b)
        << ";\n";
  }

  void analyze() {
    if (in_index_override) {
      for (int n : part.inputs) {
        auto it = in_index_override->find(n);
        in_idx[n] = it == in_index_override->end() ? 0 : it->second;   // constants: index unused
      }
    } else {
      for (size_t i = 0; i < part.inputs.size(); ++i) in_idx[part.inputs[i]] = static_cast<int>(i);
    }
    if (outs_override) outs = *outs_override;
    else
      for (size_t i = 0; i < part.outputs.size(); ++i) outs.push_back({part.outputs[i], static_cast<int>(i)});
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
        const bool small = x.k >= 1 && x.k <= 2;
        if (!shl_src.count(x.a)) {
          if (small) small_shl[x.a] = static_cast<int>(x.k);
        } else if (small_shl.count(x.a)) {
          if (small) small_shl[x.a] = std::max(small_shl[x.a], static_cast<int>(x.k));
          else small_shl.erase(x.a);
        }
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
    int nb = 0;
    for (int n : part.order)
      if (nodes[n].op == NOp::Add) cbit[n] = nb++;
    for (auto& kv : small_shl) {
      if (nb / 32 != (nb + kv.second - 1) / 32) nb = (nb / 32 + 1) * 32;   // keep a pair in one word
      mbit[kv.first] = nb;
      nb += kv.second;
    }
    n_pack = (nb + 31) / 32;
    order_for_registers();
    for (int n : emit_order) {
      const Node& x = nodes[n];
      if (x.op == NOp::Shl && x.a >= 0 && small_shl.count(x.a)) last_small_use[x.a] = n;
    }
    make_slots();
  }

  void order_for_registers() {
    std::map<int, int> users;
    std::map<int, int64_t> size;
    for (int n : part.order) {
      const Node& x = nodes[n];
      int64_t sz = 1;
      for (int o : {x.a, x.b})
        if (o >= 0 && in_part.count(o)) {
          ++users[o];
          sz += size[o];
        }
      size[n] = std::min<int64_t>(sz, int64_t(1) << 40);
    }
    std::set<int> seen;
    emit_order.clear();
    // iterative post-order DFS
    auto visit = [&](int root) {
      std::vector<std::pair<int, int>> st{{root, 0}};
      while (!st.empty()) {
        auto& [n, stage] = st.back();
        if (stage == 0) {
          if (seen.count(n)) { st.pop_back(); continue; }
          seen.insert(n);
          stage = 1;
          const Node& x = nodes[n];
          std::vector<int> kids;
          for (int o : {x.a, x.b})
            if (o >= 0 && in_part.count(o) && !seen.count(o)) kids.push_back(o);
          if (kids.size() == 2 && size[kids[0]] < size[kids[1]]) std::swap(kids[0], kids[1]);
          // push in reverse so the larger subtree is visited first
          for (auto it = kids.rbegin(); it != kids.rend(); ++it) st.push_back({*it, 0});
        } else {
          emit_order.push_back(n);
          st.pop_back();
        }
      }
    };
    std::vector<int> roots;
    for (auto& o : outs) roots.push_back(o.first);
    for (auto& p : part.pops) roots.push_back(p.first);
    for (int n : part.order)
      if (!users.count(n)) roots.push_back(n);
    for (int r : roots)
      if (in_part.count(r)) visit(r);
    for (int n : part.order)
      if (!seen.count(n)) visit(n);
  }

  // expression for an input node value at word index expression `idx`
  std::string load(int n, const std::string& idx) const {
    // Word `idx` of a stream; words below 0 are zero (shifting in zeros),
    // words at or past nw are the tail.
    const Node& x = nodes[n];
    if (x.op == NOp::Zero) return "0ull";
    if (x.op == NOp::AllOnes) return "((" + idx + ") >= 0 ? ~0ull : 0ull)";
    if (x.op == NOp::OnesMask)
      return "((" + idx + ") >= 0 && (" + idx + ") < A.nw - 1 ? ~0ull : ((" + idx +
             ") == A.nw - 1 ? A.last_mask : 0ull))";
    std::string fill = x.tail ? "~0ull" : "0ull";
    return "((" + idx + ") >= 0 && (" + idx + ") < A.nw ? __ldg(A.in[" + std::to_string(in_idx.at(n)) +
           "] + (" + idx + ")) : " + fill + ")";
  }

  // value of operand o in the current step (already computed or loaded)
  std::string opnd(int o) const { return v(o); }

  // One 32-word step.  prefetched: the load slots are already in cur<i>
  // (the owned-range loop loads them a step ahead); otherwise load here.
  void emit_step(std::ostringstream& s, bool track, bool prefetched) const {
    s << "      const long long w = base + lane;\n";
    if (masked) s << "      const u64 lm = (w == A.nw - 1) ? A.last_mask : ~0ull;\n";
    if (!prefetched) emit_loads(s, "cur", true, "w", "base", "      ");
    for (auto& kv : in_idx) s << "      const u64 " << v(kv.first) << " = " << slot_cur(t_word(kv.first)) << ";\n";
    if (track) s << "      const int rel = (int)(base - p0);\n";
    for (int n : emit_order) {
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
          const int cb = cbit.at(n);
          const std::string w = pk(cb), sh = std::to_string(cb % 32);
          s << "        const unsigned long long z = (unsigned long long)(G | P) + G + ((" << w << " >> " << sh
            << ") & 1u);\n"
            << "        const u32 cv = (u32)z ^ P;\n"
            << "        " << w << " = (" << w << " & ~(1u << " << sh << ")) | ((u32)(z >> 32) << " << sh << ");\n"
            << "        " << v(n) << " = sa + ((cv >> lane) & 1u)" << (masked ? " & lm" : "") << ";\n"
            << "      }\n";
          break;
        }
        case NOp::Shl: {
          int64_t ws = x.k / 64;
          int bs = static_cast<int>(x.k % 64);
          if (is_input(x.a) || is_const(nodes[x.a].op)) {
            s << "      u64 " << v(n) << ";\n      {\n"
              << "        const u64 lo = " << slot_cur(t_shl_lo(x)) << ";\n";
            if (bs) {
              s << "        u64 hi = __shfl_up_sync(~0u, lo, 1);\n"
                << "        if (lane == 0) hi = " << slot_cur(t_shl_edge(x)) << ";\n"
                << "        " << v(n) << " = (lo << " << bs << ") | (hi >> " << (64 - bs) << ");\n";
            } else {
              s << "        " << v(n) << " = lo;\n";
            }
            s << "      }\n";
          } else if (small_shl.count(x.a)) {
            // bits shifted in: bit 63 (and 62) of the word below, from one
            // ballot per bit; lane 0 takes the previous step's lane 31 bits
            const std::string cur = opnd(x.a);
            const int mb = mbit.at(x.a);
            const bool last = last_small_use.at(x.a) == n;
            const bool need62 = bs == 2 || (last && small_shl.at(x.a) == 2);
            const std::string w = pk(mb), sh = std::to_string(mb % 32), sh1 = std::to_string(mb % 32 + 1);
            s << "      u64 " << v(n) << ";\n      {\n"
              << "        const u32 q63 = __ballot_sync(~0u, (" << cur << " >> 63) != 0ull);\n";
            if (need62) s << "        const u32 q62 = __ballot_sync(~0u, ((" << cur << " >> 62) & 1ull) != 0ull);\n";
            s << "        const u32 m63 = (q63 << 1) | ((" << w << " >> " << sh << ") & 1u);\n";
            if (bs == 1) {
              s << "        " << v(n) << " = (" << cur << " << 1) | (u64)((m63 >> lane) & 1u);\n";
            } else {
              s << "        const u32 m62 = (q62 << 1) | ((" << w << " >> " << sh1 << ") & 1u);\n"
                << "        " << v(n) << " = (" << cur << " << 2) | (u64)(((m63 >> lane) & 1u) << 1) | "
                << "(u64)((m62 >> lane) & 1u);\n";
            }
            if (last) {
              const unsigned mask = small_shl.at(x.a) == 2 ? 3u : 1u;
              s << "        " << w << " = (" << w << " & ~(" << mask << "u << " << sh << ")) | ((q63 >> 31) << " << sh
                << ")";
              if (small_shl.at(x.a) == 2) s << " | ((q62 >> 31) << " << sh1 << ")";
              s << ";\n";
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
          int bs = static_cast<int>(x.k % 64);
          s << "      u64 " << v(n) << ";\n      {\n"
            << "        const u64 lo = " << slot_cur(t_shr_lo(x)) << ";\n";
          if (bs) {
            s << "        u64 hi = __shfl_down_sync(~0u, lo, 1);\n"
              << "        if (lane == 31) hi = " << slot_cur(t_shr_edge(x)) << ";\n"
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
    // carry previous-step values of left-shifted temporaries (1-2 bit shift
    // sources carry their edge bits at their last shift instead)
    for (int n : shl_src)
      if (!small_shl.count(n)) s << "      pv" << n << " = " << v(n) << ";\n";
    if (!track) {
      s << "      if (w < e) {\n";
      for (auto& kv : outs)
        s << "        " << (guard_outputs ? "if (A.out[" + std::to_string(kv.second) + "]) " : std::string())
          << "A.out[" << kv.second << "][w] = " << v(kv.first) << ";\n";
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

  static std::string args_struct(int ni, int no) {
    std::ostringstream s;
    s << "typedef unsigned long long u64;\ntypedef unsigned int u32;\n"
      << "struct Args {\n  const u64* in[" << std::max(1, ni) << "];\n  u64* out[" << std::max(1, no)
      << "];\n  unsigned long long* slots;\n  unsigned int* fail;\n  long long nw;\n"
      << "  long long range;\n  u64 last_mask;\n  unsigned long long one;\n};\n";
    return s.str();
  }

  // Whole kernel for one segment part: each warp owns range [s, e).
  std::string source() {
    analyze();
    std::ostringstream s;
    const int ni = static_cast<int>(part.inputs.size()), no = static_cast<int>(part.outputs.size());
    s << args_struct(ni, no)
      << "extern \"C\" __global__ void __launch_bounds__(" << warps * 32 << ", " << min_blocks
      << ")\nbsz_fused(const Args A) {\n"
      << "  const int lane = threadIdx.x & 31;\n"
      << "  const long long gw = (long long)blockIdx.x * " << warps << " + (threadIdx.x >> 5);\n"
      << "  const long long s = gw * A.range;\n"
      << "  if (s >= A.nw) return;\n"
      << "  const long long e = min(s + A.range, A.nw);\n";
    body(s);
    s << "}\n";
    return s.str();
  }

  // Device function for batches: one work item = range [s, e) of one instance.
  std::string device_function(const std::string& name) {
    analyze();
    std::ostringstream s;
    // the instance's argument block stays in global memory (read-only,
    // not aliased): copying it would pin ~20 registers for the whole item
    s << "__device__ __noinline__ void " << name
      << "(const Args* __restrict__ Ap, const long long s, const long long e, const int lane) {\n"
      << "  const Args& A = *Ap;\n";
    body(s);
    s << "}\n";
    return s.str();
  }

  void body(std::ostringstream& s) {
    std::vector<int> adds;
    for (int n : part.order)
      if (nodes[n].op == NOp::Add) adds.push_back(n);
    for (int i = 0; i < n_pack; ++i) s << "  u32 pk" << i << " = 0;\n";
    for (int n : shl_src)
      if (!small_shl.count(n)) s << "  u64 pv" << n << " = 0;\n";
    for (size_t j = 0; j < part.pops.size(); ++j) s << "  u32 pc" << j << " = 0;\n";
    // ---- warm-up (speculative, exactness-checked)
    const bool need_warm = !adds.empty() || !shl_src.empty();
    if (need_warm) {
      s << "  const long long H = " << warm << ";\n"
        << "  long long p0 = s - H;\n  if (p0 < 0) p0 = 0;\n"
        << "  for (int attempt = 0; p0 < s; ++attempt) {\n";
      for (int i = 0; i < n_pack; ++i) s << "    pk" << i << " = 0;\n";
      for (int n : shl_src)
        if (!small_shl.count(n)) s << "    pv" << n << " = 0;\n";
      for (int n : adds)
        if (dyn[n]) s << "    int res" << n << " = (p0 == 0);\n    int dh" << n << " = (p0 == 0) ? 0 : (1 << 30);\n";
      for (int n : part.order)
        if (dyn[n] && nodes[n].op != NOp::Add) s << "    int dh" << n << " = 0;\n";
      s << "    for (long long base = p0; base < s; base += 32) {\n";
      emit_step(s, true, false);
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
    // ---- owned range: the loads of step t+1 are issued before the arithmetic
    // of step t, so each warp keeps two steps of loads in flight.
    if (!prefetch) {
      s << "  for (long long base = s; base < e; base += 32) {\n";
      emit_step(s, false, false);
      s << "  }\n";
    } else {
    for (size_t i = 0; i < slot_tmpl.size(); ++i) s << "  u64 pf" << i << ";\n";
    s << "  {\n    const long long base = s;\n    const long long w = base + lane;\n";
    emit_loads(s, "pf", false, "w", "base", "    ");
    s << "  }\n";
    s << "  for (long long base = s; base < e; base += 32) {\n";
    for (size_t i = 0; i < slot_tmpl.size(); ++i) s << "      const u64 cur" << i << " = pf" << i << ";\n";
    s << "      {\n        const long long bn = base + 32;\n        if (bn < e) {\n"
      << "          const long long wn = bn + lane;\n";
    emit_loads(s, "pf", false, "wn", "bn", "          ");
    s << "        }\n      }\n";
    emit_step(s, false, true);
    s << "  }\n";
    }
    for (size_t j = 0; j < part.pops.size(); ++j) {
      s << "  {\n    unsigned long long t = pc" << j << ";\n"
        << "    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(~0u, t, o);\n"
        << "    if (lane == 0 && t) atomicAdd(A.slots + " << part.pops[j].second << ", t);\n  }\n";
    }
  }
};

// Thread-sequential form of a segment part.  Each thread owns a contiguous
// range of whole 4-word chunks and walks it in word order, so every
// cross-word operator keeps its state in the thread's registers:
//   * x + y: a 64-bit add with carry in and out (a PTX carry chain: four
//     integer instructions per word), the carry held in a register;
//   * x << k (k < 64): two funnel shifts against the previous word of x,
//     held in a register (a temporary shifted by 64 bits or more ends the
//     part: it is materialized by an earlier kernel);
//   * shifts of an input by 64 bits or more read the input at the word
//     offset directly.
// Memory: a chunk of every input is one 256-bit load per thread (one 32-byte
// sector), a chunk of every output one 256-bit store; the chunks of
// neighbouring threads are a range apart.  Chunks at the ends of the stream
// (and any chunk whose shifted loads would leave [0, nw)) take a scalar path
// with bounds, tail fill and last-word masking.  The state at the start of a
// thread's range comes from speculation as in the warp form: H warm-up words
// from an all-zero state, per-node dirt tracking (an addition is exact after
// the first word where a ^ b is not all ones, at or after its operands' dirt),
// doubled up to 8 times, then the fail flag and the exact per-op fallback.
struct GenSeq {
  const std::vector<Node>& nodes;
  const Part& part;
  int64_t N;
  int warps;
  int min_blocks;
  bool masked;
  std::map<int, int> in_idx;
  std::vector<std::pair<int, int>> outs;
  std::set<int> in_part;
  std::set<int> prev_src;            // nodes whose previous word a shift (k < 64) reads
  std::vector<uint8_t> dyn;
  std::map<int, int64_t> sdh;        // static dirt (words) of nodes without add ancestors
  int64_t warm = 4;                  // warm-up words (multiple of 4)
  std::vector<int> emit_order;
  // shifted input reads by a word offset: (node, word offset) -> slot; the
  // offset is -ws for a left shift and +ws for a right shift (|ws| >= 1 for
  // left shifts; right shifts also read offset ws + 1)
  std::map<std::pair<int, int64_t>, int> off_slot;
  int64_t fast_lo = 0;               // a chunk at c is fast if c >= fast_lo ...
  int64_t fast_hi_pad = 3;           // ... and c + fast_hi_pad <= nw - 1 - masked
  // TMA form (layout 2): inputs arrive as tensor-map boxes of `roww` words x
  // 32 threads per warp in `stages` shared-memory stages, outputs leave the
  // same way; shifted-input reads by 64 bits or more use bounded loads.
  bool tma = false;
  int roww = 8;
  int stages = 2;
  bool unroll_pairs = false;         // unroll a chunk's word pairs (more ILP, more code)
  int reg_chunk = 4;                 // register form: words per chunk (4 or 8: 32- or 64-byte sectors)
  // shifts of a word against its predecessor as integer multiply-adds by
  // 2^k (the multiply pipe) instead of funnel shifts (the logic pipe, which
  // bounds large DAGs); the multiplier comes from A.one so it stays a multiply
  bool shift_mul = false;
  std::set<int> mul_amounts;         // k % 32 of the shifts that use multipliers
  std::vector<int> mapped;           // input indices (A.in order) that are read through boxes
  // batches: fixed argument positions and outputs that may be skipped (null)
  bool guard_outputs = false;
  const std::map<int, int>* in_index_override = nullptr;
  const std::vector<std::pair<int, int>>* outs_override = nullptr;

  std::string v(int n) const { return "v" + std::to_string(n); }

  void analyze() {
    if (in_index_override) {
      for (int n : part.inputs) {
        auto it = in_index_override->find(n);
        in_idx[n] = it == in_index_override->end() ? 0 : it->second;   // constants: index unused
      }
    } else {
      for (size_t i = 0; i < part.inputs.size(); ++i) in_idx[part.inputs[i]] = static_cast<int>(i);
    }
    if (outs_override) outs = *outs_override;
    else
      for (size_t i = 0; i < part.outputs.size(); ++i) outs.push_back({part.outputs[i], static_cast<int>(i)});
    for (int n : part.order) in_part.insert(n);
    dyn.assign(nodes.size(), 0);
    // Static dirt of nodes without an addition among their ancestors, in
    // BITS: a value exact from bit B shifted left by k < 64 is exact from bit
    // B + k (sdh keeps the word form, ceil(B / 64), which the warm-up checks
    // and the run-time tracking of the other nodes use).
    std::map<int, int64_t> sbits;
    int64_t max_static_bits = 0;
    for (int n : part.order) {
      const Node& x = nodes[n];
      auto d = [&](int o) -> int64_t { return (o >= 0 && sbits.count(o)) ? sbits[o] : 0; };
      bool dy = x.op == NOp::Add;
      for (int o : {x.a, x.b})
        if (o >= 0 && dyn[o]) dy = true;
      int64_t s = std::max(d(x.a), d(x.b));
      if (x.op == NOp::Shl) {
        const int64_t ws = x.k / 64;
        if (in_part.count(x.a)) {
          if (ws > 0) throw RuntimeError("fused: shift of a temporary by 64 bits or more in a sequential part");
          if (x.k > 0) { prev_src.insert(x.a); s = d(x.a) + x.k; }
        } else if (!is_const(nodes[x.a].op)) {
          if (ws == 0) {
            // the previous word of an input is zero at the first warm-up word
            if (x.k > 0) { prev_src.insert(x.a); s = x.k; }
          } else {
            off_slot[{x.a, -ws}] = 0;
            if (x.k % 64) off_slot[{x.a, -ws - 1}] = 0;
          }
        }
      } else if (x.op == NOp::Shr && !is_const(nodes[x.a].op)) {
        const int64_t ws = x.k / 64;
        off_slot[{x.a, ws}] = 0;
        if (x.k % 64) off_slot[{x.a, ws + 1}] = 0;
      }
      dyn[n] = dy;
      if (!dy) {
        sbits[n] = s;
        sdh[n] = (s + 63) / 64;
        max_static_bits = std::max(max_static_bits, s);
      }
    }
    warm = std::max<int64_t>(4, (((max_static_bits + 63) / 64 + 2 + 3) / 4) * 4);
    int k = 0;
    for (auto& kv : off_slot) {
      kv.second = k++;
      // a fast chunk at c loads words [c + base, c + base + 8) for this slot
      const int64_t off = kv.first.second, base = slot_base(off);
      if (base < 0) fast_lo = std::max<int64_t>(fast_lo, -base);
      else fast_hi_pad = std::max<int64_t>(fast_hi_pad, base + 7);
    }
    order_for_registers();
  }

  void order_for_registers() {
    std::map<int, int> users;
    std::map<int, int64_t> size;
    for (int n : part.order) {
      const Node& x = nodes[n];
      int64_t sz = 1;
      for (int o : {x.a, x.b})
        if (o >= 0 && in_part.count(o)) {
          ++users[o];
          sz += size[o];
        }
      size[n] = std::min<int64_t>(sz, int64_t(1) << 40);
    }
    std::set<int> seen;
    auto visit = [&](int root) {
      std::vector<std::pair<int, int>> st{{root, 0}};
      while (!st.empty()) {
        auto& [n, stage] = st.back();
        if (stage == 0) {
          if (seen.count(n)) { st.pop_back(); continue; }
          seen.insert(n);
          stage = 1;
          const Node& x = nodes[n];
          std::vector<int> kids;
          for (int o : {x.a, x.b})
            if (o >= 0 && in_part.count(o) && !seen.count(o)) kids.push_back(o);
          if (kids.size() == 2 && size[kids[0]] < size[kids[1]]) std::swap(kids[0], kids[1]);
          for (auto it = kids.rbegin(); it != kids.rend(); ++it) st.push_back({*it, 0});
        } else {
          emit_order.push_back(n);
          st.pop_back();
        }
      }
    };
    std::vector<int> roots;
    for (auto& o : outs) roots.push_back(o.first);
    for (auto& p : part.pops) roots.push_back(p.first);
    for (int n : part.order)
      if (!users.count(n)) roots.push_back(n);
    for (int r : roots)
      if (in_part.count(r)) visit(r);
    for (int n : part.order)
      if (!seen.count(n)) visit(n);
  }

  // Bounded scalar read of word `idx` of an input or constant node.
  std::string ld(int n, const std::string& idx) const {
    const Node& x = nodes[n];
    if (x.op == NOp::Zero) return "0ull";
    if (x.op == NOp::AllOnes) return "((" + idx + ") >= 0 ? ~0ull : 0ull)";
    if (x.op == NOp::OnesMask)
      return "((" + idx + ") >= 0 && (" + idx + ") < A.nw - 1 ? ~0ull : ((" + idx +
             ") == A.nw - 1 ? A.last_mask : 0ull))";
    const std::string fill = x.tail ? "~0ull" : "0ull";
    return "((" + idx + ") >= 0 && (" + idx + ") < A.nw ? A.in[" + std::to_string(in_idx.at(n)) + "][" + idx +
           "] : " + fill + ")";
  }

  // Value of an input/constant at the current word in the fast path.
  std::string fast_in(int n, int j) const {
    const Node& x = nodes[n];
    if (x.op == NOp::Zero) return "0ull";
    if (x.op == NOp::AllOnes || x.op == NOp::OnesMask) return "~0ull";   // the fast path never holds the last word
    return "c" + std::to_string(in_idx.at(n)) + "_" + std::to_string(j);
  }
  // Word at offset `off` of input n (a shifted read), fast path: from the two
  // aligned chunks loaded for that slot.
  // first word (relative to the chunk) of the two aligned chunks loaded for
  // word offset `off`: they hold words j + off for j = 0..3
  static int64_t slot_base(int64_t off) { return off < 0 ? -4 * ((-off + 3) / 4) : 4 * (off / 4); }
  std::string fast_off(int n, int64_t off, int j) const {
    const int slot = off_slot.at({n, off});
    return "o" + std::to_string(slot) + "_" + std::to_string(j + off - slot_base(off));
  }

  // One word of the DAG.  mode 'f': fast (word j of the chunk at c);
  // 's': scalar at word w; 't': scalar with dirt tracking (warm-up, relative
  // word r).  Values only; the caller stores / counts.
  void emit_word(std::ostringstream& s, char mode, int j) const {
    const bool slow = mode != 'f';
    const std::string W = slow ? "w" : "(c + " + std::to_string(j) + ")";
    if (slow && masked) s << "      const u64 lm = (w == A.nw - 1) ? A.last_mask : ~0ull;\n";
    // every input and constant gets its value name (outputs and popcounts may
    // name a constant directly: folding can reduce an output to ZERO)
    for (auto& kv : in_idx)
      s << "      const u64 " << v(kv.first) << " = " << (slow ? ld(kv.first, "w") : fast_in(kv.first, j)) << ";\n";
    auto opnd = [&](int o) -> std::string {
      if (!slow && is_const(nodes[o].op)) return fast_in(o, j);
      return v(o);
    };
    auto word_at = [&](int n, int64_t off) -> std::string {
      if (slow) return ld(n, "w + (" + std::to_string(off) + "ll)");
      if (tma) return ld(n, W + " + (" + std::to_string(off) + "ll)");
      return fast_off(n, off, j);
    };
    for (int n : emit_order) {
      const Node& x = nodes[n];
      const std::string a = x.a >= 0 ? opnd(x.a) : "", b = x.b >= 0 ? opnd(x.b) : "";
      const bool mask_here = slow && masked;
      switch (x.op) {
        case NOp::Not: s << "      const u64 " << v(n) << " = ~" << a << (mask_here ? " & lm" : "") << ";\n"; break;
        case NOp::And: s << "      const u64 " << v(n) << " = " << a << " & " << b << ";\n"; break;
        case NOp::Or: s << "      const u64 " << v(n) << " = " << a << " | " << b << ";\n"; break;
        case NOp::Xor: s << "      const u64 " << v(n) << " = " << a << " ^ " << b << ";\n"; break;
        case NOp::AndNot:
          s << "      const u64 " << v(n) << " = " << a << " & ~" << b << (mask_here ? " & lm" : "") << ";\n";
          break;
        case NOp::Add:
          if (mode == 't' && dyn[n])
            s << "      if (!res" << n << " && r >= max(" << dh(x.a) << ", " << dh(x.b) << ") && (" << a << " ^ " << b
              << ") != ~0ull) { res" << n << " = 1; dh" << n << " = r + 1; }\n";
          s << "      const u64 " << v(n) << " = addc(" << a << ", " << b << ", cy" << n << ")"
            << (mask_here ? " & lm" : "") << ";\n";
          break;
        case NOp::Shl: {
          const int64_t ws = x.k / 64;
          const int bs = static_cast<int>(x.k % 64);
          std::string e;
          if (x.k == 0) e = a;
          else if (ws == 0 && !is_const(nodes[x.a].op)) {
            if (shift_mul && bs != 32)
              e = "fshl_m<" + std::to_string(bs) + ">(" + a + ", pv" + std::to_string(x.a) + ", pm" +
                  std::to_string(bs % 32) + ")";
            else
              e = "fshl<" + std::to_string(bs) + ">(" + a + ", pv" + std::to_string(x.a) + ")";
          }
          else if (is_const(nodes[x.a].op)) {
            // a constant shifted left: word w is the constant's word w - ws (and w - ws - 1)
            const std::string lo = ld(x.a, W + " - " + std::to_string(ws) + "ll");
            e = bs ? "fshl<" + std::to_string(bs) + ">(" + lo + ", " + ld(x.a, W + " - " + std::to_string(ws + 1) + "ll") + ")" : lo;
          } else {
            const std::string lo = word_at(x.a, -ws);
            e = bs ? "fshl<" + std::to_string(bs) + ">(" + lo + ", " + word_at(x.a, -ws - 1) + ")" : lo;
          }
          s << "      const u64 " << v(n) << " = " << e << (mask_here ? " & lm" : "") << ";\n";
          break;
        }
        case NOp::Shr: {
          const int64_t ws = x.k / 64;
          const int bs = static_cast<int>(x.k % 64);
          std::string e;
          if (is_const(nodes[x.a].op)) {
            const std::string lo = ld(x.a, W + " + " + std::to_string(ws) + "ll");
            e = bs ? "fshr<" + std::to_string(bs) + ">(" + lo + ", " + ld(x.a, W + " + " + std::to_string(ws + 1) + "ll") + ")" : lo;
          } else {
            const std::string lo = word_at(x.a, ws);
            e = bs ? "fshr<" + std::to_string(bs) + ">(" + lo + ", " + word_at(x.a, ws + 1) + ")" : lo;
          }
          s << "      const u64 " << v(n) << " = " << e << ";\n";
          break;
        }
        default:
          throw RuntimeError("fused: unexpected node kind");
      }
      if (mode == 't' && dyn[n] && x.op != NOp::Add) {
        if (x.op == NOp::Shl && in_part.count(x.a) && x.k > 0)
          s << "      dh" << n << " = min(" << dh(x.a) << " + 1, 1 << 30);\n";
        else
          s << "      dh" << n << " = max(" << dh(x.a) << ", " << dh(x.b) << ");\n";
      }
    }
    // previous words for the next word's shifts (after every use in this word)
    for (int n : prev_src) s << "      pv" << n << " = " << (in_part.count(n) ? v(n) : opnd(n)) << ";\n";
  }

  std::string dh(int o) const {
    if (o < 0 || !in_part.count(o)) return "0";
    if (dyn[o]) return "dh" + std::to_string(o);
    auto it = sdh.find(o);
    return std::to_string(it == sdh.end() ? 0 : it->second);
  }

  std::string guard(int o) const {
    return guard_outputs ? "if (A.out[" + std::to_string(o) + "]) " : std::string();
  }
  void emit_store_word(std::ostringstream& s) const {
    for (auto& kv : outs) s << "      " << guard(kv.second) << "A.out[" << kv.second << "][w] = " << v(kv.first) << ";\n";
    for (size_t j = 0; j < part.pops.size(); ++j) s << "      pc" << j << " += __popcll(" << v(part.pops[j].first) << ");\n";
  }

  // Mapped inputs: every non-constant input of the part (in A.in order).
  void compute_mapped() {
    mapped.clear();
    for (auto& kv : in_idx)
      if (!is_const(nodes[kv.first].op)) mapped.push_back(kv.second);
    std::sort(mapped.begin(), mapped.end());
  }
  int box_bytes() const { return roww * 8 * 32; }
  // output staging: two sets of boxes (a chunk's stores drain while the next
  // chunk is computed) when they fit, else one
  int out_stages() const {
    const int two = warps * (stages * static_cast<int>(mapped.size()) + 2 * static_cast<int>(outs.size())) *
                    box_bytes() + 1024;
    return two <= 227 * 1024 ? 2 : 1;
  }
  // shared memory per warp: `stages` boxes per mapped input + staging boxes per output
  int smem_per_warp() const {
    return (stages * static_cast<int>(mapped.size()) + out_stages() * static_cast<int>(outs.size())) * box_bytes();
  }
  int smem_bytes() const { return warps * smem_per_warp() + 1024; }

  // Argument block of the TMA form: the tensor maps (128 bytes, 64-byte
  // aligned, one per mapped input then one per output) followed by the
  // plain form's fields and the number of threads whose ranges the maps cover.
  std::string tma_prelude(int ni, int no) const {
    std::ostringstream s;
    s << "struct __align__(64) TMap { unsigned long long w[16]; };\n"
      << "struct ArgsT {\n  TMap in_map[" << std::max<size_t>(1, mapped.size()) << "];\n  TMap out_map["
      << std::max(1, no) << "];\n  const u64* in[" << std::max(1, ni) << "];\n  u64* out[" << std::max(1, no)
      << "];\n  unsigned long long* slots;\n  unsigned int* fail;\n  long long nw;\n  long long range;\n"
      << "  u64 last_mask;\n  long long nfull;\n  unsigned long long one;\n};\n"
      << "__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }\n";
    return s.str();
  }

  // The owned range through TMA boxes (see the struct comment).  All lanes of
  // a warp walk the chunks together; lanes whose rows lie past the maps'
  // rows (the one thread with a short range, and idle threads) skip the
  // arithmetic, and the short range is done afterwards by the scalar path.
  void emit_tma_body(std::ostringstream& s) const {
    const int nm = static_cast<int>(mapped.size()), no = static_cast<int>(outs.size());
    const int box = box_bytes(), rowb = roww * 8;
    const std::string sw = roww == 4 ? "((lane >> 2) & 1)" : roww == 8 ? "((lane >> 1) & 3)" : "(lane & 7)";
    s << "  extern __shared__ __align__(1024) unsigned char smraw[];\n"
      << "  __shared__ __align__(8) unsigned long long bar[" << warps << "][" << stages << "];\n"
      << "  const int warp = threadIdx.x >> 5;\n"
      << "  unsigned char* sm = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);\n"
      << "  unsigned char* wb = sm + warp * " << smem_per_warp() << ";\n"
      << "  const long long t0 = tid - lane;\n"
      << "  const bool full = tid < A.nfull;\n"
      << "  const int sw = " << sw << ";\n"
      << "  if (t0 < A.nfull) {\n"
      << "    if (lane == 0) {\n"
      << "      for (int q = 0; q < " << stages << "; ++q) asm volatile(\"mbarrier.init.shared.b64 [%0], 1;\" :: \"r\"(smem_u32(&bar[warp][q])));\n"
      << "      asm volatile(\"fence.mbarrier_init.release.cluster;\" ::: \"memory\");\n"
      << "    }\n    __syncwarp();\n"
      << "    const int nch = (int)(A.range / " << roww << ");\n"
      << "    auto issue = [&](int ch, int q) {\n"
      << "      asm volatile(\"fence.proxy.async.shared::cta;\" ::: \"memory\");\n"
      << "      __syncwarp();\n"
      << "      if (lane == 0) {\n"
      << "        const unsigned mb = smem_u32(&bar[warp][q]);\n"
      << "        asm volatile(\"mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;\" :: \"r\"(mb), \"r\"(" << nm * box
      << ") : \"memory\");\n";
    for (int k = 0; k < nm; ++k)
      s << "        asm volatile(\"cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
           "[%0], [%1, {%2, %3, %4}], [%5];\" :: \"r\"(smem_u32(wb + (q * "
        << nm << " + " << k << ") * " << box << ")), \"l\"(&A.in_map[" << k
        << "]), \"r\"(0), \"r\"(ch), \"r\"((int)t0), \"r\"(mb) : \"memory\");\n";
    s << "      }\n    };\n"
      << "    int issued = 0;\n"
      << "    for (; issued < " << stages - 1 << " && issued < nch; ++issued) issue(issued, issued % " << stages << ");\n"
      << "    unsigned phase = 0;\n    bool bail = false;\n    int waited = 0;\n"
      << "    for (int ch = 0; ch < nch && !bail; ++ch) {\n"
      << "      const int q = ch % " << stages << ";\n"
      << "      if (issued < nch) { issue(issued, issued % " << stages << "); ++issued; }\n"
      // bounded wait; a stage that never lands sets the fail flag (the host
      // then re-runs the part with the exact per-op kernels)
      << "      {\n        const unsigned mb = smem_u32(&bar[warp][q]);\n        unsigned done = 0;\n"
      << "        for (int it = 0; it < (1 << 22) && !done; ++it)\n"
      << "          asm volatile(\"{ .reg .pred p; mbarrier.try_wait.parity.shared.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }\" "
         ": \"=r\"(done) : \"r\"(mb), \"r\"((phase >> q) & 1u) : \"memory\");\n"
      << "        if (!__all_sync(~0u, done)) { if (lane == 0) atomicOr(A.fail, 2u); bail = true; break; }\n"
      << "        phase ^= 1u << q;\n        ++waited;\n      }\n"
      // the staging set this chunk writes must have been read by its last
      // stores: with two sets, the previous chunk's stores may still run
      << "      if (lane == 0) asm volatile(\"cp.async.bulk.wait_group.read " << (out_stages() - 1)
      << ";\" ::: \"memory\");\n"
      << "      __syncwarp();\n"
      << "      const long long w0 = s + (long long)ch * " << roww << ";\n"
      << "      unsigned char* ib = wb + q * " << nm * box << " + lane * " << rowb << ";\n"
      << "      unsigned char* obase = wb + " << stages * nm * box << " + " << (out_stages() == 2 ? "(ch & 1) * " + std::to_string(no * box) : std::string("0")) << ";\n"
      << "      unsigned char* ob = obase + lane * " << rowb << ";\n"
      << "      if (full) {\n"
      << "        if (" << (masked ? "w0 + " + std::to_string(roww) + " <= A.nw - 1" : std::string("true")) << ") {\n"
      << (unroll_pairs ? "#pragma unroll\n" : "#pragma unroll 1\n")
      << "          for (int pp = 0; pp < " << roww / 2 << "; ++pp) {\n"
      << "            const long long c = w0 + 2 * pp;\n"
      << "            const int po = (pp ^ sw) * 16;\n";
    for (int k = 0; k < nm; ++k) {
      const std::string i = std::to_string(mapped[k]);
      s << "            const ulonglong2 q" << i << " = *reinterpret_cast<const ulonglong2*>(ib + " << k * box
        << " + po);\n            const u64 c" << i << "_0 = q" << i << ".x, c" << i << "_1 = q" << i << ".y;\n";
    }
    for (int j = 0; j < 2; ++j) {
      s << "            u64 ";
      bool first = true;
      for (auto& kv : outs) {
        s << (first ? "" : ", ") << "r" << kv.second << "_" << j;
        first = false;
      }
      if (outs.empty()) s << "unused_" << j;
      s << ";\n            {\n";
      emit_word(s, 'f', j);
      for (auto& kv : outs) s << "      r" << kv.second << "_" << j << " = " << v(kv.first) << ";\n";
      for (size_t qq = 0; qq < part.pops.size(); ++qq)
        s << "      pc" << qq << " += __popcll(" << v(part.pops[qq].first) << ");\n";
      s << "            }\n";
    }
    for (auto& kv : outs)
      s << "            *reinterpret_cast<ulonglong2*>(ob + " << kv.second * box << " + po) = make_ulonglong2(r"
        << kv.second << "_0, r" << kv.second << "_1);\n";
    s << "          }\n        } else {\n"
      << "          for (long long w = w0; w < w0 + " << roww << "; ++w) {\n"
      << "            const int jj = (int)(w - w0);\n"
      << "            const int wo = ((jj >> 1) ^ sw) * 16 + (jj & 1) * 8;\n"
      << "            {\n";
    emit_word(s, 's', 0);
    for (auto& kv : outs)
      s << "      *reinterpret_cast<u64*>(ob + " << kv.second * box << " + wo) = " << v(kv.first) << ";\n";
    for (size_t qq = 0; qq < part.pops.size(); ++qq)
      s << "      pc" << qq << " += __popcll(" << v(part.pops[qq].first) << ");\n";
    s << "            }\n          }\n        }\n      }\n"
      << "      asm volatile(\"fence.proxy.async.shared::cta;\" ::: \"memory\");\n"
      << "      __syncwarp();\n"
      << "      if (lane == 0) {\n";
    for (int o = 0; o < no; ++o)
      s << "        asm volatile(\"cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];\" "
           ":: \"l\"(&A.out_map[" << o << "]), \"r\"(0), \"r\"(ch), \"r\"((int)t0), \"r\"(smem_u32(obase + "
        << o * box << ")) : \"memory\");\n";
    s << "        asm volatile(\"cp.async.bulk.commit_group;\" ::: \"memory\");\n"
      << "      }\n      __syncwarp();\n    }\n"
      // after a bail-out: wait (bounded) for the loads still in flight
      << "    if (bail) {\n"
      << "      for (int ch = waited; ch < issued; ++ch) {\n"
      << "        const int q = ch % " << stages << ";\n        const unsigned mb = smem_u32(&bar[warp][q]);\n"
      << "        unsigned done = 0;\n"
      << "        for (int it = 0; it < (1 << 22) && !done; ++it)\n"
      << "          asm volatile(\"{ .reg .pred p; mbarrier.test_wait.parity.shared.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }\" "
         ": \"=r\"(done) : \"r\"(mb), \"r\"((phase >> q) & 1u) : \"memory\");\n"
      << "        phase ^= 1u << q;\n      }\n    }\n"
      << "    if (lane == 0) asm volatile(\"cp.async.bulk.wait_group 0;\" ::: \"memory\");\n"
      << "  }\n"
      // the range past the maps' rows: scalar path, stores to global
      << "  if (active && !full) {\n    for (long long w = s; w < e; ++w) {\n      {\n";
    emit_word(s, 's', 0);
    emit_store_word(s);
    s << "      }\n    }\n  }\n";
  }

  std::string source() {
    analyze();
    compute_mapped();
    std::ostringstream s;
    const int ni = static_cast<int>(part.inputs.size()), no = static_cast<int>(part.outputs.size());
    s << Gen::args_struct(ni, no) << helpers();
    emit_kernel(s, ni, no);
    return s.str();
  }

  // Device helpers shared by every thread-sequential kernel / device function.
  static std::string helpers() {
    std::ostringstream s;
    s << "// funnel shift left by s in (0, 32) as multiplies, m = 2^s held in a register\n"
         "// the compiler cannot fold: (hi << s) | (lo >> (32 - s)) = hi * m + mulhi(lo, m),\n"
         "// two integer multiply-adds instead of a funnel shift on the logic pipe\n"
         "__device__ __forceinline__ u32 fmul_funnel(u32 lo, u32 hi, u32 m) {\n"
         "  u32 d;\n"
         "  asm(\"{ .reg .u32 t; mul.hi.u32 t, %1, %3; mad.lo.u32 %0, %2, %3, t; }\" : \"=r\"(d) : \"r\"(lo), \"r\"(hi), \"r\"(m));\n"
         "  return d;\n}\n"
         "template <int K> __device__ __forceinline__ u64 fshl_m(u64 x, u64 p, u32 m) {\n"
         "  const u32 xl = (u32)x, xh = (u32)(x >> 32), pl = (u32)p, ph = (u32)(p >> 32);\n"
         "  u32 lo, hi;\n"
         "  if constexpr (K < 32) { lo = fmul_funnel(ph, xl, m); hi = fmul_funnel(xl, xh, m); }\n"
         "  else if constexpr (K == 32) { lo = ph; hi = xl; }\n"
         "  else { lo = fmul_funnel(pl, ph, m); hi = fmul_funnel(ph, xl, m); }\n"
         "  return ((u64)hi << 32) | lo;\n}\n";
    s << "template <int K> __device__ __forceinline__ u64 fshl(u64 x, u64 p) {\n"
         "  const u32 xl = (u32)x, xh = (u32)(x >> 32), pl = (u32)p, ph = (u32)(p >> 32);\n"
         "  u32 lo, hi;\n"
         "  if constexpr (K < 32) { lo = __funnelshift_l(ph, xl, K); hi = __funnelshift_l(xl, xh, K); }\n"
         "  else if constexpr (K == 32) { lo = ph; hi = xl; }\n"
         "  else { lo = __funnelshift_l(pl, ph, K - 32); hi = __funnelshift_l(ph, xl, K - 32); }\n"
         "  return ((u64)hi << 32) | lo;\n}\n"
         "template <int K> __device__ __forceinline__ u64 fshr(u64 x, u64 nx) {\n"
         "  const u32 xl = (u32)x, xh = (u32)(x >> 32), nl = (u32)nx, nh = (u32)(nx >> 32);\n"
         "  u32 lo, hi;\n"
         "  if constexpr (K < 32) { lo = __funnelshift_r(xl, xh, K); hi = __funnelshift_r(xh, nl, K); }\n"
         "  else if constexpr (K == 32) { lo = xh; hi = nl; }\n"
         "  else { lo = __funnelshift_r(xh, nl, K - 32); hi = __funnelshift_r(nl, nh, K - 32); }\n"
         "  return ((u64)hi << 32) | lo;\n}\n"
         "__device__ __forceinline__ u64 addc(u64 a, u64 b, u32& c) {\n"
         "  u32 lo, hi, co;\n"
         "  asm(\"{ .reg .u32 t;\\n\\tadd.cc.u32 t, %3, 0xffffffff;\\n\\taddc.cc.u32 %0, %4, %6;\\n\\t\"\n"
         "      \"addc.cc.u32 %1, %5, %7;\\n\\taddc.u32 %2, 0, 0;\\n\\t}\"\n"
         "      : \"=&r\"(lo), \"=&r\"(hi), \"=r\"(co)\n"
         "      : \"r\"(c), \"r\"((u32)a), \"r\"((u32)(a >> 32)), \"r\"((u32)b), \"r\"((u32)(b >> 32)));\n"
         "  c = co;\n  return ((u64)hi << 32) | lo;\n}\n"
         "__device__ __forceinline__ void ld4(const u64* p, u64& a, u64& b, u64& c, u64& d) {\n"
         "  asm volatile(\"ld.global.nc.L2::128B.v4.u64 {%0,%1,%2,%3}, [%4];\" : \"=l\"(a), \"=l\"(b), \"=l\"(c), \"=l\"(d) : \"l\"(p));\n}\n"
         "__device__ __forceinline__ void st4(u64* p, u64 a, u64 b, u64 c, u64 d) {\n"
         "  asm volatile(\"st.global.v4.u64 [%0], {%1,%2,%3,%4};\" :: \"l\"(p), \"l\"(a), \"l\"(b), \"l\"(c), \"l\"(d) : \"memory\");\n}\n";
    return s.str();
  }

  // The kernel (or, with `fn_name`, the batch device function for one work
  // item [s_item, e_item) of one instance, split into 32 lane ranges).
  void emit_kernel(std::ostringstream& s, int ni, int no, const std::string& fn_name = "") const {
    if (!fn_name.empty()) {
      s << "__device__ __noinline__ void " << fn_name
        << "(const Args* __restrict__ Ap, const long long s_item, const long long e_item, const int lane) {\n"
        << "  const Args& A = *Ap;\n"
        << "  const long long L = (((e_item - s_item) + 31) / 32 + " << reg_chunk - 1 << ") / " << reg_chunk << " * "
        << reg_chunk << ";\n"
        << "  const long long s = s_item + lane * L;\n"
        << "  const bool active = s < e_item;\n"
        << "  const long long e = min(s + L, e_item);\n";
    } else if (tma) {
      s << tma_prelude(ni, no);
      s << "extern \"C\" __global__ void __launch_bounds__(" << warps * 32 << ", 1)\n"
        << "bsz_fused(const __grid_constant__ ArgsT A) {\n";
    } else {
      s << "extern \"C\" __global__ void __launch_bounds__(" << warps * 32 << ", " << min_blocks
        << ")\nbsz_fused(const Args A) {\n";
    }
    if (fn_name.empty())
      s << "  const int lane = threadIdx.x & 31;\n"
        << "  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;\n"
        << "  const long long s = tid * A.range;\n"
        << "  const bool active = s < A.nw;\n"
        << "  const long long e = min(s + A.range, A.nw);\n";
    std::vector<int> adds;
    for (int n : part.order)
      if (nodes[n].op == NOp::Add) adds.push_back(n);
    if (shift_mul) {
      std::set<int> amounts;
      for (int n : part.order) {
        const Node& x = nodes[n];
        if (x.op == NOp::Shl && x.k > 0 && x.k < 64 && x.k != 32 && !is_const(nodes[x.a].op))
          amounts.insert(static_cast<int>(x.k % 32));
      }
      for (int k : amounts) s << "  const u32 pm" << k << " = (u32)(A.one << " << k << ");\n";
    }
    for (int n : adds) s << "  u32 cy" << n << " = 0;\n";
    for (int n : prev_src) s << "  u64 pv" << n << " = 0;\n";
    for (size_t j = 0; j < part.pops.size(); ++j) s << "  u32 pc" << j << " = 0;\n";
    s << "  if (active) {\n";
    // ---- warm-up
    if (!adds.empty() || !prev_src.empty()) {
      s << "  long long p0 = s - " << warm << "ll;\n  if (p0 < 0) p0 = 0;\n"
        << "  for (int attempt = 0; p0 < s; ++attempt) {\n";
      for (int n : adds) s << "    cy" << n << " = 0;\n";
      for (int n : prev_src) s << "    pv" << n << " = 0;\n";
      for (int n : adds)
        if (dyn[n]) s << "    int res" << n << " = (p0 == 0);\n    int dh" << n << " = (p0 == 0) ? 0 : (1 << 30);\n";
      for (int n : part.order)
        if (dyn[n] && nodes[n].op != NOp::Add) s << "    int dh" << n << " = 0;\n";
      s << "    for (long long w = p0; w < s; ++w) {\n      const int r = (int)(w - p0);\n";
      emit_word(s, 't', 0);
      s << "    }\n    const int need = (int)(s - p0);\n    bool ok = true;\n";
      for (int n : adds)
        if (dyn[n]) s << "    ok = ok && res" << n << " && dh" << n << " <= need;\n";
      for (int n : prev_src) {
        if (!in_part.count(n)) continue;
        if (dyn[n]) s << "    ok = ok && dh" << n << " <= need - 1;\n";
        else if (sdh.count(n) && sdh.at(n) > 0) s << "    ok = ok && " << sdh.at(n) << " <= need - 1;\n";
      }
      s << "    if (ok || p0 == 0) break;\n"
        << "    if (attempt >= 8) { atomicOr(A.fail, 1u); break; }\n"
        << "    p0 = s - 2 * (s - p0);\n    if (p0 < 0) p0 = 0;\n"
        << "  }\n";
    }
    if (tma) {
      s << "  }\n";   // active (warm-up)
      emit_tma_body(s);
    } else {
    // ---- owned range
    const int CW = reg_chunk;
    const int pad = static_cast<int>(fast_hi_pad) + (masked && fast_hi_pad == 3 ? 1 : 0) + (CW - 4);
    s << "  long long w = s;\n"
      << "  const long long fast_end = A.nw - 1 - " << pad << "ll;   // a fast chunk at c needs c <= fast_end\n"
      << "  while (w < e) {\n"
      << "    if (w + " << CW << " <= e && w >= " << fast_lo << "ll && w <= fast_end) {\n"
      << "      const long long c = w;\n";
    for (auto& kv : in_idx) {
      if (is_const(nodes[kv.first].op)) continue;
      const std::string i = std::to_string(kv.second);
      for (int h = 0; h < CW; h += 4)
        s << "      u64 c" << i << "_" << h << ", c" << i << "_" << h + 1 << ", c" << i << "_" << h + 2 << ", c" << i
          << "_" << h + 3 << ";\n"
          << "      ld4(A.in[" << i << "] + c + " << h << ", c" << i << "_" << h << ", c" << i << "_" << h + 1 << ", c"
          << i << "_" << h + 2 << ", c" << i << "_" << h + 3 << ");\n";
    }
    for (auto& kv : off_slot) {
      const int n = kv.first.first;
      const int64_t base = slot_base(kv.first.second);
      const std::string sl = std::to_string(kv.second), i = std::to_string(in_idx.at(n));
      for (int h = 0; h < CW + 4; h += 4)
        s << "      u64 o" << sl << "_" << h << ", o" << sl << "_" << h + 1 << ", o" << sl << "_" << h + 2 << ", o" << sl
          << "_" << h + 3 << ";\n"
          << "      ld4(A.in[" << i << "] + c + (" << base + h << "ll), o" << sl << "_" << h << ", o" << sl << "_"
          << h + 1 << ", o" << sl << "_" << h + 2 << ", o" << sl << "_" << h + 3 << ");\n";
    }
    for (int j = 0; j < CW; ++j) {
      s << "      u64 ";
      bool first = true;
      for (auto& kv : outs) {
        s << (first ? "" : ", ") << "r" << kv.second << "_" << j;
        first = false;
      }
      if (outs.empty()) s << "unused_" << j;
      s << ";\n      {\n";
      emit_word(s, 'f', j);
      for (auto& kv : outs) s << "      r" << kv.second << "_" << j << " = " << v(kv.first) << ";\n";
      for (size_t q = 0; q < part.pops.size(); ++q)
        s << "      pc" << q << " += __popcll(" << v(part.pops[q].first) << ");\n";
      s << "      }\n";
    }
    for (auto& kv : outs) {
      const std::string o = std::to_string(kv.second);
      for (int h = 0; h < CW; h += 4)
        s << "      " << guard(kv.second) << "st4(A.out[" << o << "] + c + " << h << ", r" << o << "_" << h << ", r" << o
          << "_" << h + 1 << ", r" << o << "_" << h + 2 << ", r" << o << "_" << h + 3 << ");\n";
    }
    s << "      w += " << CW << ";\n    } else {\n      {\n";
    emit_word(s, 's', 0);
    emit_store_word(s);
    s << "      }\n      ++w;\n    }\n  }\n";
    s << "  }\n";   // active
    }
    for (size_t j = 0; j < part.pops.size(); ++j) {
      s << "  {\n    unsigned long long t = pc" << j << ";\n"
        << "    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(~0u, t, o);\n"
        << "    if (lane == 0 && t) atomicAdd(A.slots + " << part.pops[j].second << ", t);\n  }\n";
    }
    s << "}\n";
  }

  // Batch device function (register chunks; see emit_kernel).
  std::string device_function(const std::string& name) {
    analyze();
    std::ostringstream s;
    emit_kernel(s, 0, 0, name);
    return s.str();
  }
};

// On-disk cache of compiled kernels, so that short-lived processes (the
// bsim_cuda driver runs once per test case) do not recompile: directory
// $BSZ_KERNEL_CACHE (or ~/.cache/bitstreamzoo_b200; "off" disables), files
// <hash>.cubin next to <hash>.cu holding the full source, which is compared
// on load so a hash collision can never return the wrong kernel.
std::string cache_dir() {
  const char* env = std::getenv("BSZ_KERNEL_CACHE");
  if (env && !std::strcmp(env, "off")) return "";
  std::string d;
  if (env && *env) d = env;
  else if (const char* home = std::getenv("HOME")) d = std::string(home) + "/.cache/bitstreamzoo_b200";
  else return "";
  std::string cur;
  for (size_t i = 0; i <= d.size(); ++i) {   // mkdir -p
    if (i == d.size() || d[i] == '/') {
      if (!cur.empty()) mkdir(cur.c_str(), 0755);
    }
    if (i < d.size()) cur += d[i];
  }
  return d;
}

std::string cache_key(const std::string& src) {
  uint64_t h = 1469598103934665603ull;   // FNV-1a over the source and the target
  for (char c : src + "|sm_100a|nvrtc-12") h = (h ^ static_cast<unsigned char>(c)) * 1099511628211ull;
  char buf[32];
  std::snprintf(buf, sizeof buf, "%016llx", static_cast<unsigned long long>(h));
  return buf;
}

std::string read_file(const std::string& path) {
  std::string out;
  if (FILE* f = std::fopen(path.c_str(), "rb")) {
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, n);
    std::fclose(f);
  }
  return out;
}

std::string disk_cache_load(const std::string& src) {
  const std::string dir = cache_dir();
  if (dir.empty()) return "";
  const std::string base = dir + "/" + cache_key(src);
  if (read_file(base + ".cu") != src) return "";
  return read_file(base + ".cubin");
}

void disk_cache_store(const std::string& src, const std::string& cubin) {
  const std::string dir = cache_dir();
  if (dir.empty()) return;
  const std::string base = dir + "/" + cache_key(src);
  const std::string tag = "." + std::to_string(getpid());
  for (const auto& [ext, data] : {std::pair<std::string, const std::string*>{".cubin", &cubin},
                                  {".cu", &src}}) {
    const std::string tmp = base + ext + tag;
    if (FILE* f = std::fopen(tmp.c_str(), "wb")) {
      std::fwrite(data->data(), 1, data->size(), f);
      std::fclose(f);
      std::rename(tmp.c_str(), (base + ext).c_str());
    }
  }
}

// True when `src` is compiled in this process or present in the disk cache.
bool is_compiled(const std::string& src) {
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (cache().count(src_digest(src))) return true;
  }
  const std::string dir = cache_dir();
  if (dir.empty()) return false;
  const std::string base = dir + "/" + cache_key(src);
  FILE* f = std::fopen((base + ".cubin").c_str(), "rb");
  if (!f) return false;
  std::fclose(f);
  return read_file(base + ".cu") == src;
}

Compiled compile_source(const std::string& src, int block_threads, double* compile_ms,
                        const char* kernel = "bsz_fused") {
  const std::string digest = src_digest(src);
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = cache().find(digest);
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
  // warnings 550/177: warm-up steps compute values only the owned range stores
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device",
                        "--extra-device-vectorization", "--diag-suppress=550,177"};
  std::string cubin = disk_cache_load(src);
  if (cubin.empty()) {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "bsz_fused.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
      throw RuntimeError("nvrtcCreateProgram failed");
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
    cubin.assign(cubin_size, '\0');
    nvrtcGetCUBIN(prog, &cubin[0]);
    nvrtcDestroyProgram(&prog);
    disk_cache_store(src, cubin);
  }
  Compiled c;
  BSZ_CU(drv().module_load_data(&c.mod, cubin.data()));
  BSZ_CU(drv().module_get_function(&c.fn, c.mod, kernel));
  drv().func_get_attribute(&c.n_regs, CU_FUNC_ATTRIBUTE_NUM_REGS, c.fn);
  if (drv().occupancy(&c.blocks_per_sm, c.fn, block_threads, 0) != CUDA_SUCCESS || c.blocks_per_sm < 1)
    c.blocks_per_sm = 1;
  if (compile_ms)
    *compile_ms += std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
  std::lock_guard<std::mutex> lk(g_cache_mu);
  cache()[digest] = c;
  return c;
}

// Splits a segment into parts: a node that reads a temporary through a right
// shift, or through a left shift of 64 * shl_cut_words bits or more (2048 in
// the warp form, 64 in the thread-sequential form), starts a later part, and
// that temporary becomes an output of its own part.  Carry schemes
// (cut_adds): 0, every addition inside the generated kernel (speculative
// carry state); 1, the same, with every addition's result materialized; 2,
// every addition of two streams is a part of its own run by the plain
// carry-scan kernel (decoupled look-back), its operands and result
// materialized.
std::vector<Part> split(const std::vector<Node>& nodes, const Segment& seg, int cut_adds,
                        int64_t shl_cut_words = 32) {
  std::map<int, int> level;
  std::set<int> computed(seg.order.begin(), seg.order.end());
  std::set<int> cut_src;
  for (int n : seg.order) {
    const Node& x = nodes[n];
    int lv = 0;
    for (int o : {x.a, x.b}) {
      if (o < 0 || !computed.count(o)) continue;
      int l = level[o];
      bool cut = (x.op == NOp::Shr) || (x.op == NOp::Shl && x.k / 64 >= shl_cut_words) ||
                 (cut_adds && nodes[o].op == NOp::Add) || (cut_adds == 2 && x.op == NOp::Add);
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
  std::vector<std::vector<int>> adds_at(max_lv + 1);
  for (int n : seg.order) {
    // carry scheme 2: an addition reads only materialized operands and is
    // read only from memory, so it shares its level with nothing it depends
    // on or that depends on it, and leaves that level's kernel
    if (cut_adds == 2 && nodes[n].op == NOp::Add) adds_at[level[n]].push_back(n);
    else parts[level[n]].order.push_back(n);
  }
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
  std::map<int, std::vector<std::pair<int, int64_t>>> add_pops;
  for (auto& pp : seg.pops) {
    if (cut_adds == 2 && computed.count(pp.first) && nodes[pp.first].op == NOp::Add) {
      add_pops[pp.first].push_back(pp);
      continue;
    }
    int L = computed.count(pp.first) ? level[pp.first] : 0;
    Part& p = parts[L];
    p.pops.push_back(pp);
    if (!computed.count(pp.first) &&
        std::find(p.inputs.begin(), p.inputs.end(), pp.first) == p.inputs.end())
      p.inputs.push_back(pp.first);
  }
  if (cut_adds != 2) return parts;
  std::vector<Part> out;
  for (int L = 0; L <= max_lv; ++L) {
    for (int n : adds_at[L]) {
      Part a;
      a.lookback_add = true;
      a.order = {n};
      a.inputs = {nodes[n].a, nodes[n].b};
      a.outputs = {n};
      a.pops = add_pops[n];
      out.push_back(std::move(a));
    }
    out.push_back(std::move(parts[L]));
  }
  return out;
}

}  // namespace

namespace {

// Generating a part's source costs tens of microseconds per run; a compact
// key of everything the generator reads (the part's nodes, its inputs'
// kinds and tails, outputs, popcount slots, masking and schedule) maps a
// repeated part straight to its compiled kernel and warm-up length.
struct PartKernel {
  Compiled c;
  int64_t warm = 0;
  // TMA form: chunk words, dynamic shared memory, resident CTAs per SM at
  // that size, and the A.in indices read through tensor maps (in map order)
  int roww = 0;
  int smem = 0;
  int tma_blocks_per_sm = 0;
  std::vector<int> mapped;
};
std::mutex g_part_mu;
std::unordered_map<std::string, PartKernel>& part_cache() {
  static std::unordered_map<std::string, PartKernel> m;
  return m;
}

// Key of a node list as the generator reads it: ids, kind, tail,
// cleanliness, operands, shift amount; then outputs, popcount slots,
// masking and the schedule.
std::string graph_key(const std::vector<Node>& nodes, const std::vector<int>& order, const std::vector<int>& inputs,
                      const std::vector<int>& outputs, const std::vector<std::pair<int, int64_t>>& pops,
                      bool masked, const Schedule& sc) {
  std::string k;
  k.reserve(40 * (order.size() + inputs.size()) + 16 * pops.size() + 8 * outputs.size() + 64);
  auto put = [&](int64_t v) { k.append(reinterpret_cast<const char*>(&v), sizeof v); };
  auto node = [&](int n) {
    const Node& x = nodes[n];
    put(n);
    put(static_cast<int64_t>(x.op) | (static_cast<int64_t>(x.tail) << 8) | (static_cast<int64_t>(x.clean) << 16));
    put(x.a);
    put(x.b);
    put(x.k);
  };
  put(static_cast<int64_t>(order.size()));
  for (int n : order) node(n);
  put(static_cast<int64_t>(inputs.size()));
  for (int n : inputs) node(n);
  put(static_cast<int64_t>(outputs.size()));
  for (int n : outputs) put(n);
  put(static_cast<int64_t>(pops.size()));
  for (auto& q : pops) {
    put(q.first);
    put(q.second);
  }
  put(masked);
  put(sc.warps);
  put(sc.min_blocks);
  put(sc.prefetch);
  put(sc.cut_adds);
  put(sc.layout);
  put(sc.chunk_words);
  put(sc.stages);
  put(sc.unroll);
  put(sc.shift_mul);
  return k;
}

std::string part_key(const std::vector<Node>& nodes, const Part& p, bool masked, const Schedule& sc) {
  return graph_key(nodes, p.order, p.inputs, p.outputs, p.pops, masked, sc);
}

// A segment's launch plan: its parts (split) with their kernels, keyed by
// the segment's graph, so a segment seen before is neither split nor keyed
// part by part again.
struct SegPlan {
  std::vector<Part> parts;
  std::vector<PartKernel> kernels;
};
constexpr size_t kMaxPlans = 4096;
std::mutex g_plan_mu;
std::unordered_map<std::string, std::shared_ptr<const SegPlan>>& plan_cache() {
  static std::unordered_map<std::string, std::shared_ptr<const SegPlan>> m;
  return m;
}

PartKernel part_kernel(const std::vector<Node>& nodes, const Part& p, int64_t N, const Schedule& sc,
                       double* compile_ms) {
  const std::string key = part_key(nodes, p, (N % 64) != 0, sc);
  {
    std::lock_guard<std::mutex> lk(g_part_mu);
    auto it = part_cache().find(key);
    if (it != part_cache().end()) return it->second;
  }
  PartKernel pk;
  // the TMA form's argument block holds a 128-byte tensor map per read input
  // and per output; past 24 of them the part takes the register form
  int n_maps = static_cast<int>(p.outputs.size());
  for (int n : p.inputs)
    if (!is_const(nodes[n].op)) ++n_maps;
  if (sc.layout == 2 && n_maps > 24) {
    Schedule s1 = sc;
    s1.layout = 1;
    s1.min_blocks = 1;
    return part_kernel(nodes, p, N, s1, compile_ms);
  }
  if (sc.layout == 2) {
    GenSeq g{nodes, p, N, sc.warps, 1, (N % 64) != 0};
    g.tma = true;
    g.roww = sc.chunk_words == 4 ? 4 : 8;
    g.stages = sc.stages == 3 ? 3 : 2;
    g.unroll_pairs = sc.unroll != 0;
    g.shift_mul = sc.shift_mul != 0;
    const std::string src = g.source();
    pk.c = compile_source(src, sc.warps * 32, compile_ms);
    pk.warm = g.warm;
    pk.roww = g.roww;
    pk.smem = g.smem_bytes();
    pk.mapped = g.mapped;
    if (pk.smem > 227 * 1024 ||
        drv().func_set_attribute(pk.c.fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, pk.smem) != CUDA_SUCCESS ||
        drv().occupancy(&pk.tma_blocks_per_sm, pk.c.fn, sc.warps * 32, pk.smem) != CUDA_SUCCESS ||
        pk.tma_blocks_per_sm < 1) {
      // the boxes of this part do not fit in one SM's shared memory at this
      // CTA size: the part takes the register form
      Schedule s1 = sc;
      s1.layout = 1;
      s1.min_blocks = 1;
      return part_kernel(nodes, p, N, s1, compile_ms);
    }
  } else if (sc.layout == 1) {
    GenSeq g{nodes, p, N, sc.warps, sc.min_blocks, (N % 64) != 0};
    g.shift_mul = sc.shift_mul != 0;
    g.reg_chunk = sc.chunk_words == 8 ? 8 : 4;
    pk.c = compile_source(g.source(), sc.warps * 32, compile_ms);
    pk.warm = g.warm;
  } else {
    Gen g{nodes, p, N, sc.warps, sc.min_blocks, (N % 64) != 0, sc.prefetch != 0};
    pk.c = compile_source(g.source(), sc.warps * 32, compile_ms);
    pk.warm = g.warm;
  }
  std::lock_guard<std::mutex> lk(g_part_mu);
  part_cache()[key] = pk;
  return pk;
}

}  // namespace

// A launched segment whose speculation flags have not been read yet: its
// parts, a copy of every node they compute or read (with the buffers, so
// none returns to the cache while a re-run may need it) and where its
// popcounts go.
struct PendingSegment {
  std::shared_ptr<const void> plan;          // keeps `parts` alive
  const std::vector<Part>* parts = nullptr;
  std::unordered_map<int, Node> nodes;
  int64_t N = 0, nw = 0;
  unsigned long long* d_slots = nullptr;
  std::string spec_key;   // non-empty: the segment ran with speculative carries (scheme 0)
};

// Segments (graph and schedule keys) whose speculative carry state could not
// be proven once: whether it can depends on how the DAG correlates the
// operands of its additions, so the next run of the same segment would most
// likely fail again and pay for the exact re-run.  Such a segment runs its
// additions with the look-back carry scan (carry scheme 2) from then on.
std::mutex g_spec_mu;
std::unordered_set<std::string>& spec_failed() {
  static std::unordered_set<std::string> s;
  return s;
}

struct FusedBackend::Impl {
  Device& dev;
  ExecOptions opt;
  BufRef fail_buf;   // from the device's buffer cache: no cudaMalloc/cudaFree per run
  unsigned int* d_fail = nullptr;   // one flag per part of the launched segment
  int64_t fail_cap = 0;
  std::unique_ptr<PendingSegment> pending;
  Impl(Device& d, const ExecOptions& o) : dev(d), opt(o) { ensure_flags(64); }
  void ensure_flags(int64_t n) {
    if (n <= fail_cap) return;
    fail_cap = std::max<int64_t>(n, 2 * fail_cap);
    fail_buf = dev.alloc_stream((fail_cap + 1) / 2);
    d_fail = reinterpret_cast<unsigned int*>(fail_buf->p);
  }
};

FusedBackend::FusedBackend(Device& dev, const ExecOptions& opt)
    : impl_(std::make_unique<Impl>(dev, opt)) {}
FusedBackend::~FusedBackend() = default;

void FusedBackend::set_schedule(const Schedule& s) {
  Schedule c = s;
  c.warps = std::max(1, std::min(c.warps, 16));
  c.range_steps = std::max(1, c.range_steps);
  c.ctas_per_sm = std::max(-1, c.ctas_per_sm);
  c.min_blocks = std::max(1, std::min(c.min_blocks, 32));
  c.layout = std::max(0, std::min(c.layout, 2));
  c.cut_adds = std::max(0, std::min(c.cut_adds, 2));
  c.chunk_words = c.chunk_words == 8 ? 8 : 4;
  c.stages = c.stages == 3 ? 3 : 2;
  c.unroll = c.unroll ? 1 : 0;
  c.shift_mul = c.shift_mul ? 1 : 0;
  impl_->opt.sched = c;
}

bool FusedBackend::all_compiled(const std::vector<Node>& nodes, const Segment& seg, int64_t N) {
  const Schedule& sc = impl_->opt.sched;
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    if (plan_cache().count(graph_key(nodes, seg.order, seg.inputs, seg.outputs, seg.pops, (N % 64) != 0, sc)))
      return true;
  }
  std::vector<Part> parts = split(nodes, seg, sc.cut_adds, sc.layout >= 1 ? 1 : 32);
  for (Part& p : parts) {
    if ((p.order.empty() && p.pops.empty()) || p.lookback_add) continue;
    if (p.inputs.size() > kMaxInputs) return false;
    {
      std::lock_guard<std::mutex> lk(g_part_mu);
      if (part_cache().count(part_key(nodes, p, (N % 64) != 0, sc))) continue;
    }
    if (sc.layout == 2) {
      GenSeq g{nodes, p, N, sc.warps, 1, (N % 64) != 0};
      g.tma = true;
      g.roww = sc.chunk_words == 4 ? 4 : 8;
      g.stages = sc.stages == 3 ? 3 : 2;
      g.unroll_pairs = sc.unroll != 0;
      g.shift_mul = sc.shift_mul != 0;
      if (!is_compiled(g.source())) return false;
    } else if (sc.layout == 1) {
      GenSeq g{nodes, p, N, sc.warps, sc.min_blocks, (N % 64) != 0};
      g.shift_mul = sc.shift_mul != 0;
      g.reg_chunk = sc.chunk_words == 8 ? 8 : 4;
      if (!is_compiled(g.source())) return false;
    } else {
      Gen g{nodes, p, N, sc.warps, sc.min_blocks, (N % 64) != 0, sc.prefetch != 0};
      if (!is_compiled(g.source())) return false;
    }
  }
  return true;
}


void FusedBackend::run(std::vector<Node>& nodes, const Segment& seg, int64_t N, int64_t nw,
                       unsigned long long* d_slots, double* compile_ms) {
  Device& dev = impl_->dev;
  const ExecOptions& opt = impl_->opt;
  Schedule sc = opt.sched;
  if (sc.layout >= 1) {
    // the thread-sequential forms move 32-byte sectors: every input must be
    // 32-byte aligned (the library's own buffers are 256-byte aligned; a
    // borrowed caller buffer may not be), else the segment takes the warp form
    for (int n : seg.inputs)
      if (nodes[n].buf && (reinterpret_cast<uintptr_t>(nodes[n].buf->p) & 31)) sc.layout = 0;
  }
  // the TMA form pays off on long streams only (its boxes cover 32 threads'
  // ranges); short ones take the register form
  if (sc.layout == 2 && nw < (int64_t(1) << 16)) sc.layout = 1;
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); };
  auto tp = clk::now();
  std::string skey = graph_key(nodes, seg.order, seg.inputs, seg.outputs, seg.pops, (N % 64) != 0, sc);
  std::string spec_key;
  if (sc.cut_adds == 0) {
    bool failed_before;
    {
      std::lock_guard<std::mutex> lk(g_spec_mu);
      failed_before = spec_failed().count(skey) != 0;
    }
    if (failed_before) {
      sc.cut_adds = 2;
      skey = graph_key(nodes, seg.order, seg.inputs, seg.outputs, seg.pops, (N % 64) != 0, sc);
    } else {
      spec_key = skey;
    }
  }
  std::shared_ptr<const SegPlan> plan;
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = plan_cache().find(skey);
    if (it != plan_cache().end()) plan = it->second;
  }
  if (!plan) {
    auto np = std::make_shared<SegPlan>();
    for (Part& p : split(nodes, seg, sc.cut_adds, sc.layout >= 1 ? 1 : 32)) {
      if (p.order.empty() && p.pops.empty()) continue;
      if (p.inputs.size() > kMaxInputs) throw RuntimeError("fused: too many inputs in one segment");
      np->kernels.push_back(p.lookback_add ? PartKernel{} : part_kernel(nodes, p, N, sc, compile_ms));
      np->parts.push_back(std::move(p));
    }
    std::lock_guard<std::mutex> lk(g_plan_mu);
    if (plan_cache().size() >= kMaxPlans) plan_cache().clear();
    plan_cache()[skey] = np;
    plan = np;
  }
  // one speculation flag per part, read once by resolve()
  resolve();
  impl_->ensure_flags(static_cast<int64_t>(plan->parts.size()));
  BSZ_CUDA(cudaMemsetAsync(impl_->d_fail, 0, 4 * plan->parts.size(), dev.stream()));
  for (size_t pi = 0; pi < plan->parts.size(); ++pi) {
    const Part& p = plan->parts[pi];
    const PartKernel& pk = plan->kernels[pi];
    const Compiled& c = pk.c;
    // outputs
    for (int n : p.outputs)
      if (!nodes[n].buf) nodes[n].buf = dev.alloc_stream(nw);
    if (p.lookback_add) {
      // carry scheme 2: the plain single-pass carry scan on materialized
      // operands (a constant operand is filled into a temporary first)
      const Node& x = nodes[p.order[0]];
      const uint64_t lm = mask_for_bits(N);
      BufRef tmp[2];
      const uint64_t* opnd[2];
      for (int k = 0; k < 2; ++k) {
        const Node& y = nodes[k == 0 ? x.a : x.b];
        if (y.buf) {
          opnd[k] = y.buf->p;
        } else if (is_const(y.op)) {
          tmp[k] = dev.alloc_stream(nw);
          const uint64_t val = y.op == NOp::Zero ? 0 : ~uint64_t(0);
          launch_fill(dev, tmp[k]->p, nw, val, y.op == NOp::OnesMask ? lm : val);
          opnd[k] = tmp[k]->p;
        } else {
          throw RuntimeError("fused: an addition operand without a buffer");
        }
      }
      launch_add(dev, nodes[p.order[0]].buf->p, opnd[0], opnd[1], nw, lm);
      for (auto& pp : p.pops) launch_popcount(dev, nodes[pp.first].buf->p, nw, d_slots + pp.second);
      continue;
    }
    // argument block, laid out as the generated struct
    const int ni = std::max<int>(1, static_cast<int>(p.inputs.size()));
    const int no = std::max<int>(1, static_cast<int>(p.outputs.size()));
    std::vector<uint64_t> args(ni + no + 6, 0);
    args[ni + no + 5] = 1;   // `one`: a 1 the compiler cannot see (see GenSeq::shift_mul)
    for (size_t i = 0; i < p.inputs.size(); ++i) {
      const Node& x = nodes[p.inputs[i]];
      args[i] = x.buf ? reinterpret_cast<uint64_t>(x.buf->p) : 0;
    }
    for (size_t i = 0; i < p.outputs.size(); ++i) args[ni + i] = reinterpret_cast<uint64_t>(nodes[p.outputs[i]].buf->p);
    int64_t range = 0;
    int blocks = 1;
    const int per_sm = sc.ctas_per_sm > 0 ? std::min(sc.ctas_per_sm, c.blocks_per_sm) : c.blocks_per_sm;
    std::vector<uint8_t> targs;   // the TMA form's argument block
    if (pk.roww > 0) {
      const int R = pk.roww;
      const int per = sc.ctas_per_sm > 0 ? std::min(sc.ctas_per_sm, pk.tma_blocks_per_sm) : pk.tma_blocks_per_sm;
      const int64_t threads_cap = static_cast<int64_t>(dev.sm_count()) * per * sc.warps * 32;
      const int64_t min_range = std::max<int64_t>(64, 16 * pk.warm);
      int64_t threads = std::max<int64_t>(1, std::min(threads_cap, (nw + min_range - 1) / min_range));
      range = ((nw + threads - 1) / threads + R - 1) / R * R;
      range = std::min<int64_t>(std::max<int64_t>(range, R), int64_t(1) << 25);
      const int64_t total = (nw + range - 1) / range;
      blocks = static_cast<int>((total + sc.warps * 32 - 1) / (sc.warps * 32));
      const int64_t nfull = nw / range;
      const int nm = static_cast<int>(pk.mapped.size());
      const int nmp = std::max(1, nm), nop = std::max(1, static_cast<int>(p.outputs.size()));
      const size_t maps_bytes = 128 * static_cast<size_t>(nmp + nop);
      targs.assign(((maps_bytes + 8 * (ni + no + 7)) + 63) / 64 * 64, 0);
      auto encode = [&](void* dst, const uint64_t* base) {
        cuuint64_t dims[3] = {static_cast<cuuint64_t>(R), static_cast<cuuint64_t>(range / R),
                              static_cast<cuuint64_t>(nfull)};
        cuuint64_t strides[2] = {static_cast<cuuint64_t>(R) * 8, static_cast<cuuint64_t>(range) * 8};
        cuuint32_t box[3] = {static_cast<cuuint32_t>(R), 1, 32};
        cuuint32_t es[3] = {1, 1, 1};
        BSZ_CU(drv().tensor_map_encode_tiled(
            reinterpret_cast<CUtensorMap*>(dst), CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<uint64_t*>(base), dims,
            strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            R == 4 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE));
      };
      if (nfull > 0) {
        for (int k = 0; k < nm; ++k) encode(targs.data() + 128 * k, reinterpret_cast<const uint64_t*>(args[pk.mapped[k]]));
        for (size_t o = 0; o < p.outputs.size(); ++o)
          encode(targs.data() + 128 * (nmp + o), reinterpret_cast<const uint64_t*>(args[ni + o]));
      }
      uint64_t* tail = reinterpret_cast<uint64_t*>(targs.data() + maps_bytes);
      for (int i = 0; i < ni + no; ++i) tail[i] = args[i];
      tail[ni + no + 0] = reinterpret_cast<uint64_t>(d_slots);
      tail[ni + no + 1] = reinterpret_cast<uint64_t>(impl_->d_fail + pi);
      tail[ni + no + 2] = static_cast<uint64_t>(nw);
      tail[ni + no + 3] = static_cast<uint64_t>(range);
      tail[ni + no + 4] = mask_for_bits(N);
      tail[ni + no + 5] = static_cast<uint64_t>(nfull);
      tail[ni + no + 6] = 1;
    } else if (sc.layout >= 1) {
      // thread-sequential: one range of whole 4-word chunks per thread, at
      // least 16 warm-ups long; a persistent grid of what stays resident
      const int64_t threads_cap = sc.ctas_per_sm < 0 ? std::numeric_limits<int64_t>::max() / 2
                                                     : static_cast<int64_t>(dev.sm_count()) * per_sm * sc.warps * 32;
      const int64_t min_range = std::max<int64_t>(64, 16 * pk.warm);
      int64_t threads = std::max<int64_t>(1, std::min(threads_cap, (nw + min_range - 1) / min_range));
      const int64_t cw = sc.chunk_words == 8 ? 8 : 4;
      range = ((nw + threads - 1) / threads + cw - 1) / cw * cw;
      range = std::min<int64_t>(std::max<int64_t>(range, cw), int64_t(1) << 25);   // per-thread popcounts fit u32
      const int64_t total = (nw + range - 1) / range;
      blocks = static_cast<int>((total + sc.warps * 32 - 1) / (sc.warps * 32));
    } else {
      // grid: contiguous ranges of whole 32-word steps, at least 8 warm-ups long
      const int64_t steps = (nw + 31) / 32;
      // persistent grid: as many warps as the compiled kernel keeps resident;
      // ctas_per_sm < 0: no persistent cap, every warp takes one range of the
      // minimum length (more warps, shorter ranges, more warm-up work)
      const int64_t max_warps = sc.ctas_per_sm < 0 ? std::numeric_limits<int64_t>::max() / 2
                                                   : static_cast<int64_t>(dev.sm_count()) * per_sm * sc.warps;
      int64_t min_range_steps = std::max<int64_t>(sc.range_steps, (pk.warm / 32) * 8);
      int64_t warps_needed = std::max<int64_t>(1, std::min(max_warps, (steps + min_range_steps - 1) / min_range_steps));
      range = ((steps + warps_needed - 1) / warps_needed) * 32;
      int64_t total_warps = (nw + range - 1) / range;
      blocks = static_cast<int>((total_warps + sc.warps - 1) / sc.warps);
    }
    args[ni + no + 0] = reinterpret_cast<uint64_t>(d_slots);
    args[ni + no + 1] = reinterpret_cast<uint64_t>(impl_->d_fail + pi);
    args[ni + no + 2] = static_cast<uint64_t>(nw);
    args[ni + no + 3] = static_cast<uint64_t>(range);
    args[ni + no + 4] = mask_for_bits(N);
    void* kparams[] = {pk.roww > 0 ? static_cast<void*>(targs.data()) : static_cast<void*>(args.data())};
    {
      ProfScope prof(dev, "fused");
      BSZ_CU(drv().launch_kernel(c.fn, blocks, 1, 1, sc.warps * 32, 1, 1, pk.roww > 0 ? pk.smem : 0,
                            reinterpret_cast<CUstream>(dev.stream()), kparams, nullptr));
    }
    ++dev.n_launches;
    ++launches;
    t_prelaunch_ms += ms_since(tp);
    tp = clk::now();
  }
  // the segment stays pending until resolve(): keep its parts and a copy of
  // every node they compute or read, buffers included
  auto pend = std::make_unique<PendingSegment>();
  pend->plan = plan;
  pend->parts = &plan->parts;
  pend->N = N;
  pend->nw = nw;
  pend->d_slots = d_slots;
  pend->spec_key = std::move(spec_key);
  for (const Part& p : plan->parts) {
    for (int n : p.order) pend->nodes.emplace(n, nodes[n]);
    for (int n : p.inputs) pend->nodes.emplace(n, nodes[n]);
    for (auto& pp : p.pops) pend->nodes.emplace(pp.first, nodes[pp.first]);
  }
  impl_->pending = std::move(pend);
}

bool FusedBackend::pending() const { return impl_->pending != nullptr; }

namespace {

// Re-runs one part with the exact per-op kernels (its popcount slots are
// cleared first), reading and writing the buffers recorded with it.
void rerun_part_exact(Device& dev, const Part& p, std::unordered_map<int, Node>& nodes, int64_t N, int64_t nw,
                      unsigned long long* d_slots) {
  for (auto& pp : p.pops) BSZ_CUDA(cudaMemsetAsync(d_slots + pp.second, 0, 8, dev.stream()));
  const uint64_t lm = mask_for_bits(N);
  std::map<int, BufRef> tmp;
  auto node = [&](int n) -> Node& {
    auto it = nodes.find(n);
    if (it == nodes.end()) throw RuntimeError("fused re-run: a node was not recorded");
    return it->second;
  };
  auto opnd = [&](int o) -> const uint64_t* {
    const Node& y = node(o);
    if (y.buf) return y.buf->p;
    auto it = tmp.find(o);
    if (it != tmp.end()) return it->second->p;
    if (is_const(y.op)) {
      BufRef b = dev.alloc_stream(nw);
      const uint64_t val = y.op == NOp::Zero ? 0 : ~uint64_t(0);
      launch_fill(dev, b->p, nw, val, y.op == NOp::OnesMask ? lm : val);
      return tmp.emplace(o, b).first->second->p;
    }
    throw RuntimeError("fused re-run: operand without a buffer");
  };
  for (int n : p.order) {
    const Node& x = node(n);
    BufRef out = x.buf ? x.buf : dev.alloc_stream(nw);
    uint64_t* D = out->p;
    switch (x.op) {
      case NOp::Not: launch_not(dev, D, opnd(x.a), nw, lm); break;
      case NOp::And: launch_bitwise(dev, kAnd, D, opnd(x.a), opnd(x.b), nw); break;
      case NOp::Or: launch_bitwise(dev, kOr, D, opnd(x.a), opnd(x.b), nw); break;
      case NOp::Xor: launch_bitwise(dev, kXor, D, opnd(x.a), opnd(x.b), nw); break;
      case NOp::AndNot: launch_bitwise(dev, kAndNot, D, opnd(x.a), opnd(x.b), nw); break;
      case NOp::Add: launch_add(dev, D, opnd(x.a), opnd(x.b), nw, lm); break;
      case NOp::Shl: launch_shl(dev, D, opnd(x.a), x.k, nw, lm); break;
      case NOp::Shr: launch_shr(dev, D, opnd(x.a), x.k, nw, node(x.a).tail ? ~uint64_t(0) : 0); break;
      default: throw RuntimeError("fused re-run: unexpected node");
    }
    if (!x.buf) tmp[n] = out;
  }
  for (auto& pp : p.pops) launch_popcount(dev, opnd(pp.first), nw, d_slots + pp.second);
}

}  // namespace

void FusedBackend::resolve() {
  if (!impl_->pending) return;
  Device& dev = impl_->dev;
  using clk = std::chrono::steady_clock;
  auto tw = clk::now();
  std::vector<uint32_t> flags(impl_->pending->parts->size(), 0);
  BSZ_CUDA(cudaMemcpyAsync(flags.data(), impl_->d_fail, 4 * flags.size(), cudaMemcpyDeviceToHost, dev.stream()));
  BSZ_CUDA(cudaStreamSynchronize(dev.stream()));
  t_wait_ms += std::chrono::duration<double, std::milli>(clk::now() - tw).count();
  resolve_with(flags.data());
}

int64_t FusedBackend::pending_parts() const {
  return impl_->pending ? static_cast<int64_t>(impl_->pending->parts->size()) : 0;
}

void FusedBackend::enqueue_flags(uint32_t* host) {
  if (!impl_->pending) return;
  BSZ_CUDA(cudaMemcpyAsync(host, impl_->d_fail, 4 * impl_->pending->parts->size(), cudaMemcpyDeviceToHost,
                           impl_->dev.stream()));
}

bool FusedBackend::resolve_with(const uint32_t* flags) {
  if (!impl_->pending) return false;
  std::unique_ptr<PendingSegment> pend = std::move(impl_->pending);
  const std::vector<Part>& parts = *pend->parts;
  size_t first = parts.size();
  for (size_t i = 0; i < parts.size(); ++i)
    if (flags[i]) {
      first = i;
      break;
    }
  // Speculation could not be proven exact in part `first`: redo it, and
  // every later part (which may have read its outputs), with the plain
  // per-op kernels (exact by construction).
  for (size_t i = first; i < parts.size(); ++i) {
    rerun_part_exact(impl_->dev, parts[i], pend->nodes, pend->N, pend->nw, pend->d_slots);
    if (flags[i]) ++fallbacks;
  }
  if (first < parts.size() && !pend->spec_key.empty()) {
    std::lock_guard<std::mutex> lk(g_spec_mu);
    if (spec_failed().size() >= kMaxPlans) spec_failed().clear();
    spec_failed().insert(pend->spec_key);
  }
  return first < parts.size();
}

// ================================================================ batches ==

namespace {

struct BatchProg {
  Executor::Traced t;
  Part part;
  std::map<int, int> in_index;
  std::vector<std::pair<int, int>> outs;
  std::string fn;
  int64_t warm = 64;
};

struct BatchItem {   // layout shared with the generated kernel's Item
  int32_t inst;
  int32_t dag;
  int64_t s;
  int64_t e;
};

int64_t eval_postfix(const std::vector<std::pair<char, int64_t>>& prog, const uint64_t* slots) {
  std::vector<int64_t> st;
  for (const auto& op : prog) {
    if (op.first == 'k') {
      st.push_back(op.second);
    } else if (op.first == 's') {
      st.push_back(static_cast<int64_t>(slots[op.second]));
    } else {
      int64_t b = st.back();
      st.pop_back();
      int64_t a = st.back();
      st.pop_back();
      st.push_back(op.first == '+' ? a + b : op.first == '-' ? a - b : a * b);
    }
  }
  return st.empty() ? 0 : st.back();
}

// Builds the single part of a traced straight-line program.
void plan_batch_program(BatchProg& bp) {
  const Executor::Traced& t = bp.t;
  const auto& nodes = t.nodes;
  std::vector<uint8_t> need(nodes.size(), 0);
  std::vector<int> stack;
  for (int n : t.output_nodes)
    if (n >= 0) stack.push_back(n);
  for (auto& p : t.pops) stack.push_back(p.first);
  auto computed = [&](int n) {
    NOp op = nodes[n].op;
    return op != NOp::Buf && op != NOp::Zero && op != NOp::OnesMask && op != NOp::AllOnes;
  };
  while (!stack.empty()) {
    int n = stack.back();
    stack.pop_back();
    if (need[n]) continue;
    need[n] = 1;
    if (!computed(n)) continue;
    for (int o : {nodes[n].a, nodes[n].b})
      if (o >= 0) stack.push_back(o);
  }
  for (size_t n = 0; n < nodes.size(); ++n) {
    if (!need[n]) continue;
    if (computed(static_cast<int>(n))) {
      const Node& x = nodes[n];
      if (x.op == NOp::Shr && computed(x.a))
        throw RuntimeError("batch: a right shift of a temporary is not supported in batches");
      if (x.op == NOp::Shl && computed(x.a) && x.k / 64 >= 32)
        throw RuntimeError("batch: a left shift of a temporary by 2048 bits or more is not supported");
      bp.part.order.push_back(static_cast<int>(n));
    } else {
      bp.part.inputs.push_back(static_cast<int>(n));
    }
  }
  for (size_t i = 0; i < t.input_nodes.size(); ++i) bp.in_index[t.input_nodes[i]] = static_cast<int>(i);
  for (size_t j = 0; j < t.output_nodes.size(); ++j)
    if (t.output_nodes[j] >= 0) bp.outs.push_back({t.output_nodes[j], static_cast<int>(j)});
  bp.part.pops = t.pops;
}

}  // namespace

struct BatchRunner::Impl {
  Device& dev;
  Schedule sched;
  std::vector<BatchProg> progs;
  std::vector<const Program*> srcs;
  std::vector<BatchInstance> inst;
  std::vector<int64_t> slot_base;
  int64_t n_slots = 0;
  int64_t n_items = 0;
  int max_in = 1, max_out = 1;
  Compiled kern;
  void* d_args = nullptr;
  void* d_items = nullptr;
  unsigned long long* d_slots = nullptr;
  unsigned int* d_ctrl = nullptr;   // [0] work counter, [1] speculation-failed flag
  int blocks = 1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> h_slots;
  std::vector<std::vector<int64_t>> ints;
  explicit Impl(Device& d) : dev(d) {}
  ~Impl() {
    cudaStreamSynchronize(dev.stream());
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : {d_args, d_items, static_cast<void*>(d_slots), static_cast<void*>(d_ctrl)})
      if (p) cudaFree(p);
  }
  void* upload(const void* host, size_t bytes) {
    void* p = nullptr;
    BSZ_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 256)));
    ++dev.n_mallocs;
    if (bytes) BSZ_CUDA(cudaMemcpyAsync(p, host, bytes, cudaMemcpyHostToDevice, dev.stream()));
    return p;
  }
};

BatchRunner::BatchRunner(Device& dev, const std::vector<const Program*>& progs,
                         std::vector<BatchInstance> instances, const Schedule& sched)
    : impl_(std::make_unique<Impl>(dev)) {
  Impl& m = *impl_;
  m.sched = sched;
  m.srcs = progs;
  m.inst = std::move(instances);
  // the thread-sequential form (register chunks; batches have no TMA form)
  // needs every instance buffer 32-byte aligned
  bool seq = sched.layout >= 1;
  for (const BatchInstance& bi : m.inst) {
    for (const uint64_t* q : bi.inputs)
      if (reinterpret_cast<uintptr_t>(q) & 31) seq = false;
    for (const uint64_t* q : bi.outputs)
      if (reinterpret_cast<uintptr_t>(q) & 31) seq = false;
  }
  // 1. trace every program symbolically and plan its DAG
  ExecOptions eo;
  eo.mode = ExecMode::Fused;
  eo.sched = sched;
  std::string fns;
  std::vector<BatchProg> traced(progs.size());
  for (size_t k = 0; k < progs.size(); ++k) {
    {
      Executor ex(dev, *progs[k], int64_t(1) << 20, eo);
      traced[k].t = ex.trace();
    }
    plan_batch_program(traced[k]);
    // a temporary shifted left by 64 bits or more needs words a lane no
    // longer holds: such programs keep the warp form
    for (int n : traced[k].part.order) {
      const Node& x = traced[k].t.nodes[n];
      const NOp ao = x.a >= 0 ? traced[k].t.nodes[x.a].op : NOp::Buf;
      const bool temp = ao != NOp::Buf && ao != NOp::Zero && ao != NOp::OnesMask && ao != NOp::AllOnes;
      if (x.op == NOp::Shl && temp && x.k >= 64) seq = false;
    }
  }
  for (size_t k = 0; k < progs.size(); ++k) {
    BatchProg bp = std::move(traced[k]);
    if (seq) {
      GenSeq g{bp.t.nodes, bp.part, 0, sched.warps, sched.min_blocks, true};
      g.shift_mul = sched.shift_mul != 0;
      g.reg_chunk = sched.chunk_words == 8 ? 8 : 4;
      g.guard_outputs = true;
      g.in_index_override = &bp.in_index;
      g.outs_override = &bp.outs;
      bp.fn = g.device_function("dag_" + std::to_string(k));
      bp.warm = g.warm;
    } else {
      Gen g{bp.t.nodes, bp.part, 0, sched.warps, sched.min_blocks, true, sched.prefetch != 0};
      g.guard_outputs = true;
      g.in_index_override = &bp.in_index;
      g.outs_override = &bp.outs;
      bp.fn = g.device_function("dag_" + std::to_string(k));
      bp.warm = g.warm;
    }
    m.max_in = std::max<int>(m.max_in, static_cast<int>(bp.t.input_nodes.size()));
    m.max_out = std::max<int>(m.max_out, static_cast<int>(bp.t.output_nodes.size()));
    fns += bp.fn;
    m.progs.push_back(std::move(bp));
  }
  // 2. one kernel: every program's DAG as a device function + a work loop
  std::ostringstream src;
  src << Gen::args_struct(m.max_in, m.max_out) << (seq ? GenSeq::helpers() : std::string()) << fns
      << "struct Item { int inst; int dag; long long s; long long e; };\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << sched.warps * 32 << ", "
      << sched.min_blocks << ")\nbsz_batch(const Args* __restrict__ insts, "
      << "const Item* __restrict__ items, const long long n_items, unsigned int* __restrict__ ctrl) {\n"
      << "  const int lane = threadIdx.x & 31;\n"
      << "  for (;;) {\n"
      << "    unsigned int it = 0;\n"
      << "    if (lane == 0) it = atomicAdd(ctrl, 1u);\n"
      << "    it = __shfl_sync(~0u, it, 0);\n"
      << "    if (it >= n_items) return;\n"
      << "    const Item I = items[it];\n"
      << "    switch (I.dag) {\n";
  for (size_t k = 0; k < m.progs.size(); ++k)
    src << "      case " << k << ": dag_" << k << "(insts + I.inst, I.s, I.e, lane); break;\n";
  src << "      default: break;\n    }\n  }\n}\n";
  m.kern = compile_source(src.str(), sched.warps * 32, &compile_ms, "bsz_batch");
  // 3. argument blocks (one Args per instance), slots and work items
  const size_t stride = static_cast<size_t>(m.max_in + m.max_out + 6);
  std::vector<uint64_t> args(stride * m.inst.size(), 0);
  BSZ_CUDA(cudaMalloc(&m.d_ctrl, 256));
  ++dev.n_mallocs;
  std::vector<BatchItem> items;
  for (size_t i = 0; i < m.inst.size(); ++i) {
    const BatchInstance& bi = m.inst[i];
    if (bi.program < 0 || bi.program >= static_cast<int>(m.progs.size()))
      throw std::invalid_argument("batch: instance program index out of range");
    const BatchProg& bp = m.progs[bi.program];
    if (bi.inputs.size() != bp.t.input_nodes.size() || bi.outputs.size() != bp.t.output_nodes.size())
      throw std::invalid_argument("batch: instance " + std::to_string(i) +
                                  " does not give one pointer per declared input/output stream");
    m.slot_base.push_back(m.n_slots);
    m.n_slots += static_cast<int64_t>(bp.t.pops.size());
    const int64_t nw = std::max<int64_t>(1, (bi.bitlength + 63) / 64);
    // work items: warp form, runs of 32-word steps; thread-sequential form,
    // 32 lane ranges of whole register chunks, each at least 16 warm-ups long
    const int64_t cw = sched.chunk_words == 8 ? 8 : 4;
    const int64_t range = seq ? 32 * cw * ((std::max<int64_t>(64, 16 * bp.warm) + cw - 1) / cw)
                              : 32 * std::max<int64_t>(sched.range_steps, (bp.warm / 32) * 8);
    for (int64_t s0 = 0; s0 < nw; s0 += range)
      items.push_back({static_cast<int32_t>(i), bi.program, s0, std::min(nw, s0 + range)});
    uint64_t* a = args.data() + stride * i;
    for (size_t j = 0; j < bi.inputs.size(); ++j) a[j] = reinterpret_cast<uint64_t>(bi.inputs[j]);
    for (size_t j = 0; j < bi.outputs.size(); ++j) a[m.max_in + j] = reinterpret_cast<uint64_t>(bi.outputs[j]);
    a[m.max_in + m.max_out + 1] = reinterpret_cast<uint64_t>(m.d_ctrl + 1);
    a[m.max_in + m.max_out + 2] = static_cast<uint64_t>(nw);
    a[m.max_in + m.max_out + 3] = static_cast<uint64_t>(range);
    a[m.max_in + m.max_out + 4] = mask_for_bits(bi.bitlength > 0 ? bi.bitlength : 64 * nw);
    a[m.max_in + m.max_out + 5] = 1;
  }
  // items of one program together (warps then run the same device function,
  // so the instruction cache holds one DAG at a time), longest first within
  // it so the atomic work queue balances the tail
  std::stable_sort(items.begin(), items.end(), [](const BatchItem& x, const BatchItem& y) {
    if (x.dag != y.dag) return x.dag < y.dag;
    return (x.e - x.s) > (y.e - y.s);
  });
  m.n_items = static_cast<int64_t>(items.size());
  BSZ_CUDA(cudaMalloc(&m.d_slots, static_cast<size_t>(std::max<int64_t>(m.n_slots, 1)) * 8));
  ++dev.n_mallocs;
  for (size_t i = 0; i < m.inst.size(); ++i)
    args[stride * i + m.max_in + m.max_out] = reinterpret_cast<uint64_t>(m.d_slots + m.slot_base[i]);
  m.d_args = m.upload(args.data(), args.size() * 8);
  m.d_items = m.upload(items.data(), items.size() * sizeof(BatchItem));
  const int64_t per_sm = sched.ctas_per_sm > 0 ? std::min(sched.ctas_per_sm, m.kern.blocks_per_sm)
                                               : m.kern.blocks_per_sm;
  const int64_t want = (m.n_items + sched.warps - 1) / sched.warps;
  m.blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, dev.sm_count() * per_sm)));
  // 4. capture: reset the counters and slots, launch; replayed by launch()
  BSZ_CUDA(cudaStreamSynchronize(dev.stream()));
  BSZ_CUDA(cudaStreamBeginCapture(dev.stream(), cudaStreamCaptureModeThreadLocal));
  BSZ_CUDA(cudaMemsetAsync(m.d_ctrl, 0, 8, dev.stream()));
  BSZ_CUDA(cudaMemsetAsync(m.d_slots, 0, static_cast<size_t>(std::max<int64_t>(m.n_slots, 1)) * 8,
                           dev.stream()));
  long long n_items_arg = m.n_items;
  void* kp[] = {&m.d_args, &m.d_items, &n_items_arg, &m.d_ctrl};
  BSZ_CU(drv().launch_kernel(m.kern.fn, m.blocks, 1, 1, sched.warps * 32, 1, 1, 0,
                             reinterpret_cast<CUstream>(dev.stream()), kp, nullptr));
  BSZ_CUDA(cudaStreamEndCapture(dev.stream(), &m.graph));
  BSZ_CUDA(cudaGraphInstantiate(&m.exec, m.graph, 0));
  m.ints.assign(m.inst.size(), {});
}

BatchRunner::~BatchRunner() = default;

int64_t BatchRunner::n_items() const { return impl_->n_items; }

void BatchRunner::launch() {
  Impl& m = *impl_;
  ProfScope prof(m.dev, "bsz_batch");
  BSZ_CUDA(cudaGraphLaunch(m.exec, m.dev.stream()));
  ++m.dev.n_launches;
  ++launches;
}

void BatchRunner::finish() {
  Impl& m = *impl_;
  unsigned int fail = 0;
  m.h_slots.assign(static_cast<size_t>(std::max<int64_t>(m.n_slots, 1)), 0);
  BSZ_CUDA(cudaMemcpyAsync(&fail, m.d_ctrl + 1, 4, cudaMemcpyDeviceToHost, m.dev.stream()));
  BSZ_CUDA(cudaMemcpyAsync(m.h_slots.data(), m.d_slots, m.h_slots.size() * 8, cudaMemcpyDeviceToHost,
                           m.dev.stream()));
  BSZ_CUDA(cudaStreamSynchronize(m.dev.stream()));
  if (fail) {
    // Speculation unproven somewhere: recompute every instance with the
    // exact per-op kernels (rare; correctness first).
    ++fallbacks;
    for (size_t i = 0; i < m.inst.size(); ++i) {
      const BatchInstance& bi = m.inst[i];
      const Program& prog = *m.srcs[bi.program];
      const int64_t nw = std::max<int64_t>(1, (bi.bitlength + 63) / 64);
      ExecOptions eo;
      eo.mode = ExecMode::Plain;
      Executor ex(m.dev, prog, bi.bitlength, eo);
      size_t j = 0;
      for (int id : prog.inputs) {
        auto b = std::make_shared<DevStream>();
        b->p = const_cast<uint64_t*>(bi.inputs[j++]);
        b->n_words = nw;
        ex.bind_input(id, b, 0, false);
      }
      ex.run();
      j = 0;
      for (int id : prog.outputs) {
        uint64_t* dst = bi.outputs[j++];
        if (dst && ex.has_stream(id))
          BSZ_CUDA(cudaMemcpyAsync(dst, ex.stream_value(id)->p, nw * 8, cudaMemcpyDeviceToDevice,
                                   m.dev.stream()));
      }
      std::vector<int64_t> v;
      for (int id : prog.output_ints) {
        int64_t x = 0;
        ex.int_value(id, &x);
        v.push_back(x);
      }
      m.ints[i] = std::move(v);
    }
    BSZ_CUDA(cudaStreamSynchronize(m.dev.stream()));
    return;
  }
  for (size_t i = 0; i < m.inst.size(); ++i) {
    const BatchProg& bp = m.progs[m.inst[i].program];
    std::vector<int64_t> v;
    for (const auto& post : bp.t.int_outputs) v.push_back(eval_postfix(post, m.h_slots.data() + m.slot_base[i]));
    m.ints[i] = std::move(v);
  }
}

const std::vector<int64_t>& BatchRunner::ints(int64_t i) const { return impl_->ints.at(i); }

int64_t BatchRunner::op_count(int64_t i) const {
  return impl_->progs.at(impl_->inst.at(i).program).t.op_count;
}

}  // namespace bsz
