// Executor implementation (see engine.h).
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <functional>

#include "fused.h"
#include "vm.h"

namespace bsz {
namespace {

constexpr int kMaxWhileIters = 10000;          // simulator/pythonsim/interpreter.py:20
constexpr int64_t kSlotChunk = 1 << 16;
// A straight-line run longer than this (unrolled loop nests reach tens of
// millions of operations) is flushed at the next statement boundary, which
// bounds host memory and lets the device work while the walk continues.
constexpr size_t kAutoFlushNodes = size_t(1) << 20;
// Segments with more operations than this never become one generated
// kernel: NVRTC time and register pressure grow with the segment.
constexpr size_t kMaxFusedOps = 3000;

using Bits = std::vector<uint64_t>;
inline bool bit(const Bits& b, int i) { return (b[i >> 6] >> (i & 63)) & 1u; }
inline void set_bit(Bits& b, int i) { b[i >> 6] |= uint64_t(1) << (i & 63); }
inline void clr_bit(Bits& b, int i) { b[i >> 6] &= ~(uint64_t(1) << (i & 63)); }
inline void or_into(Bits& d, const Bits& s) {
  for (size_t i = 0; i < d.size(); ++i) d[i] |= s[i];
}

bool commutative(NOp op) {
  return op == NOp::And || op == NOp::Or || op == NOp::Xor || op == NOp::Add;
}

template <class T>
void put_raw(std::string& s, T v) {
  s.append(reinterpret_cast<const char*>(&v), sizeof v);
}

// At most this many cached walks per program (oldest evicted first).
constexpr size_t kMaxWalks = 16;

}  // namespace

// A straight-line walk: everything run() reads after exec_block() and before
// the final flush.  Nodes below n0 (the constants and the bound inputs, the
// same ids for the same bindings) are not stored; the stored ones have no
// buffers.
struct Executor::WalkSnap {
  size_t n0 = 0;
  std::vector<Node> nodes;
  std::vector<int> var;
  std::vector<IntV> ints;
  std::vector<uint8_t> int_def;
  std::vector<std::unique_ptr<Arr>> arrs;
  std::vector<IE> iexpr;
  std::vector<std::pair<int, int64_t>> pops;
  int64_t n_slots = 0;
  int64_t op_count = 0;
  int64_t op_class[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

struct Executor::ExecCache {
  std::shared_ptr<const Liveness> live;
  std::unordered_map<std::string, std::shared_ptr<const WalkSnap>> walks;
  std::vector<std::string> order;   // insertion order, for eviction
};

Executor::ExecCache& Executor::exec_cache() const {
  std::lock_guard<std::mutex> lk(prog_.exec_mu);
  if (!prog_.exec_cache) prog_.exec_cache = std::make_shared<ExecCache>();
  return *static_cast<ExecCache*>(prog_.exec_cache.get());
}

std::string Executor::walk_key() const {
  std::string k = bind_sig_;
  put_raw(k, N_);
  put_raw(k, static_cast<int>(opt_.mode));
  put_raw(k, opt_.simplify);
  return k;
}

bool Executor::replay_walk(const std::string& key) {
  std::shared_ptr<const WalkSnap> s;
  {
    ExecCache& c = exec_cache();
    std::lock_guard<std::mutex> lk(prog_.exec_mu);
    auto it = c.walks.find(key);
    if (it == c.walks.end()) return false;
    s = it->second;
  }
  if (nodes_.size() != s->n0 || n_slots_ != 0 || !pending_pops_.empty()) return false;
  nodes_.insert(nodes_.end(), s->nodes.begin(), s->nodes.end());
  var_ = s->var;
  ints_ = s->ints;
  int_def_ = s->int_def;
  for (size_t i = 0; i < arrs_.size(); ++i)
    arrs_[i] = s->arrs[i] ? std::make_unique<Arr>(*s->arrs[i]) : nullptr;
  iexpr_ = s->iexpr;
  if (s->n_slots > 0) ensure_slots(s->n_slots);
  n_slots_ = s->n_slots;
  pending_pops_ = s->pops;
  op_count = s->op_count;
  for (int k = 0; k < 8; ++k) op_class_[k] = s->op_class[k];
  return true;
}

// The stored walk keeps only the nodes the final flush can reach (from the
// stream names live at the end, every array element and every pending
// popcount), renumbered in order; names whose computed value is dead there
// read -2, as the flush would leave them.  A replay then copies and scans
// the live DAG only.
void Executor::save_walk(const std::string& key, size_t n0) {
  const size_t n = nodes_.size();
  for (size_t i = n0; i < n; ++i)
    if (nodes_[i].buf) return;   // not a pure walk
  std::vector<uint8_t> need(n, 0);
  std::vector<int> stack;
  auto target = [&](int x) {
    if (x >= 0) stack.push_back(x);
  };
  for (size_t v = 0; v < var_.size(); ++v)
    if (bit(live_->end, static_cast<int>(v))) target(var_[v]);
  for (auto& a : arrs_)
    if (a) for (auto& kv : a->elems) target(kv.second);
  for (auto& p : pending_pops_) target(p.first);
  while (!stack.empty()) {
    int x = stack.back();
    stack.pop_back();
    if (need[x]) continue;
    need[x] = 1;
    if (nodes_[x].a >= 0) stack.push_back(nodes_[x].a);
    if (nodes_[x].b >= 0) stack.push_back(nodes_[x].b);
  }
  std::vector<int> remap(n, -2);
  for (size_t i = 0; i < n0; ++i) remap[i] = static_cast<int>(i);
  auto s = std::make_shared<WalkSnap>();
  s->n0 = n0;
  for (size_t i = n0; i < n; ++i) {
    if (!need[i]) continue;
    remap[i] = static_cast<int>(n0 + s->nodes.size());
    Node x = nodes_[i];
    if (x.a >= 0) x.a = remap[x.a];
    if (x.b >= 0) x.b = remap[x.b];
    s->nodes.push_back(std::move(x));
  }
  auto map = [&](int x) { return x < 0 ? x : remap[x]; };
  s->var.resize(var_.size());
  for (size_t v = 0; v < var_.size(); ++v) s->var[v] = map(var_[v]);
  s->ints = ints_;
  s->int_def = int_def_;
  s->arrs.resize(arrs_.size());
  for (size_t i = 0; i < arrs_.size(); ++i)
    if (arrs_[i]) {
      s->arrs[i] = std::make_unique<Arr>(*arrs_[i]);
      for (auto& kv : s->arrs[i]->elems) kv.second = map(kv.second);
    }
  s->iexpr = iexpr_;
  s->pops = pending_pops_;
  for (auto& p : s->pops) p.first = map(p.first);
  s->n_slots = n_slots_;
  s->op_count = op_count;
  for (int k = 0; k < 8; ++k) s->op_class[k] = op_class_[k];
  ExecCache& c = exec_cache();
  std::lock_guard<std::mutex> lk(prog_.exec_mu);
  if (c.walks.count(key)) return;
  if (c.walks.size() >= kMaxWalks) {
    c.walks.erase(c.order.front());
    c.order.erase(c.order.begin());
  }
  c.walks.emplace(key, std::move(s));
  c.order.push_back(key);
}

Executor::Executor(Device& dev, const Program& prog, int64_t bitlength, ExecOptions opt)
    : dev_(dev), prog_(prog), opt_(opt) {
  N_ = bitlength;
  nw_ = std::max<int64_t>(1, (bitlength + 63) / 64);
  if (bitlength <= 0) N_ = 64 * nw_;   // no bitlength: bounded by the storage width
  last_mask_ = mask_for_bits(N_);
  const size_t nn = prog.names.size();
  var_.assign(nn, -1);
  ints_.assign(nn, IntV{});
  int_def_.assign(nn, 0);
  arrs_.resize(nn);
  zero_ = mk_raw(NOp::Zero, -1, -1, 0, 0);
  ones_mask_ = mk_raw(NOp::OnesMask, -1, -1, 0, 0);
  all_ones_ = mk_raw(NOp::AllOnes, -1, -1, 0, 1);
  // Inputs that are not bound read as ZERO (interpreter.py:232-238).
  for (int id : prog.inputs) var_[id] = zero_;
  if (opt_.mode != ExecMode::Plain) opt_.simplify = true;
  if (opt_.mode == ExecMode::Fused || opt_.mode == ExecMode::Auto)
    fused_ = std::make_unique<FusedBackend>(dev_, opt_);
  flag_buf_ = dev_.alloc_stream(32);
  d_flag_ = reinterpret_cast<unsigned int*>(flag_buf_->p);
  ExecCache& c = exec_cache();
  std::lock_guard<std::mutex> lk(prog_.exec_mu);
  if (!c.live) c.live = compute_liveness();
  live_ = c.live;
}

Executor::~Executor() {
  if (std::getenv("BSZ_HOST_TIMES"))
    std::fprintf(stderr,
                 "[bsz] segments=%lld vm=%lld fused=%lld ops=%lld replayed=%d host ms: segment %.3f policy %.3f "
                 "run %.3f (fused prelaunch %.3f wait %.3f) compact %.3f compile %.2f\n",
                 static_cast<long long>(n_segments), static_cast<long long>(vm_launches),
                 static_cast<long long>(fused_launches()), static_cast<long long>(op_count),
                 walk_replayed ? 1 : 0, t_segment_ms, t_policy_ms, t_run_ms,
                 fused_ ? fused_->t_prelaunch_ms : 0.0, fused_ ? fused_->t_wait_ms : 0.0, t_compact_ms,
                 compile_ms);
  // A finished run's device work is complete.  Otherwise wait for it before
  // its buffers go back to the device's cache (reuse is stream-ordered, but a
  // caller may free a borrowed input as soon as the run is gone).  Waiting
  // after finish() would also wait for whatever another run enqueued since.
  if (!finished_) cudaStreamSynchronize(dev_.stream());
  if (done_ev_) cudaEventDestroy(done_ev_);
  // flag, slot and VM buffers go back to the device's cache with their BufRefs
}

void Executor::set_schedule(const Schedule& s) {
  opt_.sched = s;
  if (fused_) fused_->set_schedule(s);
}

int64_t Executor::fused_launches() const { return fused_ ? fused_->launches : 0; }
int64_t Executor::fused_fallbacks() const { return fused_ ? fused_->fallbacks : 0; }

void Executor::set_param(int name, int64_t v) {
  if (name < 0) return;
  put_raw(bind_sig_, 'p');
  put_raw(bind_sig_, name);
  put_raw(bind_sig_, v);
  ints_[name] = IntV{v, -1};
  int_def_[name] = 1;
}

void Executor::bind_input(int name, BufRef buf, uint8_t tail, bool clean) {
  put_raw(bind_sig_, 's');
  put_raw(bind_sig_, name);
  put_raw(bind_sig_, static_cast<uint8_t>(tail | (clean ? 2 : 0)));
  var_[name] = buf_node(std::move(buf), tail, clean);
}

void Executor::bind_input_array(int name, int64_t idx, BufRef buf, uint8_t tail, bool clean) {
  put_raw(bind_sig_, 'a');
  put_raw(bind_sig_, name);
  put_raw(bind_sig_, idx);
  put_raw(bind_sig_, static_cast<uint8_t>(tail | (clean ? 2 : 0)));
  if (!arrs_[name]) arrs_[name] = std::make_unique<Arr>();
  Arr& a = *arrs_[name];
  a.defined = true;
  a.elems[idx] = buf_node(std::move(buf), tail, clean);
  if (var_[name] == zero_) var_[name] = -1;   // it is an array, not a scalar input
}

void Executor::bind_broadcast(int name, const std::vector<uint8_t>& ones) {
  put_raw(bind_sig_, 'b');
  put_raw(bind_sig_, name);
  put_raw(bind_sig_, static_cast<int64_t>(ones.size()));
  bind_sig_.append(reinterpret_cast<const char*>(ones.data()), ones.size());
  if (!arrs_[name]) arrs_[name] = std::make_unique<Arr>();
  Arr& a = *arrs_[name];
  a.defined = true;
  a.broadcast = true;
  a.bcast = ones;
  if (var_[name] == zero_) var_[name] = -1;
}

// ------------------------------------------------------------------ graph --

int Executor::mk_raw(NOp op, int a, int b, int64_t k, uint8_t tail) {
  Node n;
  n.op = op;
  n.a = a;
  n.b = b;
  n.k = k;
  n.tail = tail;
  auto cl = [&](int x) { return x >= 0 && nodes_[x].clean; };
  switch (op) {
    case NOp::Zero: case NOp::OnesMask: case NOp::Not: case NOp::Add: case NOp::Shl:
    case NOp::AndNot:
      n.clean = 1; break;
    case NOp::And: n.clean = cl(a) || cl(b); break;
    case NOp::Or: case NOp::Xor: n.clean = cl(a) && cl(b); break;
    case NOp::Shr: n.clean = cl(a); break;
    default: n.clean = 0; break;
  }
  nodes_.push_back(std::move(n));
  return static_cast<int>(nodes_.size()) - 1;
}

int Executor::buf_node(BufRef buf, uint8_t tail, bool clean) {
  int id = mk_raw(NOp::Buf, -1, -1, 0, tail);
  nodes_[id].buf = std::move(buf);
  nodes_[id].clean = clean && tail == 0;
  return id;
}

bool Executor::pending(int node) const {
  const Node& n = nodes_[node];
  return n.op != NOp::Buf && n.op != NOp::Zero && n.op != NOp::OnesMask &&
         n.op != NOp::AllOnes && !n.buf;
}

int Executor::mk(NOp op, int a, int b, int64_t k) {
  const uint8_t ta = a >= 0 ? nodes_[a].tail : 0, tb = b >= 0 ? nodes_[b].tail : 0;
  uint8_t tail = 0;
  switch (op) {
    case NOp::And: tail = ta & tb; break;
    case NOp::Or: tail = ta | tb; break;
    case NOp::Xor: tail = ta ^ tb; break;
    case NOp::Shr: tail = ta; break;
    default: tail = 0; break;
  }
  if (opt_.simplify) {
    auto is = [&](int x, NOp o) { return x >= 0 && nodes_[x].op == o; };
    auto clean = [&](int x) { return nodes_[x].clean != 0; };
    if (commutative(op) && b >= 0 && a > b) std::swap(a, b);
    switch (op) {
      case NOp::And:
        if (a == b) return a;
        if (is(a, NOp::Zero) || is(b, NOp::Zero)) return zero_;
        if (is(a, NOp::AllOnes)) return b;
        if (is(b, NOp::AllOnes)) return a;
        if (is(a, NOp::OnesMask) && clean(b)) return b;
        if (is(b, NOp::OnesMask) && clean(a)) return a;
        break;
      case NOp::Or:
        if (a == b) return a;
        if (is(a, NOp::Zero)) return b;
        if (is(b, NOp::Zero)) return a;
        if (is(a, NOp::AllOnes) || is(b, NOp::AllOnes)) return all_ones_;
        if (is(a, NOp::OnesMask) && clean(b)) return a;
        if (is(b, NOp::OnesMask) && clean(a)) return b;
        break;
      case NOp::Xor:
        if (a == b) return zero_;
        if (is(a, NOp::Zero)) return b;
        if (is(b, NOp::Zero)) return a;
        break;
      case NOp::Not:
        if (is(a, NOp::Zero)) return ones_mask_;
        if (is(a, NOp::OnesMask) || is(a, NOp::AllOnes)) return zero_;
        if (is(a, NOp::Not) && clean(nodes_[a].a)) return nodes_[a].a;
        break;
      case NOp::Add:
        if (is(a, NOp::Zero) && clean(b)) return b;
        if (is(b, NOp::Zero) && clean(a)) return a;
        break;
      case NOp::Shl:
        if (is(a, NOp::Zero) || (!tracing_ && k >= N_)) return zero_;
        if (k == 0 && clean(a)) return a;
        break;
      case NOp::Shr:
        if (k == 0) return a;
        if (is(a, NOp::Zero) || is(a, NOp::AllOnes)) return a;
        break;
      default: break;
    }
    uint64_t key = (static_cast<uint64_t>(op) << 56) ^ (static_cast<uint64_t>(a + 1) << 28) ^
                   static_cast<uint64_t>(b + 1) ^ (static_cast<uint64_t>(k) * 0x9E3779B97F4A7C15ull);
    auto it = cse_.find(key);
    if (it != cse_.end()) {
      const Node& m = nodes_[it->second];
      if (m.op == op && m.a == a && m.b == b && m.k == k) return it->second;
    }
    int id = mk_raw(op, a, b, k, tail);
    cse_[key] = id;
    return id;
  }
  return mk_raw(op, a, b, k, tail);
}

// ------------------------------------------------------------------ walk ---

// Per-class counters on the walk's hot path; op_mix (keyed by the
// reference's op names) is filled from them when the run ends.
void Executor::count(const char* op) {
  ++op_count;
  int k;
  switch (op[0]) {
    case '~': k = 0; break;
    case '&': k = 1; break;
    case '|': k = 2; break;
    case '^': k = 3; break;
    case '+': k = 4; break;
    case '<': k = 5; break;
    case '>': k = 6; break;
    default: k = 7; break;   // popcount
  }
  ++op_class_[k];
}

void Executor::publish_op_mix() {
  static const char* const kNames[8] = {"~", "&", "|", "^", "+", "<<", ">>", "popcount"};
  for (int k = 0; k < 8; ++k)
    if (op_class_[k]) op_mix[kNames[k]] += op_class_[k];
  for (auto& c : op_class_) c = 0;
}

int Executor::read_var(int name) {
  int n = var_[name];
  if (n >= 0) return n;
  if (n == -2)
    throw RuntimeError("internal: variable '" + prog_.names[name] + "' read after being found dead");
  throw RuntimeError("undefined stream variable: " + prog_.names[name]);
}

int Executor::elem(const SExpr& e) {
  int64_t idx = force(ival(*e.index));
  Arr* a = arrs_[e.name].get();
  if (!a || !a->defined) throw RuntimeError("undefined array: " + prog_.names[e.name]);
  auto it = a->elems.find(idx);
  if (it != a->elems.end()) return it->second;
  if (a->broadcast && idx >= 0 && idx < static_cast<int64_t>(a->bcast.size()))
    return a->bcast[idx] ? all_ones_ : zero_;
  return zero_;
}

// Operand read (interpreter.py:70-84): ONES is the N-bit mask here.
int Executor::operand(const SExpr& e) {
  switch (e.kind) {
    case SExpr::Var: return read_var(e.name);
    case SExpr::Zero: return zero_;
    case SExpr::Ones: return ones_mask_;
    case SExpr::Elem: return elem(e);
    default: throw RuntimeError("internal: operand is not a primary");
  }
}

// Right-hand side (interpreter.py:150-218): a copy of ONES is all ones with
// tail 1; ~ + << are masked (the mask is applied by the kernels).
int Executor::rhs(const SExpr& e) {
  switch (e.kind) {
    case SExpr::Var: return read_var(e.name);
    case SExpr::Zero: return zero_;
    case SExpr::Ones: return all_ones_;
    case SExpr::Elem: return elem(e);
    case SExpr::Not: {
      int a = operand(*e.a);
      count("~");
      return mk(NOp::Not, a);
    }
    case SExpr::Bin: {
      int a = operand(*e.a);
      int b = operand(*e.b);
      NOp op = e.op == '&' ? NOp::And : e.op == '|' ? NOp::Or : e.op == '^' ? NOp::Xor : NOp::Add;
      const char* name = e.op == '&' ? "&" : e.op == '|' ? "|" : e.op == '^' ? "^" : "+";
      count(name);
      return mk(op, a, b);
    }
    case SExpr::Shift: {
      int a = operand(*e.a);
      int64_t k = force(ival(*e.index));
      if (k < 0) throw RuntimeError("negative shift count");
      count(e.op == '<' ? "<<" : ">>");
      return mk(e.op == '<' ? NOp::Shl : NOp::Shr, a, -1, k);
    }
  }
  throw RuntimeError("internal: unknown stream expression");
}

Executor::IntV Executor::ival(const IExpr& e) {
  switch (e.kind) {
    case IExpr::Lit: return IntV{e.value, -1};
    case IExpr::Var:
      if (!int_def_[e.name]) throw RuntimeError("undefined int variable: " + prog_.names[e.name]);
      return ints_[e.name];
    case IExpr::Bin: {
      IntV a = ival(*e.a), b = ival(*e.b);
      if (a.e < 0 && b.e < 0) {
        int64_t v = e.op == '+' ? a.v + b.v : e.op == '-' ? a.v - b.v : a.v * b.v;
        return IntV{v, -1};
      }
      auto leaf = [&](const IntV& x) {
        if (x.e >= 0) return x.e;
        iexpr_.push_back(IE{'k', -1, -1, x.v});
        return static_cast<int32_t>(iexpr_.size() - 1);
      };
      int32_t la = leaf(a), lb = leaf(b);
      iexpr_.push_back(IE{e.op, la, lb, 0});
      return IntV{0, static_cast<int32_t>(iexpr_.size() - 1)};
    }
    case IExpr::Pop: {
      if (e.arg->kind != SExpr::Var) throw RuntimeError("popcount arg must be a variable");
      return popcount(read_var(e.arg->name));
    }
  }
  throw RuntimeError("internal: unknown int expression");
}

Executor::IntV Executor::popcount(int node) {
  const Node& n = nodes_[node];
  if (n.tail) throw RuntimeError("popcount on negative value (infinite bits set)");
  count("popcount");
  if (n.op == NOp::Zero) return IntV{0, -1};
  if (n.op == NOp::OnesMask && !tracing_) return IntV{N_, -1};
  if (!tracing_) ensure_slots(1);
  int64_t slot = n_slots_++;
  pending_pops_.push_back({node, slot});
  iexpr_.push_back(IE{'s', -1, -1, slot});
  return IntV{0, static_cast<int32_t>(iexpr_.size() - 1)};
}

int64_t Executor::eval_ie(int32_t e) {
  const IE& x = iexpr_[e];
  switch (x.op) {
    case 'k': return x.v;
    case 's': return static_cast<int64_t>(slot_val_[x.v]);
    case '+': return eval_ie(x.a) + eval_ie(x.b);
    case '-': return eval_ie(x.a) - eval_ie(x.b);
    default: return eval_ie(x.a) * eval_ie(x.b);
  }
}

int64_t Executor::force(const IntV& x) {
  if (x.e < 0) return x.v;
  resolve_slots();
  return eval_ie(x.e);
}

bool Executor::nonzero(int node, const Stmt* at) {
  const Node& n = nodes_[node];
  if (n.tail) return true;                // negative value: nonzero
  if (n.op == NOp::Zero) return false;
  if (n.op == NOp::OnesMask || n.op == NOp::AllOnes) return N_ > 0;
  int x = node;
  auto it = at ? live_->at.find(at->id) : live_->at.end();
  flush(it == live_->at.end() ? nullptr : &it->second, &x);
  if (fused_) fused_->resolve();   // the condition reads the segment's output
  BSZ_CUDA(cudaMemsetAsync(d_flag_, 0, 4, dev_.stream()));
  launch_any(dev_, nodes_[x].buf->p, nw_, d_flag_);
  unsigned int h = 0;
  BSZ_CUDA(cudaMemcpyAsync(&h, d_flag_, 4, cudaMemcpyDeviceToHost, dev_.stream()));
  dev_.sync();
  ++n_syncs;
  if (uint32_t err = dev_.take_error()) throw RuntimeError(describe_device_error(err));
  return h != 0;
}

void Executor::exec_block(const std::vector<Stmt>& v) {
  for (const auto& s : v) {
    exec(s);
    if (!tracing_ && nodes_.size() > nodes_after_flush_ + kAutoFlushNodes) flush(nullptr, nullptr);
  }
}

void Executor::exec(const Stmt& s) {
  switch (s.kind) {
    case Stmt::LocalDecl:
      var_[s.name] = s.e ? rhs(*s.e) : zero_;
      break;
    case Stmt::Assign:
      var_[s.name] = rhs(*s.e);
      break;
    case Stmt::ArrayDecl: {
      int64_t n = force(ival(*s.ie));
      if (!arrs_[s.name]) arrs_[s.name] = std::make_unique<Arr>();
      Arr& a = *arrs_[s.name];
      a.defined = true;
      a.broadcast = false;
      a.bcast.clear();
      a.elems.clear();
      a.decl_size = std::max<int64_t>(n, 0);
      break;
    }
    case Stmt::ArrayAssign: {
      int64_t idx = force(ival(*s.ie));
      int v = rhs(*s.e);
      if (!arrs_[s.name]) arrs_[s.name] = std::make_unique<Arr>();
      Arr& a = *arrs_[s.name];
      a.defined = true;
      a.elems[idx] = v;
      break;
    }
    case Stmt::IntDecl:
    case Stmt::IntAssign:
      ints_[s.name] = ival(*s.ie);
      int_def_[s.name] = 1;
      break;
    case Stmt::If:
      if (nonzero(read_var(s.e->name), &s)) exec_block(s.body);
      break;
    case Stmt::While: {
      for (int it = 0; it < kMaxWhileIters; ++it) {
        if (!nonzero(read_var(s.e->name), &s)) return;
        exec_block(s.body);
      }
      throw RuntimeError("while loop exceeded 10000 iterations");
    }
    case Stmt::For: {
      int64_t lo = force(ival(*s.ie));
      int64_t hi = force(ival(*s.ie2));
      for (int64_t i = lo; i < hi; ++i) {
        ints_[s.name] = IntV{i, -1};
        int_def_[s.name] = 1;
        exec_block(s.body);
      }
      break;
    }
  }
}

namespace {
bool has_control_flow(const std::vector<Stmt>& v) {
  for (const auto& s : v) {
    if (s.kind == Stmt::If || s.kind == Stmt::While) return true;
    if (s.kind == Stmt::For && has_control_flow(s.body)) return true;
  }
  return false;
}
}  // namespace

void Executor::run(bool finish_now) {
  // Programs with if/while on short streams: the whole program, branches
  // included, runs as one launch of the device interpreter (no host round
  // trip per condition) when it qualifies.
  if (!tracing_ && has_control_flow(prog_.stmts) &&
      (opt_.mode == ExecMode::Vm || (opt_.mode == ExecMode::Auto && nw_ <= kVmMaxWords)) &&
      run_vm_program()) {
    ran_as_vm_program = true;
    return;
  }
  // Straight-line programs: restore a cached walk, or walk and cache it when
  // the walk needed no flush (no popcount forced, no automatic flush).
  const bool straight = !tracing_ && !has_control_flow(prog_.stmts);
  std::string key;
  if (straight) key = walk_key();
  walk_replayed = straight && replay_walk(key);
  if (!walk_replayed) {
    const size_t n0 = nodes_.size();
    const int64_t f0 = n_flushes_;
    exec_block(prog_.stmts);
    if (straight && n_flushes_ == f0) save_walk(key, n0);
  }
  flush(&live_->end, nullptr);
  publish_op_mix();
  // Outputs bound to constants get a buffer so the caller can read them.
  auto materialize = [&](int& node) {
    Node& n = nodes_[node];
    if (n.op == NOp::Buf || n.buf) return;
    BufRef b = dev_.alloc_stream(nw_);
    if (n.op == NOp::Zero) launch_fill(dev_, b->p, nw_, 0, 0);
    else if (n.op == NOp::OnesMask) launch_fill(dev_, b->p, nw_, ~uint64_t(0), last_mask_);
    else launch_fill(dev_, b->p, nw_, ~uint64_t(0), ~uint64_t(0));
    node = buf_node(b, n.tail, n.clean);
  };
  for (int id : prog_.outputs) {
    if (var_[id] >= 0) materialize(var_[id]);
    if (arrs_[id])
      for (auto& kv : arrs_[id]->elems) materialize(kv.second);
  }
  if (finish_now) finish();
  else enqueue_readback();
}

void Executor::enqueue_readback() {
  rb_slots_ = n_slots_ - resolved_upto_;
  rb_flags_ = fused_ ? fused_->pending_parts() : 0;
  readback_ = dev_.pinned_block(static_cast<size_t>(8 * rb_slots_ + 4 * rb_flags_ + 8));
  char* h = static_cast<char*>(readback_.get());
  if (rb_slots_ > 0)
    BSZ_CUDA(cudaMemcpyAsync(h, d_slots_ + (resolved_upto_ - slot_base_), static_cast<size_t>(rb_slots_) * 8,
                             cudaMemcpyDeviceToHost, dev_.stream()));
  if (rb_flags_ > 0) fused_->enqueue_flags(reinterpret_cast<uint32_t*>(h + 8 * rb_slots_));
  BSZ_CUDA(cudaMemcpyAsync(h + 8 * rb_slots_ + 4 * rb_flags_, dev_.error_word(), 4, cudaMemcpyDeviceToHost,
                           dev_.stream()));
  if (!done_ev_) BSZ_CUDA(cudaEventCreateWithFlags(&done_ev_, cudaEventDisableTiming));
  BSZ_CUDA(cudaEventRecord(done_ev_, dev_.stream()));
}

void Executor::finish() {
  if (finished_) return;
  if (readback_) {
    // wait for this run's work and read-backs only
    BSZ_CUDA(cudaEventSynchronize(done_ev_));
    const char* h = static_cast<const char*>(readback_.get());
    uint32_t err = 0;
    std::memcpy(&err, h + 8 * rb_slots_ + 4 * rb_flags_, 4);
    const bool reran = rb_flags_ > 0 && fused_->resolve_with(reinterpret_cast<const uint32_t*>(h + 8 * rb_slots_));
    if (!reran && rb_slots_ > 0) {
      std::memcpy(slot_val_.data() + resolved_upto_, h, static_cast<size_t>(rb_slots_) * 8);
      resolved_upto_ += rb_slots_;
    }
    readback_.reset();
    if (err) {
      BSZ_CUDA(cudaMemsetAsync(dev_.error_word(), 0, 4, dev_.stream()));
      throw RuntimeError(describe_device_error(err));
    }
    if (!reran) {
      finished_ = true;
      return;
    }
    // a re-run rewrote popcount slots: read them again below (synchronously)
  }
  if (fused_) fused_->resolve();
  resolve_slots();
  if (uint32_t err = dev_.take_error()) throw RuntimeError(describe_device_error(err));
  finished_ = true;
}

// ----------------------------------------------------------------- flush ---

void Executor::flush(const Bits* live, int* extra) {
  if (tracing_)
    throw RuntimeError("batch execution needs straight-line programs: this one needs the device "
                       "during the walk (a stream condition, or a popcount used as a loop bound, "
                       "index or shift amount)");
  using clk = std::chrono::steady_clock;
  auto ms_since = [](clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); };
  // a fused segment still pending (its speculation unchecked) must be exact
  // before anything runs after it
  if (fused_) fused_->resolve();
  auto t0 = clk::now();
  ++n_flushes_;
  const int n_nodes = static_cast<int>(nodes_.size());
  std::vector<uint8_t> is_target(n_nodes, 0), need(n_nodes, 0);
  Segment seg;
  auto add_target = [&](int n) {
    if (n >= 0 && pending(n) && !is_target[n]) {
      is_target[n] = 1;
      seg.outputs.push_back(n);
    }
  };
  for (size_t v = 0; v < var_.size(); ++v) {
    int n = var_[v];
    if (n < 0 || !pending(n)) continue;
    if (!live || bit(*live, static_cast<int>(v))) add_target(n);
    else var_[v] = -2;
  }
  for (auto& a : arrs_)
    if (a) for (auto& kv : a->elems) add_target(kv.second);
  if (extra) add_target(*extra);
  std::vector<int> stack(seg.outputs.begin(), seg.outputs.end());
  for (auto& p : pending_pops_) stack.push_back(p.first);
  while (!stack.empty()) {
    int n = stack.back();
    stack.pop_back();
    if (need[n]) continue;
    need[n] = 1;
    const Node& x = nodes_[n];
    if (!pending(n)) continue;
    if (x.a >= 0) stack.push_back(x.a);
    if (x.b >= 0) stack.push_back(x.b);
  }
  for (int i = 0; i < n_nodes; ++i) {
    if (!need[i]) continue;
    if (pending(i)) seg.order.push_back(i);
    else seg.inputs.push_back(i);
  }
  for (auto& p : pending_pops_) seg.pops.push_back({p.first, p.second - slot_base_});
  if (!seg.pops.empty()) {
    // this segment's popcount slots (allocated consecutively since the last
    // flush) start at zero: the kernels accumulate into them
    int64_t lo = seg.pops.front().second, hi = lo;
    for (auto& p : seg.pops) {
      lo = std::min(lo, p.second);
      hi = std::max(hi, p.second);
    }
    BSZ_CUDA(cudaMemsetAsync(d_slots_ + lo, 0, static_cast<size_t>(hi - lo + 1) * 8, dev_.stream()));
  }
  t_segment_ms += ms_since(t0);
  if (!seg.order.empty() || !seg.pops.empty()) {
    ++n_segments;
    auto t1 = clk::now();
    bool fuse = false, vm = false;
    switch (opt_.mode) {
      case ExecMode::Plain: break;
      case ExecMode::Vm: vm = true; break;
      case ExecMode::Fused: fuse = seg.order.size() <= kMaxFusedOps; break;
      case ExecMode::Auto:
        if (nw_ <= kVmMaxWords) vm = true;
        else fuse = seg.order.size() <= kMaxFusedOps && fused_pays(seg);
        break;
    }
    t_policy_ms += ms_since(t1);
    auto t2 = clk::now();
    if (vm) {
      run_vm(seg);
    } else if (fuse) {
      // constants need no buffer: the generated code computes their words
      fused_->run(nodes_, seg, N_, nw_, d_slots_, &compile_ms);
    } else {
      run_plain(seg);
    }
    t_run_ms += ms_since(t2);
  }
  auto t3 = clk::now();
  pending_pops_.clear();
  max_live_buffers = std::max(max_live_buffers, live_buffer_count());
  compact(extra);
  t_compact_ms += ms_since(t3);
}

int64_t Executor::live_buffer_count() const {
  int64_t c = 0;
  for (const auto& n : nodes_)
    if (n.buf) ++c;
  return c;
}

const uint64_t* Executor::const_ptr(int node) {
  Node& n = nodes_[node];
  if (n.buf) return n.buf->p;
  BufRef* slot = nullptr;
  uint64_t v = 0, last = 0;
  switch (n.op) {
    case NOp::Zero: slot = &c_zero_; v = 0; last = 0; break;
    case NOp::OnesMask: slot = &c_mask_; v = ~uint64_t(0); last = last_mask_; break;
    case NOp::AllOnes: slot = &c_all_; v = ~uint64_t(0); last = ~uint64_t(0); break;
    default: throw RuntimeError("internal: operand not materialized");
  }
  if (!*slot) {
    *slot = dev_.alloc_stream(nw_);
    launch_fill(dev_, (*slot)->p, nw_, v, last);
  }
  return (*slot)->p;
}

void Executor::run_plain(const Segment& seg) {
  const int n_nodes = static_cast<int>(nodes_.size());
  std::vector<int> uses(n_nodes, 0);
  std::vector<uint8_t> keep(n_nodes, 0);
  for (int o : seg.outputs) keep[o] = 1;
  std::vector<std::vector<int64_t>> pops_of(n_nodes);
  for (auto& p : seg.pops) pops_of[p.first].push_back(p.second);
  for (int id : seg.order) {
    const Node& n = nodes_[id];
    if (n.a >= 0 && pending(n.a)) ++uses[n.a];
    if (n.b >= 0 && pending(n.b)) ++uses[n.b];
  }
  auto launch_pops = [&](int id) {
    for (int64_t slot : pops_of[id])
      launch_popcount(dev_, nodes_[id].buf ? nodes_[id].buf->p : const_ptr(id), nw_, d_slots_ + slot);
  };
  for (int i : seg.inputs) launch_pops(i);
  for (int id : seg.order) {
    Node& n = nodes_[id];
    const uint64_t* A = n.a >= 0 ? (nodes_[n.a].buf ? nodes_[n.a].buf->p : const_ptr(n.a)) : nullptr;
    const uint64_t* B = n.b >= 0 ? (nodes_[n.b].buf ? nodes_[n.b].buf->p : const_ptr(n.b)) : nullptr;
    BufRef out = dev_.alloc_stream(nw_);
    uint64_t* D = out->p;
    switch (n.op) {
      case NOp::Not: launch_not(dev_, D, A, nw_, last_mask_); break;
      case NOp::And: launch_bitwise(dev_, kAnd, D, A, B, nw_); break;
      case NOp::Or: launch_bitwise(dev_, kOr, D, A, B, nw_); break;
      case NOp::Xor: launch_bitwise(dev_, kXor, D, A, B, nw_); break;
      case NOp::AndNot: launch_bitwise(dev_, kAndNot, D, A, B, nw_); break;
      case NOp::Add: launch_add(dev_, D, A, B, nw_, last_mask_); break;
      case NOp::Shl: launch_shl(dev_, D, A, n.k, nw_, last_mask_); break;
      case NOp::Shr:
        launch_shr(dev_, D, A, n.k, nw_, nodes_[n.a].tail ? ~uint64_t(0) : 0);
        break;
      default: throw RuntimeError("internal: unexpected node in plain segment");
    }
    n.buf = std::move(out);
    launch_pops(id);
    for (int operand : {n.a, n.b}) {
      if (operand >= 0 && pending(operand) == false && nodes_[operand].op != NOp::Buf &&
          uses[operand] > 0 && --uses[operand] == 0 && !keep[operand])
        nodes_[operand].buf.reset();
    }
  }
  max_live_buffers = std::max(max_live_buffers, live_buffer_count());
}

// Auto mode, long streams: a generated kernel pays when it is already
// compiled (in this process or in the on-disk cache), or when the segment's
// per-op form would take longer than compiling it.  Per-op time: launch
// (~4 us) plus 24 bytes per word at HBM speed; compile time ~60 ms plus
// ~0.4 ms per operation.
bool Executor::fused_pays(const Segment& seg) {
  const double ops = static_cast<double>(seg.order.size() + seg.pops.size());
  const double per_op_ms = 0.004 + 24.0 * static_cast<double>(nw_) / 6.5e9;
  const double compile_ms_est = 60.0 + 0.4 * static_cast<double>(seg.order.size());
  if (ops * per_op_ms > compile_ms_est) return true;
  return fused_->all_compiled(nodes_, seg, N_);
}

void Executor::run_vm(const Segment& seg) {
  const int n_nodes = static_cast<int>(nodes_.size());
  constexpr int32_t kNone = INT32_MIN;
  std::vector<int32_t> loc(n_nodes, kNone);
  std::vector<const uint64_t*> ext;
  auto ext_of = [&](const uint64_t* p) {
    ext.push_back(p);
    return -static_cast<int32_t>(ext.size());
  };
  for (int i : seg.inputs) loc[i] = ext_of(nodes_[i].buf ? nodes_[i].buf->p : const_ptr(i));
  std::vector<uint8_t> is_out(n_nodes, 0);
  for (int o : seg.outputs) is_out[o] = 1;
  std::vector<int64_t> last(n_nodes, -1);
  for (size_t t = 0; t < seg.order.size(); ++t) {
    const Node& x = nodes_[seg.order[t]];
    if (x.a >= 0) last[x.a] = static_cast<int64_t>(t);
    if (x.b >= 0) last[x.b] = static_cast<int64_t>(t);
  }
  // popcounts sorted by node (segment order is increasing node id)
  std::vector<std::pair<int, int64_t>> pops(seg.pops.begin(), seg.pops.end());
  std::stable_sort(pops.begin(), pops.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
  std::vector<VmOp> ops;
  ops.reserve(seg.order.size() + pops.size());
  auto emit_pops = [&](int node) {
    auto it = std::lower_bound(pops.begin(), pops.end(), std::make_pair(node, int64_t(INT64_MIN)));
    for (; it != pops.end() && it->first == node; ++it) {
      VmOp op{};
      op.code = kVmPop;
      op.a = loc[node];
      op.dst = static_cast<int32_t>(it->second);
      ops.push_back(op);
    }
  };
  for (int i : seg.inputs) emit_pops(i);
  std::vector<int32_t> free_slots;
  int32_t n_slots = 0;
  const int64_t kmax = 64 * nw_;
  for (size_t t = 0; t < seg.order.size(); ++t) {
    const int id = seg.order[t];
    Node& n = nodes_[id];
    int32_t dst;
    if (is_out[id]) {
      n.buf = dev_.alloc_stream(nw_);
      dst = ext_of(n.buf->p);
    } else if (!free_slots.empty()) {
      dst = free_slots.back();
      free_slots.pop_back();
    } else {
      dst = n_slots++;
    }
    loc[id] = dst;
    VmOp op{};
    op.dst = dst;
    op.a = loc[n.a];
    switch (n.op) {
      case NOp::Not: op.code = kVmNot; break;
      case NOp::And: op.code = kVmAnd; op.b = loc[n.b]; break;
      case NOp::Or: op.code = kVmOr; op.b = loc[n.b]; break;
      case NOp::Xor: op.code = kVmXor; op.b = loc[n.b]; break;
      case NOp::AndNot: op.code = kVmAndNot; op.b = loc[n.b]; break;
      case NOp::Add: op.code = kVmAdd; op.b = loc[n.b]; break;
      case NOp::Shl: op.code = kVmShl; op.b = static_cast<int32_t>(std::min<int64_t>(n.k, kmax)); break;
      case NOp::Shr:
        op.code = kVmShr;
        op.b = static_cast<int32_t>(std::min<int64_t>(n.k, kmax));
        op.fill = nodes_[n.a].tail ? 1 : 0;
        break;
      default: throw RuntimeError("internal: unexpected node in VM segment");
    }
    if (op.a == kNone || ((n.op == NOp::And || n.op == NOp::Or || n.op == NOp::Xor || n.op == NOp::AndNot ||
                           n.op == NOp::Add) && op.b == kNone))
      throw RuntimeError("internal: VM operand has no location");
    ops.push_back(op);
    emit_pops(id);
    for (int operand : {n.a, n.b}) {
      if (operand < 0 || loc[operand] < 0 || last[operand] != static_cast<int64_t>(t)) continue;
      if (operand == n.b && n.a == n.b) continue;   // x op x: free once
      free_slots.push_back(loc[operand]);
    }
    if (!is_out[id] && last[id] < 0) free_slots.push_back(dst);   // computed only for its popcounts
  }
  if (ops.empty()) return;
  // device copies: instruction list | pointer table | slot file (if global)
  auto align = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t ops_b = ops.size() * sizeof(VmOp);
  const size_t ext_b = std::max<size_t>(1, ext.size()) * sizeof(uint64_t*);
  const bool smem = vm_smem_bytes(n_slots, nw_) > 0;
  const size_t file_b = smem ? 0 : static_cast<size_t>(n_slots) * static_cast<size_t>(nw_) * 8;
  const size_t total = align(ops_b) + align(ext_b) + file_b;
  if (total > vm_cap_) {
    // the old block returns to the device cache; stream order keeps it
    // alive for work already queued on it
    vm_cap_ = std::max<size_t>(total, size_t(1) << 20);
    vm_mem_ = dev_.alloc_stream(static_cast<int64_t>((vm_cap_ + 7) / 8));
    vm_buf_ = vm_mem_->p;
  }
  char* base = static_cast<char*>(vm_buf_);
  VmOp* d_ops = reinterpret_cast<VmOp*>(base);
  const uint64_t** d_ext = reinterpret_cast<const uint64_t**>(base + align(ops_b));
  uint64_t* d_file = smem ? nullptr : reinterpret_cast<uint64_t*>(base + align(ops_b) + align(ext_b));
  BSZ_CUDA(cudaMemcpyAsync(d_ops, ops.data(), ops_b, cudaMemcpyHostToDevice, dev_.stream()));
  if (!ext.empty())
    BSZ_CUDA(cudaMemcpyAsync(d_ext, ext.data(), ext.size() * sizeof(uint64_t*), cudaMemcpyHostToDevice,
                             dev_.stream()));
  VmLaunch L{d_ops, static_cast<int64_t>(ops.size()), d_ext, d_file, n_slots, nw_, last_mask_, d_slots_};
  launch_vm(dev_, L);
  ++vm_launches;
  max_live_buffers = std::max(max_live_buffers, live_buffer_count() + n_slots);
}

void Executor::compact(int* extra) {
  std::vector<Node> old;
  old.swap(nodes_);
  cse_.clear();
  std::vector<int> remap(old.size(), -1);
  zero_ = mk_raw(NOp::Zero, -1, -1, 0, 0);
  ones_mask_ = mk_raw(NOp::OnesMask, -1, -1, 0, 0);
  all_ones_ = mk_raw(NOp::AllOnes, -1, -1, 0, 1);
  auto map = [&](int n) -> int {
    if (n < 0) return n;
    if (remap[n] >= 0) return remap[n];
    const Node& x = old[n];
    int id;
    switch (x.op) {
      case NOp::Zero: id = zero_; break;
      case NOp::OnesMask: id = ones_mask_; break;
      case NOp::AllOnes: id = all_ones_; break;
      default:
        if (!x.buf) throw RuntimeError("internal: live value was not materialized");
        id = buf_node(x.buf, x.tail, x.clean);
    }
    remap[n] = id;
    return id;
  };
  for (auto& v : var_) v = map(v);
  for (auto& a : arrs_)
    if (a) for (auto& kv : a->elems) kv.second = map(kv.second);
  if (extra) *extra = map(*extra);
  nodes_after_flush_ = nodes_.size();
}

// ----------------------------------------------------------------- slots ---

void Executor::ensure_slots(int64_t need) {
  if (slot_cap_ == 0) {
    slot_cap_ = kSlotChunk;
    slots_buf_ = dev_.alloc_stream(slot_cap_);
    d_slots_ = reinterpret_cast<unsigned long long*>(slots_buf_->p);
  }
  if (n_slots_ - slot_base_ + need > slot_cap_) {
    resolve_slots();
    slot_base_ = n_slots_;
  }
  // (the slots a segment accumulates into are zeroed when it runs: flush())
  if (static_cast<int64_t>(slot_val_.size()) < n_slots_ + need) slot_val_.resize(n_slots_ + need + 1024);
}

void Executor::resolve_slots() {
  if (!pending_pops_.empty()) flush(nullptr, nullptr);
  if (fused_) fused_->resolve();
  if (resolved_upto_ < n_slots_) {
    int64_t from = resolved_upto_ - slot_base_;
    int64_t cnt = n_slots_ - resolved_upto_;
    BSZ_CUDA(cudaMemcpyAsync(slot_val_.data() + resolved_upto_, d_slots_ + from,
                             static_cast<size_t>(cnt) * 8, cudaMemcpyDeviceToHost, dev_.stream()));
    dev_.sync();
    ++n_syncs;
    resolved_upto_ = n_slots_;
  }
}

// -------------------------------------------------------------- liveness ---
// Backward dataflow over the AST: for every if/while statement, the scalar
// stream names that may be read at or after it (loops iterate to a fixed
// point).  At a flush only those values are materialized; temporaries that
// are dead there are never computed.

std::shared_ptr<const Executor::Liveness> Executor::compute_liveness() const {
  auto live = std::make_shared<Liveness>();
  auto& live_at = live->at;
  const int nn = static_cast<int>(prog_.names.size());
  const size_t nb = (static_cast<size_t>(nn) + 63) / 64;
  auto scalar = [&](int id) { return id >= 0 && !prog_.is_array[id]; };
  std::function<void(const IExpr&, Bits&)> gen_i;
  std::function<void(const SExpr&, Bits&)> gen_s = [&](const SExpr& e, Bits& L) {
    switch (e.kind) {
      case SExpr::Var: if (scalar(e.name)) set_bit(L, e.name); break;
      case SExpr::Elem: gen_i(*e.index, L); break;
      case SExpr::Not: gen_s(*e.a, L); break;
      case SExpr::Bin: gen_s(*e.a, L); gen_s(*e.b, L); break;
      case SExpr::Shift: gen_s(*e.a, L); gen_i(*e.index, L); break;
      default: break;
    }
  };
  gen_i = [&](const IExpr& e, Bits& L) {
    if (e.kind == IExpr::Pop) gen_s(*e.arg, L);
    else if (e.kind == IExpr::Bin) { gen_i(*e.a, L); gen_i(*e.b, L); }
  };
  std::function<Bits(const std::vector<Stmt>&, Bits)> block = [&](const std::vector<Stmt>& v, Bits L) {
    for (auto it = v.rbegin(); it != v.rend(); ++it) {
      const Stmt& s = *it;
      switch (s.kind) {
        case Stmt::LocalDecl:
        case Stmt::Assign:
          if (scalar(s.name)) clr_bit(L, s.name);
          if (s.e) gen_s(*s.e, L);
          break;
        case Stmt::ArrayAssign: gen_s(*s.e, L); gen_i(*s.ie, L); break;
        case Stmt::ArrayDecl: gen_i(*s.ie, L); break;
        case Stmt::IntDecl:
        case Stmt::IntAssign: gen_i(*s.ie, L); break;
        case Stmt::If: {
          Bits in = block(s.body, L);
          or_into(L, in);
          set_bit(L, s.e->name);
          live_at[s.id] = L;
          break;
        }
        case Stmt::While: {
          const Bits out = L;
          Bits X = out;
          set_bit(X, s.e->name);
          for (int guard = 0; guard < 1000; ++guard) {
            Bits B = block(s.body, X);
            Bits Xn = out;
            or_into(Xn, B);
            set_bit(Xn, s.e->name);
            if (Xn == X) break;
            X = std::move(Xn);
          }
          live_at[s.id] = X;
          L = X;
          break;
        }
        case Stmt::For: {
          gen_i(*s.ie, L);
          gen_i(*s.ie2, L);
          const Bits out = L;
          Bits X = out;
          for (int guard = 0; guard < 1000; ++guard) {
            Bits B = block(s.body, X);
            Bits Xn = out;
            or_into(Xn, B);
            if (Xn == X) break;
            X = std::move(Xn);
          }
          L = X;
          break;
        }
      }
    }
    return L;
  };
  live->end.assign(nb, 0);
  for (int id : prog_.outputs)
    if (scalar(id)) set_bit(live->end, id);
  block(prog_.stmts, live->end);
  return live;
}

// --------------------------------------------------------------- results ---

bool Executor::has_stream(int name) const { return name >= 0 && var_[name] >= 0; }

BufRef Executor::stream_value(int name) {
  if (!has_stream(name)) return nullptr;
  Node& n = nodes_[var_[name]];
  return n.buf;
}

uint8_t Executor::stream_tail(int name) const { return has_stream(name) ? nodes_[var_[name]].tail : 0; }

bool Executor::has_array(int name) const {
  return name >= 0 && arrs_[name] && arrs_[name]->defined;
}

std::vector<int64_t> Executor::array_indices(int name) const {
  std::vector<int64_t> idx;
  if (!has_array(name)) return idx;
  const Arr& a = *arrs_[name];
  for (int64_t i = 0; i < a.decl_size; ++i) idx.push_back(i);
  if (a.broadcast)
    for (int64_t i = 0; i < static_cast<int64_t>(a.bcast.size()); ++i) idx.push_back(i);
  for (auto& kv : a.elems) idx.push_back(kv.first);
  std::sort(idx.begin(), idx.end());
  idx.erase(std::unique(idx.begin(), idx.end()), idx.end());
  return idx;
}

BufRef Executor::array_value(int name, int64_t idx) {
  if (!has_array(name)) return nullptr;
  Arr& a = *arrs_[name];
  auto it = a.elems.find(idx);
  int node;
  if (it != a.elems.end()) node = it->second;
  else if (a.broadcast && idx >= 0 && idx < static_cast<int64_t>(a.bcast.size()))
    node = a.bcast[idx] ? all_ones_ : zero_;
  else node = zero_;
  if (!nodes_[node].buf) const_ptr(node);
  Node& n = nodes_[node];
  if (n.buf) return n.buf;
  return n.op == NOp::Zero ? c_zero_ : n.op == NOp::OnesMask ? c_mask_ : c_all_;
}

bool Executor::int_value(int name, int64_t* v) {
  if (name < 0 || !int_def_[name]) return false;
  *v = force(ints_[name]);
  return true;
}

}  // namespace bsz

// ----------------------------------------------------------------- trace ---

namespace bsz {

Executor::Traced Executor::trace() {
  tracing_ = true;
  Traced t;
  for (int id : prog_.inputs) {
    if (prog_.is_array[id]) throw RuntimeError("batch execution does not take input arrays");
    int n = buf_node(nullptr, 0, false);   // symbolic input: no buffer, length-independent
    var_[id] = n;
    t.input_nodes.push_back(n);
  }
  exec_block(prog_.stmts);
  for (int id : prog_.outputs) {
    if (prog_.is_array[id]) throw RuntimeError("batch execution does not produce output arrays");
    t.output_nodes.push_back(var_[id] >= 0 ? var_[id] : -1);
  }
  t.pops = pending_pops_;
  std::function<void(int32_t, std::vector<std::pair<char, int64_t>>&)> post =
      [&](int32_t e, std::vector<std::pair<char, int64_t>>& out) {
        const IE& x = iexpr_[e];
        if (x.op == 'k' || x.op == 's') {
          out.push_back({x.op, x.v});
          return;
        }
        post(x.a, out);
        post(x.b, out);
        out.push_back({x.op, 0});
      };
  for (int id : prog_.output_ints) {
    std::vector<std::pair<char, int64_t>> prog;
    const IntV& v = ints_[id];
    if (v.e < 0) prog.push_back({'k', v.v});
    else post(v.e, prog);
    t.int_outputs.push_back(std::move(prog));
  }
  t.nodes = nodes_;
  t.op_count = op_count;
  tracing_ = false;
  return t;
}

}  // namespace bsz
