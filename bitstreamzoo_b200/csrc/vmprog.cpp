// Whole programs on the device interpreter: the AST, control flow included,
// compiled to one instruction list that a single CTA runs (vm.cu, program
// mode).  An if/while condition is a CTA-wide OR on the device, so a program
// such as a multi-pattern regex matcher (thousands of `if` guards, a while
// loop per MatchStar fixpoint) costs one launch and one read-back instead of
// one host round trip per condition.
//
// Compilation mirrors the host walk (engine.cpp: exec, rhs, operand, ival,
// popcount; the reference's interpreter.py:30-253): every scalar stream
// variable and array element gets a fixed slot (assignments overwrite it, so
// the branches need no merge), for-loops unroll with host-known bounds,
// ints known on the host stay constants, and ints that depend on a popcount
// or on a branch live in device registers.  Tails are device state because a
// branch can change them.  Op counts are counted on the device per class.
//
// A program runs here only if nothing in it needs the host mid-run: a device
// int used as a loop bound, array index, array size or shift amount; an
// array declared, or an array element created, under a condition; a
// variable read after the region that alone defined it; a for-loop that
// assigns its own variable; a read of an undefined name.  Any of these makes
// compile throw NotEligible and the executor falls back to its host-driven
// walk (which also reports the reference's errors for bad programs).
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "engine.h"
#include "vm.h"

namespace bsz {

namespace {
struct NotEligible {};
constexpr int32_t kSlotZero = 0, kSlotMask = 1, kSlotAll = 2, kSlotTmp = 3, kFixedSlots = 4;
}  // namespace

struct VmCompiler {
  Executor& ex;
  const Program& prog;
  std::vector<VmOp> code;
  std::vector<const uint64_t*> ext;
  int32_t n_slots = kFixedSlots;
  int32_t n_iregs = 0;
  int depth = 0;
  int32_t zero_reg = -1;

  // scalar streams
  std::vector<int32_t> slot_of;
  std::vector<uint8_t> cond_only;   // not reliably defined at this point
  // ints
  struct IntVal {
    bool def = false;
    bool dev = false;
    int64_t v = 0;
    int32_t reg = -1;
  };
  std::vector<IntVal> ints;
  std::vector<uint8_t> int_cond_only;
  // arrays
  struct ArrC {
    bool defined = false;
    bool broadcast = false;
    std::vector<uint8_t> bcast;
    int64_t decl_size = 0;
    std::map<int64_t, int32_t> elems;
  };
  std::vector<ArrC> arrs;
  // names (re)defined inside each open region without being reliably
  // defined before it
  std::vector<std::vector<int>> region_streams, region_ints;

  explicit VmCompiler(Executor& e) : ex(e), prog(e.prog_) {
    const size_t nn = prog.names.size();
    slot_of.assign(nn, -1);
    cond_only.assign(nn, 0);
    ints.assign(nn, IntVal{});
    int_cond_only.assign(nn, 0);
    arrs.assign(nn, ArrC{});
  }

  void op(VmCode c, int32_t dst, int32_t a = 0, int32_t b = 0, uint8_t cls = kClsNone, uint8_t fill = 0) {
    VmOp o{};
    o.code = c;
    o.dst = dst;
    o.a = a;
    o.b = b;
    o.cls = cls;
    o.fill = fill;
    code.push_back(o);
  }
  int32_t new_slot() { return n_slots++; }
  int32_t new_ireg() { return n_iregs++; }
  int32_t ext_of(const uint64_t* p) {
    ext.push_back(p);
    return static_cast<int32_t>(ext.size() - 1);
  }
  void iconst(int32_t reg, int64_t v) {
    const uint64_t u = static_cast<uint64_t>(v);
    op(kVmIConst, reg, static_cast<int32_t>(static_cast<uint32_t>(u)),
       static_cast<int32_t>(static_cast<uint32_t>(u >> 32)));
  }

  // ---- initial state from the executor's bindings
  void load_value(int node, int32_t slot) {
    const Node& n = ex.nodes_[node];
    switch (n.op) {
      case NOp::Zero: op(kVmCopy, slot, kSlotZero); break;
      case NOp::OnesMask: op(kVmCopy, slot, kSlotMask); break;
      case NOp::AllOnes: op(kVmCopy, slot, kSlotAll); break;
      case NOp::Buf: op(kVmLoad, slot, ext_of(n.buf->p), 0, kClsNone, n.tail); break;
      default: throw NotEligible{};   // a pending computation: not a fresh run
    }
  }

  void init() {
    op(kVmFill, kSlotZero, 0, 0, kClsNone, 0);
    op(kVmFill, kSlotMask, 0, 0, kClsNone, 1);
    op(kVmFill, kSlotAll, 0, 0, kClsNone, 2);
    zero_reg = new_ireg();
    iconst(zero_reg, 0);
    for (size_t id = 0; id < prog.names.size(); ++id) {
      if (ex.var_[id] >= 0) {
        slot_of[id] = new_slot();
        load_value(ex.var_[id], slot_of[id]);
      }
      if (ex.arrs_[id]) {
        const auto& a = *ex.arrs_[id];
        ArrC& c = arrs[id];
        c.defined = a.defined;
        c.broadcast = a.broadcast;
        c.bcast = a.bcast;
        c.decl_size = a.decl_size;
        for (auto& kv : a.elems) {
          const int32_t s = new_slot();
          load_value(kv.second, s);
          c.elems[kv.first] = s;
        }
      }
      if (ex.int_def_[id]) {
        if (ex.ints_[id].e >= 0) throw NotEligible{};
        ints[id].def = true;
        ints[id].v = ex.ints_[id].v;
      }
    }
  }

  // ---- definedness
  bool defined(int name) const { return slot_of[name] >= 0 && !cond_only[name]; }
  bool int_defined(int name) const { return ints[name].def && !int_cond_only[name]; }

  // Destination of an assignment to `name`.  A name (re)defined inside a
  // region that it was not reliably defined before becomes conditionally
  // defined again when the region ends.
  int32_t slot_for_write(int name) {
    const bool fresh = !defined(name);
    if (slot_of[name] < 0) slot_of[name] = new_slot();
    if (depth > 0 && fresh) region_streams.back().push_back(name);
    cond_only[name] = 0;
    return slot_of[name];
  }
  void mark_int_defined(int name) {
    if (depth > 0 && !int_defined(name)) region_ints.back().push_back(name);
    ints[name].def = true;
    int_cond_only[name] = 0;
  }

  // ---- reads
  int32_t read_var(int name) {
    if (!defined(name)) throw NotEligible{};
    return slot_of[name];
  }
  IntVal read_int(int name) {
    if (!int_defined(name)) throw NotEligible{};
    return ints[name];
  }
  int64_t host_int(const IExpr& e) {
    IntVal v = ival(e);
    if (v.dev) throw NotEligible{};
    return v.v;
  }
  int32_t elem_slot(const SExpr& e) {
    const int64_t idx = host_int(*e.index);
    ArrC& a = arrs[e.name];
    if (!a.defined) throw NotEligible{};
    auto it = a.elems.find(idx);
    if (it != a.elems.end()) return it->second;
    if (a.broadcast && idx >= 0 && idx < static_cast<int64_t>(a.bcast.size()))
      return a.bcast[idx] ? kSlotAll : kSlotZero;
    return kSlotZero;
  }
  // operand read: ONES is the N-bit mask
  int32_t operand(const SExpr& e) {
    switch (e.kind) {
      case SExpr::Var: return read_var(e.name);
      case SExpr::Zero: return kSlotZero;
      case SExpr::Ones: return kSlotMask;
      case SExpr::Elem: return elem_slot(e);
      default: throw NotEligible{};
    }
  }
  static bool refs(const SExpr& e, int name) {
    if ((e.kind == SExpr::Var || e.kind == SExpr::Elem) && e.name == name) return true;
    return (e.a && refs(*e.a, name)) || (e.b && refs(*e.b, name));
  }

  // ---- int expressions
  int32_t as_reg(const IntVal& v) {
    if (v.dev) return v.reg;
    const int32_t r = new_ireg();
    iconst(r, v.v);
    return r;
  }
  IntVal ival(const IExpr& e) {
    switch (e.kind) {
      case IExpr::Lit: return IntVal{true, false, e.value, -1};
      case IExpr::Var: return read_int(e.name);
      case IExpr::Bin: {
        IntVal a = ival(*e.a), b = ival(*e.b);
        if (!a.dev && !b.dev) {
          const uint64_t x = static_cast<uint64_t>(a.v), y = static_cast<uint64_t>(b.v);
          const uint64_t r = e.op == '+' ? x + y : e.op == '-' ? x - y : x * y;
          return IntVal{true, false, static_cast<int64_t>(r), -1};
        }
        const int32_t ra = as_reg(a), rb = as_reg(b), rd = new_ireg();
        op(e.op == '+' ? kVmIAdd : e.op == '-' ? kVmISub : kVmIMul, rd, ra, rb);
        return IntVal{true, true, 0, rd};
      }
      case IExpr::Pop: {
        if (e.arg->kind != SExpr::Var) throw NotEligible{};
        const int32_t s = read_var(e.arg->name), rd = new_ireg();
        op(kVmPopI, rd, s, 0, kClsPop);
        return IntVal{true, true, 0, rd};
      }
    }
    throw NotEligible{};
  }

  // ---- stream right-hand sides, written into `dst`
  void rhs(const SExpr& e, int32_t dst) {
    switch (e.kind) {
      case SExpr::Var: op(kVmCopy, dst, read_var(e.name)); return;
      case SExpr::Zero: op(kVmCopy, dst, kSlotZero); return;
      case SExpr::Ones: op(kVmCopy, dst, kSlotAll); return;   // a copy of ONES: all ones, tail 1
      case SExpr::Elem: op(kVmCopy, dst, elem_slot(e)); return;
      case SExpr::Not: op(kVmNot, dst, operand(*e.a), 0, kClsNot); return;
      case SExpr::Bin: {
        const int32_t a = operand(*e.a), b = operand(*e.b);
        switch (e.op) {
          case '&': op(kVmAnd, dst, a, b, kClsAnd); return;
          case '|': op(kVmOr, dst, a, b, kClsOr); return;
          case '^': op(kVmXor, dst, a, b, kClsXor); return;
          default: op(kVmAdd, dst, a, b, kClsAdd); return;
        }
      }
      case SExpr::Shift: {
        const int32_t a = operand(*e.a);
        const int64_t k = host_int(*e.index);
        if (k < 0) {   // raised only if this instruction runs
          op(kVmErr, 0, kVmErrNegShift);
          return;
        }
        const int32_t kk = static_cast<int32_t>(std::min<int64_t>(k, 64 * ex.nw_));
        // a shift reads other threads' words: never in place
        const int32_t t = (a == dst) ? kSlotTmp : dst;
        op(e.op == '<' ? kVmShl : kVmShr, t, a, kk, e.op == '<' ? kClsShl : kClsShr);
        if (t != dst) op(kVmCopy, dst, t);
        return;
      }
    }
    throw NotEligible{};
  }

  void assign_int(int name, const IntVal& v) {
    IntVal& t = ints[name];
    if (depth == 0) {
      t = v;
      t.def = true;
      int_cond_only[name] = 0;
      return;
    }
    // inside a region the target lives in a register (set up by prescan)
    if (!t.dev) throw NotEligible{};
    if (v.dev) op(kVmIAdd, t.reg, v.reg, zero_reg);
    else iconst(t.reg, v.v);
    mark_int_defined(name);
  }

  // Ints assigned anywhere in a conditional body become device registers
  // before the branch, holding their current value, so that both paths
  // leave the right value behind.
  void prescan(const std::vector<Stmt>& body) {
    for (const auto& s : body) {
      int name = -1;
      if (s.kind == Stmt::IntDecl || s.kind == Stmt::IntAssign || s.kind == Stmt::For) name = s.name;
      if (name >= 0 && !ints[name].dev) {
        IntVal& t = ints[name];
        const int32_t r = new_ireg();
        if (int_defined(name)) iconst(r, t.v);
        else int_cond_only[name] = 1;   // not defined on this path yet
        t.dev = true;
        t.reg = r;
      }
      if (s.kind == Stmt::If || s.kind == Stmt::While || s.kind == Stmt::For) prescan(s.body);
    }
  }

  void enter_region() {
    region_streams.emplace_back();
    region_ints.emplace_back();
  }
  void leave_region() {
    for (int n : region_streams.back()) cond_only[n] = 1;
    for (int n : region_ints.back()) int_cond_only[n] = 1;
    region_streams.pop_back();
    region_ints.pop_back();
  }

  static bool assigns_int(const std::vector<Stmt>& body, int name) {
    for (const auto& s : body) {
      if ((s.kind == Stmt::IntDecl || s.kind == Stmt::IntAssign || s.kind == Stmt::For) && s.name == name)
        return true;
      if ((s.kind == Stmt::If || s.kind == Stmt::While || s.kind == Stmt::For) && assigns_int(s.body, name))
        return true;
    }
    return false;
  }

  void stmts(const std::vector<Stmt>& v) {
    for (const auto& s : v) stmt(s);
  }

  void stmt(const Stmt& s) {
    switch (s.kind) {
      case Stmt::LocalDecl:
      case Stmt::Assign: {
        if (!s.e) {
          op(kVmCopy, slot_for_write(s.name), kSlotZero);
          return;
        }
        // a right-hand side that reads the target needs its old value
        if (!defined(s.name) && refs(*s.e, s.name)) throw NotEligible{};
        const int32_t d = slot_for_write(s.name);
        rhs(*s.e, d);
        return;
      }
      case Stmt::ArrayDecl: {
        if (depth > 0) throw NotEligible{};
        const int64_t n = host_int(*s.ie);
        ArrC& a = arrs[s.name];
        a.defined = true;
        a.broadcast = false;
        a.bcast.clear();
        a.elems.clear();
        a.decl_size = std::max<int64_t>(n, 0);
        return;
      }
      case Stmt::ArrayAssign: {
        const int64_t idx = host_int(*s.ie);
        ArrC& a = arrs[s.name];
        auto it = a.elems.find(idx);
        int32_t d;
        if (it == a.elems.end()) {
          if (depth > 0) throw NotEligible{};   // the element set would depend on the branch
          d = new_slot();
        } else {
          d = it->second;
        }
        rhs(*s.e, d);
        a.defined = true;
        a.elems[idx] = d;
        return;
      }
      case Stmt::IntDecl:
      case Stmt::IntAssign:
        assign_int(s.name, ival(*s.ie));
        return;
      case Stmt::If: {
        const int32_t c = read_var(s.e->name);
        enter_region();
        prescan(s.body);
        const size_t jz = code.size();
        op(kVmJz, 0, c, 0);
        ++depth;
        stmts(s.body);
        --depth;
        leave_region();
        code[jz].b = static_cast<int32_t>(code.size());
        return;
      }
      case Stmt::While: {
        enter_region();
        prescan(s.body);
        const int32_t ctr = new_ireg();
        iconst(ctr, 0);
        const int32_t top = static_cast<int32_t>(code.size());
        const int32_t c = read_var(s.e->name);
        const size_t jz = code.size();
        op(kVmJz, 0, c, 0);
        op(kVmTick, ctr);
        ++depth;
        stmts(s.body);
        --depth;
        leave_region();
        op(kVmJmp, 0, 0, top);
        code[jz].b = static_cast<int32_t>(code.size());
        return;
      }
      case Stmt::For: {
        const int64_t lo = host_int(*s.ie), hi = host_int(*s.ie2);
        if (assigns_int(s.body, s.name)) throw NotEligible{};
        const IntVal before = ints[s.name];
        const uint8_t before_cond = int_cond_only[s.name];
        for (int64_t i = lo; i < hi; ++i) {
          ints[s.name] = IntVal{true, false, i, -1};
          int_cond_only[s.name] = 0;
          stmts(s.body);
        }
        if (lo >= hi) {
          ints[s.name] = before;   // the loop variable keeps its value
          int_cond_only[s.name] = before_cond;
        } else if (before.dev) {
          // the loop sits in a conditional region: its final value goes to
          // the register that both paths read afterwards
          iconst(before.reg, hi - 1);
          ints[s.name] = before;
          int_cond_only[s.name] = before_cond;
          mark_int_defined(s.name);
        } else {
          ints[s.name] = IntVal{true, false, hi - 1, -1};
        }
        return;
      }
    }
    throw NotEligible{};
  }
};

bool Executor::run_vm_program() {
  if (nw_ > (int64_t(1) << 24)) return false;
  VmCompiler c(*this);
  try {
    c.init();
    c.stmts(prog_.stmts);
  } catch (const NotEligible&) {
    return false;
  }
  // outputs: every output stream / array element that holds a value is
  // stored into a buffer of its own at the end
  struct Out { int name; int64_t idx; int32_t slot; BufRef buf; };
  std::vector<Out> outs;
  for (int id : prog_.outputs) {
    if (prog_.is_array[id]) {
      for (auto& kv : c.arrs[id].elems) outs.push_back({id, kv.first, kv.second, nullptr});
    } else if (c.slot_of[id] >= 0) {
      if (c.cond_only[id]) return false;
      outs.push_back({id, -1, c.slot_of[id], nullptr});
    }
  }
  for (int id : prog_.output_ints)
    if (c.ints[id].def && c.int_cond_only[id]) return false;
  for (auto& o : outs) {
    o.buf = dev_.alloc_stream(nw_);
    c.op(kVmStore, c.ext_of(o.buf->p), o.slot);
  }

  // device buffers: instructions | pointer table | state | slot file (if global)
  auto align = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t ops_b = c.code.size() * sizeof(VmOp);
  const size_t ext_b = std::max<size_t>(1, c.ext.size()) * sizeof(uint64_t*);
  const size_t state_b = vm_state_bytes(c.n_iregs, c.n_slots);
  const bool smem = vm_smem_bytes(c.n_slots, nw_) > 0;
  const size_t file_b = smem ? 0 : static_cast<size_t>(c.n_slots) * static_cast<size_t>(nw_) * 8;
  const size_t total = align(ops_b) + align(ext_b) + align(state_b) + file_b;
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
  uint8_t* d_state = reinterpret_cast<uint8_t*>(base + align(ops_b) + align(ext_b));
  uint64_t* d_file =
      smem ? nullptr : reinterpret_cast<uint64_t*>(base + align(ops_b) + align(ext_b) + align(state_b));
  dev_.h2d(d_ops, c.code.data(), ops_b);
  if (!c.ext.empty())
    BSZ_CUDA(cudaMemcpyAsync(d_ext, c.ext.data(), c.ext.size() * sizeof(uint64_t*), cudaMemcpyHostToDevice,
                             dev_.stream()));
  BSZ_CUDA(cudaMemsetAsync(d_state, 0, state_b, dev_.stream()));
  VmProgLaunch L{{d_ops, static_cast<int64_t>(c.code.size()), d_ext, d_file, c.n_slots, nw_, last_mask_, nullptr},
                 d_state, c.n_iregs};
  launch_vm_program(dev_, L);
  ++vm_launches;
  ++n_segments;
  std::vector<uint8_t> st(state_b);
  BSZ_CUDA(cudaMemcpyAsync(st.data(), d_state, state_b, cudaMemcpyDeviceToHost, dev_.stream()));
  dev_.sync();
  ++n_syncs;
  uint32_t err = 0;
  std::memcpy(&err, st.data(), 4);
  if (err == kVmErrBudget) return false;   // re-run by the host-driven walk
  if (err == kVmErrNegPop) throw RuntimeError("popcount on negative value (infinite bits set)");
  if (err == kVmErrWhile) throw RuntimeError("while loop exceeded 10000 iterations");
  if (err == kVmErrNegShift) throw RuntimeError("negative shift count");
  if (err) throw RuntimeError("device interpreter error " + std::to_string(err));
  static const char* const kNames[kClsCount] = {"", "~", "&", "|", "^", "+", "<<", ">>", "popcount"};
  for (int k = 1; k < kClsCount; ++k) {
    uint64_t n = 0;
    std::memcpy(&n, st.data() + 8 + 8 * k, 8);
    if (n) {
      op_count += static_cast<int64_t>(n);
      op_mix[kNames[k]] += static_cast<int64_t>(n);
    }
  }
  const uint8_t* tails = st.data() + 8 + 8 * kClsCount + 8 * static_cast<size_t>(c.n_iregs);
  auto ireg = [&](int32_t r) {
    int64_t v = 0;
    std::memcpy(&v, st.data() + 8 + 8 * kClsCount + 8 * static_cast<size_t>(r), 8);
    return v;
  };
  // results into the executor's state, as its own walk would leave them
  for (auto& o : outs) {
    const int node = buf_node(o.buf, tails[o.slot], false);
    if (o.idx < 0) {
      var_[o.name] = node;
    } else {
      if (!arrs_[o.name]) arrs_[o.name] = std::make_unique<Arr>();
      arrs_[o.name]->elems[o.idx] = node;
    }
  }
  for (int id : prog_.outputs) {
    if (!prog_.is_array[id]) continue;
    const auto& a = c.arrs[id];
    if (!arrs_[id]) arrs_[id] = std::make_unique<Arr>();
    Arr& t = *arrs_[id];
    t.defined = a.defined;
    t.broadcast = a.broadcast;
    t.bcast = a.bcast;
    t.decl_size = a.decl_size;
    for (auto it = t.elems.begin(); it != t.elems.end();) {
      if (!a.elems.count(it->first)) it = t.elems.erase(it);
      else ++it;
    }
  }
  for (int id : prog_.output_ints) {
    const auto& v = c.ints[id];
    if (!v.def) continue;
    ints_[id] = IntV{v.dev ? ireg(v.reg) : v.v, -1};
    int_def_[id] = 1;
  }
  max_live_buffers = std::max(max_live_buffers, static_cast<int64_t>(c.n_slots));
  return true;
}

}  // namespace bsz
