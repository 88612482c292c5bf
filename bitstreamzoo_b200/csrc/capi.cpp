// extern "C" boundary (include/bsz.h).  Exceptions never cross it: each
// entry point catches, stores the message for bsz_last_error() and returns a
// status.
#include "../../include/bsz.h"

#include <chrono>
#include <cstring>
#include <memory>
#include <string>

#include "device.h"
#include "engine.h"
#include "frontend.h"
#include "fused.h"
#include "io.h"
#include "mlp.h"

// Lifetimes: runs keep their program alive and programs keep their context
// alive, so the handles may be freed in any order.
struct bsz_ctx {
  std::unique_ptr<bsz::Device> dev;
  int refs = 1;
};

struct bsz_program {
  bsz_ctx* ctx;
  std::unique_ptr<bsz::Program> prog;
  int refs = 1;
};

static void ctx_unref(bsz_ctx* c) {
  if (c && --c->refs == 0) delete c;
}

static void prog_unref(bsz_program* p) {
  if (p && --p->refs == 0) {
    bsz_ctx* c = p->ctx;
    delete p;
    ctx_unref(c);
  }
}

struct bsz_run {
  bsz_program* prog;
  int64_t bitlength;
  int mode;
  std::unique_ptr<bsz::Executor> ex;
  std::vector<std::pair<int, int64_t>> params;
  bool launched = false;   // bsz_execute_async enqueued its work
  bool done = false;       // finished: results readable
  int64_t l0 = 0, l1 = 0;  // the device's launch count before and after this run's launches
  cudaEvent_t ev[2] = {nullptr, nullptr};   // device-time window of this run
  ~bsz_run() {
    ex.reset();
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    prog_unref(prog);
  }
};

namespace {

thread_local std::string g_err;
thread_local std::string g_json;

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
  } catch (...) {
    g_err = "unknown error";
  }
  return 1;
}

int64_t words_of(int64_t bitlength) { return bitlength > 0 ? (bitlength + 63) / 64 : 1; }

bsz::Executor& executor(bsz_run* r) {
  if (!r->ex) {
    bsz::ExecOptions o;
    o.mode = static_cast<bsz::ExecMode>(r->mode);
    r->ex = std::make_unique<bsz::Executor>(*r->prog->ctx->dev, *r->prog->prog, r->bitlength, o);
  }
  return *r->ex;
}

// Declared input name (or -1): inputs the program does not declare are
// ignored, as both reference executors load only declared inputs
// (interpreter.py:232-238, interpreter.inl:288-312).
int input_id(bsz_run* r, const char* name) {
  const bsz::Program& p = *r->prog->prog;
  int id = p.find(name ? name : "");
  if (id < 0) return -1;
  for (int x : p.inputs)
    if (x == id) return id;
  return -1;
}

// Page-locked (or managed) host memory copies at link speed directly;
// pageable memory goes through the device's pinned staging buffers.
bool is_pinned(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeManaged;
}

int name_id(bsz_run* r, const char* name) {
  int id = r->prog->prog->find(name ? name : "");
  if (id < 0) throw std::invalid_argument(std::string("unknown name: ") + (name ? name : "(null)"));
  return id;
}

}  // namespace

namespace bsz {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace bsz

extern "C" {

const char* bsz_version(void) { return "bitstreamzoo_b200 0.1 (sm_100a)"; }
const char* bsz_last_error(void) { return g_err.c_str(); }

bsz_ctx* bsz_create(int device) {
  bsz_ctx* c = nullptr;
  if (guard([&] {
        auto ctx = std::make_unique<bsz_ctx>();
        ctx->dev = std::make_unique<bsz::Device>(device);
        c = ctx.release();
      }))
    return nullptr;
  return c;
}

void bsz_destroy(bsz_ctx* ctx) { ctx_unref(ctx); }

void* bsz_stream(bsz_ctx* ctx) { return ctx ? static_cast<void*>(ctx->dev->stream()) : nullptr; }

int bsz_profile(bsz_ctx* ctx, int enable) {
  return guard([&] {
    ctx->dev->prof_reset();
    ctx->dev->profiling = enable != 0;
  });
}

const char* bsz_profile_report(bsz_ctx* ctx) {
  int rc = guard([&] { g_json = ctx->dev->prof_report(); });
  return rc ? nullptr : g_json.c_str();
}

int bsz_sync(bsz_ctx* ctx) {
  return guard([&] {
    ctx->dev->sync();
    if (uint32_t e = ctx->dev->take_error())
      throw bsz::RuntimeError(bsz::describe_device_error(e));
  });
}

bsz_program* bsz_compile(bsz_ctx* ctx, const char* source, size_t len) {
  bsz_program* p = nullptr;
  if (guard([&] {
        auto prog = std::make_unique<bsz_program>();
        prog->ctx = ctx;
        prog->prog = bsz::parse_program(std::string(source, len));
        if (ctx) ++ctx->refs;
        p = prog.release();
      }))
    return nullptr;
  return p;
}

void bsz_program_free(bsz_program* prog) { prog_unref(prog); }

int64_t bsz_static_ops(bsz_program* prog, const char* const* names, const int64_t* values, int n) {
  std::unordered_map<std::string, int64_t> params;
  for (int i = 0; i < n; ++i) params[names[i]] = values[i];
  return bsz::count_static_ops(*prog->prog, params);
}

bsz_run* bsz_run_create(bsz_program* prog, int64_t bitlength, int mode) {
  bsz_run* r = nullptr;
  if (guard([&] {
        auto run = std::make_unique<bsz_run>();
        run->prog = prog;
        run->bitlength = bitlength;
        if (mode < BSZ_MODE_PLAIN || mode > BSZ_MODE_VM) throw bsz::RuntimeError("bsz_run_create: bad mode");
        run->mode = mode;
        ++prog->refs;
        try {
          executor(run.get());
        } catch (...) {
          run->ex.reset();
          throw;
        }
        r = run.release();
      }))
    return nullptr;
  return r;
}

void bsz_run_free(bsz_run* run) { delete run; }

int bsz_set_param(bsz_run* run, const char* name, int64_t value) {
  return guard([&] {
    int id = run->prog->prog->find(name);
    if (id >= 0) executor(run).set_param(id, value);
  });
}

int bsz_run_set_schedule(bsz_run* run, const bsz_schedule* s) {
  return guard([&] {
    bsz::Schedule c;
    c.warps = s->warps;
    c.range_steps = s->range_steps;
    c.ctas_per_sm = s->ctas_per_sm;
    c.min_blocks = s->min_blocks;
    c.prefetch = s->prefetch;
    c.cut_adds = s->cut_adds;
    c.layout = s->layout;
    c.chunk_words = s->chunk_words;
    c.stages = s->stages;
    c.unroll = s->unroll;
    c.shift_mul = s->shift_mul;
    executor(run).set_schedule(c);
  });
}

int bsz_bind_input(bsz_run* run, const char* name, int64_t index, const uint64_t* words,
                   uint64_t n_words, int tail, int on_device) {
  return guard([&] {
    bsz::Device& dev = *run->prog->ctx->dev;
    const int id = input_id(run, name);
    if (id < 0) return;
    const int64_t nw = words_of(run->bitlength);
    if (on_device == 2) {   // borrowed device buffer: no copy, caller keeps it alive
      if (static_cast<int64_t>(n_words) < nw)
        throw std::invalid_argument("borrowed input shorter than ceil(bitlength/64) words");
      auto b = std::make_shared<bsz::DevStream>();
      b->p = const_cast<uint64_t*>(words);
      b->n_words = nw;
      if (index < 0) executor(run).bind_input(id, b, tail ? 1 : 0, false);
      else executor(run).bind_input_array(id, index, b, tail ? 1 : 0, false);
      return;
    }
    bsz::BufRef b = dev.alloc_stream(nw);
    const int64_t have = std::min<int64_t>(static_cast<int64_t>(n_words), nw);
    if (have > 0) {
      if (on_device || is_pinned(words))
        BSZ_CUDA(cudaMemcpyAsync(b->p, words, have * 8,
                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 dev.stream()));
      else
        dev.h2d(b->p, words, static_cast<size_t>(have) * 8);   // pageable: staged
    }
    if (have < nw) {
      uint64_t fill = tail ? ~uint64_t(0) : 0;
      bsz::launch_fill(dev, b->p + have, nw - have, fill, fill);
    }
    // Host inputs: check the bits at and above the bitlength.  Device inputs
    // are treated as possibly dirty there (the executor then keeps them).
    bool clean = false;
    if (!on_device && !tail && run->bitlength > 0) {
      clean = true;
      const int64_t lw = words_of(run->bitlength);
      if (have >= lw && (words[lw - 1] & ~bsz::mask_for_bits(run->bitlength))) clean = false;
    }
    if (index < 0) executor(run).bind_input(id, b, tail ? 1 : 0, clean);
    else executor(run).bind_input_array(id, index, b, tail ? 1 : 0, clean);
  });
}

int bsz_bind_broadcast(bsz_run* run, const char* name, const uint8_t* ones, int64_t count) {
  return guard([&] {
    const int id = input_id(run, name);
    if (id < 0) return;
    std::vector<uint8_t> v(ones, ones + count);
    for (auto& x : v) x = x ? 1 : 0;
    executor(run).bind_broadcast(id, v);
  });
}

static void launch_run(bsz_run* run) {
  if (run->done || run->launched) throw bsz::RuntimeError("bsz_execute: run already executed");
  bsz::Device& dev = *run->prog->ctx->dev;
  bsz::Executor& ex = executor(run);
  for (cudaEvent_t& e : run->ev)
    if (!e) BSZ_CUDA(cudaEventCreate(&e));
  run->l0 = dev.n_launches;
  BSZ_CUDA(cudaEventRecord(run->ev[0], dev.stream()));
  ex.run(false);
  BSZ_CUDA(cudaEventRecord(run->ev[1], dev.stream()));
  run->l1 = dev.n_launches;   // other runs may launch before this one is waited on
  run->launched = true;
}

static void finish_run(bsz_run* run, bsz_stats* stats) {
  if (!run->launched) throw bsz::RuntimeError("bsz_run_wait: run not launched");
  bsz::Device& dev = *run->prog->ctx->dev;
  bsz::Executor& ex = executor(run);
  if (!run->done) {
    const int64_t f0 = dev.n_launches;
    ex.finish();   // may re-run unproven fused parts
    run->l1 += dev.n_launches - f0;
    BSZ_CUDA(cudaEventSynchronize(run->ev[1]));
    run->done = true;
  }
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, run->ev[0], run->ev[1]);
    stats->op_count = ex.op_count;
    stats->n_kernel_launches = run->l1 - run->l0;
    stats->n_mallocs = dev.n_mallocs;
    stats->n_segments = ex.n_segments;
    stats->n_syncs = ex.n_syncs;
    stats->peak_bytes = dev.bytes_peak;
    stats->max_live = ex.max_live_buffers;
    stats->kernel_ms = ms;
    stats->compile_ms = ex.compile_ms;
    stats->n_fused_launches = ex.fused_launches();
    stats->n_fused_fallbacks = ex.fused_fallbacks();
    stats->n_vm_launches = ex.vm_launches;
    stats->walk_replayed = ex.walk_replayed ? 1 : 0;
  }
}

// Results of a launched run are readable once it has finished.
static void ensure_finished(bsz_run* run) {
  if (run->launched && !run->done) finish_run(run, nullptr);
}

int bsz_execute(bsz_run* run, bsz_stats* stats) {
  return guard([&] {
    launch_run(run);
    finish_run(run, stats);
  });
}

int bsz_execute_async(bsz_run* run) {
  return guard([&] { launch_run(run); });
}

int bsz_run_wait(bsz_run* run, bsz_stats* stats) {
  return guard([&] { finish_run(run, stats); });
}

static bsz::BufRef find_stream(bsz_run* run, const char* name, int64_t index) {
  ensure_finished(run);
  bsz::Executor& ex = executor(run);
  int id = name_id(run, name);
  bsz::BufRef b = index < 0 ? ex.stream_value(id) : ex.array_value(id, index);
  if (!b || (index >= 0 && !ex.has_array(id)) || (index < 0 && !ex.has_stream(id)))
    throw std::invalid_argument(std::string("no such output: ") + name);
  return b;
}

int bsz_get_stream(bsz_run* run, const char* name, int64_t index, uint64_t* host, uint64_t n_words) {
  return guard([&] {
    bsz::Device& dev = *run->prog->ctx->dev;
    bsz::BufRef b = find_stream(run, name, index);
    const int64_t nw = words_of(run->bitlength);
    const int64_t n = std::min<int64_t>(nw, static_cast<int64_t>(n_words));
    if (is_pinned(host)) {
      BSZ_CUDA(cudaMemcpyAsync(host, b->p, n * 8, cudaMemcpyDeviceToHost, dev.stream()));
      dev.sync();
    } else {
      dev.d2h(host, b->p, static_cast<size_t>(n) * 8);   // pageable: staged
    }
    if (n == nw && run->bitlength > 0) host[nw - 1] &= bsz::mask_for_bits(run->bitlength);
  });
}

int bsz_get_stream_device(bsz_run* run, const char* name, int64_t index, const uint64_t** dptr) {
  return guard([&] { *dptr = find_stream(run, name, index)->p; });
}

int bsz_get_int(bsz_run* run, const char* name, int64_t* value) {
  return guard([&] {
    ensure_finished(run);
    if (!executor(run).int_value(name_id(run, name), value))
      throw std::invalid_argument(std::string("no such int: ") + name);
  });
}

int64_t bsz_array_indices(bsz_run* run, const char* name, int64_t* indices, int64_t cap) {
  int64_t count = -1;
  guard([&] {
    ensure_finished(run);
    int id = name_id(run, name);
    if (!executor(run).has_array(id)) return;
    auto idx = executor(run).array_indices(id);
    count = static_cast<int64_t>(idx.size());
    for (int64_t i = 0; i < count && i < cap; ++i) indices[i] = idx[i];
  });
  return count;
}

int bsz_program_features(bsz_ctx* ctx, bsz_program* prog, float* out, int capacity) {
  int count = -1;
  guard([&] {
    bsz::ExecOptions eo;
    eo.mode = bsz::ExecMode::Fused;
    bsz::Executor ex(*ctx->dev, *prog->prog, int64_t(1) << 20, eo);
    bsz::Executor::Traced t = ex.trace();
    const auto& nd = t.nodes;
    std::vector<uint8_t> live(nd.size(), 0);
    std::vector<int> stack;
    for (int n : t.output_nodes)
      if (n >= 0) stack.push_back(n);
    for (auto& p : t.pops) stack.push_back(p.first);
    while (!stack.empty()) {
      int n = stack.back();
      stack.pop_back();
      if (live[n]) continue;
      live[n] = 1;
      for (int o : {nd[n].a, nd[n].b})
        if (o >= 0) stack.push_back(o);
    }
    auto is_leaf = [&](int n) {
      auto op = nd[n].op;
      return op == bsz::NOp::Buf || op == bsz::NOp::Zero || op == bsz::NOp::OnesMask ||
             op == bsz::NOp::AllOnes;
    };
    double n_ops = 0, n_bit = 0, n_not = 0, n_shl_t = 0, n_shl_i = 0, n_add = 0, n_shr = 0, n_in = 0;
    double max_ws = 0;
    std::vector<int> depth(nd.size(), 0), adepth(nd.size(), 0);
    int max_depth = 0, max_adepth = 0;
    for (size_t i = 0; i < nd.size(); ++i) {
      if (!live[i]) continue;
      const bsz::Node& x = nd[i];
      if (is_leaf(static_cast<int>(i))) {
        if (x.op == bsz::NOp::Buf) ++n_in;
        continue;
      }
      ++n_ops;
      int d = 0, ad = 0;
      for (int o : {x.a, x.b})
        if (o >= 0) {
          d = std::max(d, depth[o]);
          ad = std::max(ad, adepth[o]);
        }
      depth[i] = d + 1;
      adepth[i] = ad + (x.op == bsz::NOp::Add ? 1 : 0);
      max_depth = std::max(max_depth, depth[i]);
      max_adepth = std::max(max_adepth, adepth[i]);
      switch (x.op) {
        case bsz::NOp::And: case bsz::NOp::Or: case bsz::NOp::Xor: ++n_bit; break;
        case bsz::NOp::Not: case bsz::NOp::AndNot: ++n_not; break;
        case bsz::NOp::Add: ++n_add; break;
        case bsz::NOp::Shr: ++n_shr; max_ws = std::max<double>(max_ws, x.k / 64.0); break;
        case bsz::NOp::Shl:
          if (is_leaf(x.a)) ++n_shl_i;
          else ++n_shl_t;
          max_ws = std::max<double>(max_ws, x.k / 64.0);
          break;
        default: break;
      }
    }
    // peak number of simultaneously live computed values in node order (a
    // proxy for the generated kernel's register demand per step)
    std::vector<int64_t> last_use(nd.size(), -1);
    for (size_t i = 0; i < nd.size(); ++i) {
      if (!live[i]) continue;
      for (int o : {nd[i].a, nd[i].b})
        if (o >= 0) last_use[o] = static_cast<int64_t>(i);
    }
    for (int n : t.output_nodes)
      if (n >= 0) last_use[n] = static_cast<int64_t>(nd.size());
    for (auto& p : t.pops) last_use[p.first] = std::max<int64_t>(last_use[p.first], static_cast<int64_t>(nd.size()));
    std::vector<int> ends(nd.size() + 1, 0);
    int64_t cur = 0, peak = 0;
    for (size_t i = 0; i < nd.size(); ++i) {
      if (live[i] && !is_leaf(static_cast<int>(i)) && last_use[i] >= 0) {
        ++cur;
        peak = std::max(peak, cur);
        ++ends[std::min<size_t>(static_cast<size_t>(last_use[i]), nd.size())];
      }
      cur -= ends[i];
      ends[i] = 0;
    }
    const double tot = std::max(1.0, n_ops);
    const float f[BSZ_NUM_FEATURES] = {
        static_cast<float>(std::log2(1 + n_ops)), static_cast<float>(n_bit / tot),
        static_cast<float>(n_not / tot), static_cast<float>(n_shl_t / tot),
        static_cast<float>(n_shl_i / tot), static_cast<float>(n_add / tot),
        static_cast<float>(n_shr / tot), static_cast<float>(std::log2(1.0 + max_depth)),
        static_cast<float>(std::log2(1.0 + max_adepth)), static_cast<float>(std::log2(1 + max_ws)),
        static_cast<float>(std::log2(1 + n_in)),
        static_cast<float>(std::log2(1.0 + t.output_nodes.size() + t.pops.size())),
        static_cast<float>(std::log2(1 + n_shl_t)), static_cast<float>(std::log2(1 + n_add)),
        static_cast<float>(std::log2(1.0 + static_cast<double>(peak)))};
    for (int i = 0; i < BSZ_NUM_FEATURES && i < capacity; ++i) out[i] = f[i];
    count = BSZ_NUM_FEATURES;
  });
  return count;
}

struct bsz_mlp {
  bsz_ctx* ctx;
  std::unique_ptr<bsz::Mlp> net;
};

bsz_mlp* bsz_mlp_create(bsz_ctx* ctx, int in_dim, int hidden, int layers, uint64_t seed) {
  bsz_mlp* out = nullptr;
  if (guard([&] {
        auto m = std::make_unique<bsz_mlp>();
        m->ctx = ctx;
        m->net = std::make_unique<bsz::Mlp>(in_dim, hidden, layers, seed, ctx->dev->stream());
        ++ctx->refs;
        out = m.release();
      }))
    return nullptr;
  return out;
}

int64_t bsz_mlp_num_params(bsz_mlp* m) { return m->net->n_params(); }

int bsz_mlp_train_step(bsz_mlp* m, const float* x, const float* y, int n, float lr, float* loss) {
  return guard([&] {
    float l = m->net->train_step(x, y, n, lr);
    if (loss) *loss = l;
  });
}

int bsz_mlp_predict(bsz_mlp* m, const float* x, int n, float* out) {
  return guard([&] { m->net->predict(x, n, out); });
}

int bsz_mlp_gradients(bsz_mlp* m, const float* x, const float* y, int n, float* grad, float* loss) {
  return guard([&] {
    float l = m->net->gradients(x, y, n, grad);
    if (loss) *loss = l;
  });
}

int bsz_mlp_params(bsz_mlp* m, float* params, int get) {
  return guard([&] {
    if (get) m->net->get_params(params);
    else m->net->set_params(params);
  });
}

int bsz_mlp_set_weight_decay(bsz_mlp* m, float weight_decay) {
  return guard([&] {
    if (!(weight_decay >= 0.f)) throw bsz::RuntimeError("bsz_mlp_set_weight_decay: negative or NaN");
    m->net->set_weight_decay(weight_decay);
  });
}

void bsz_mlp_free(bsz_mlp* m) {
  if (!m) return;
  bsz_ctx* c = m->ctx;
  m->net.reset();
  delete m;
  ctx_unref(c);
}

struct bsz_batch {
  bsz_ctx* ctx;
  std::vector<bsz_program*> progs;
  std::unique_ptr<bsz::BatchRunner> runner;
  int64_t launches0 = 0;
};

bsz_batch* bsz_batch_create(bsz_ctx* ctx, bsz_program* const* programs, int n_programs,
                            const bsz_instance* instances, int64_t n_instances,
                            const bsz_schedule* schedule) {
  bsz_batch* out = nullptr;
  if (guard([&] {
        auto b = std::make_unique<bsz_batch>();
        b->ctx = ctx;
        std::vector<const bsz::Program*> progs;
        for (int i = 0; i < n_programs; ++i) {
          b->progs.push_back(programs[i]);
          progs.push_back(programs[i]->prog.get());
        }
        std::vector<bsz::BatchInstance> inst(static_cast<size_t>(n_instances));
        for (int64_t i = 0; i < n_instances; ++i) {
          const bsz_instance& x = instances[i];
          if (x.program < 0 || x.program >= n_programs)
            throw std::invalid_argument("bsz_batch_create: program index out of range");
          const bsz::Program& p = *progs[x.program];
          inst[i].program = x.program;
          inst[i].bitlength = x.bitlength;
          inst[i].inputs.assign(x.inputs, x.inputs + p.inputs.size());
          inst[i].outputs.assign(x.outputs, x.outputs + p.outputs.size());
        }
        bsz::Schedule s;
        if (schedule) {
          s.warps = std::max(1, std::min(schedule->warps, 16));
          s.range_steps = std::max(1, schedule->range_steps);
          s.ctas_per_sm = std::max(0, schedule->ctas_per_sm);
          s.min_blocks = std::max(1, schedule->min_blocks);
          s.prefetch = schedule->prefetch;
          s.cut_adds = 0;
          s.layout = std::max(0, std::min(schedule->layout, 2));
          s.chunk_words = schedule->chunk_words == 8 ? 8 : 4;
          s.stages = schedule->stages == 3 ? 3 : 2;
          s.shift_mul = schedule->shift_mul ? 1 : 0;
        }
        b->runner = std::make_unique<bsz::BatchRunner>(*ctx->dev, progs, std::move(inst), s);
        for (auto* p : b->progs) ++p->refs;
        out = b.release();
      }))
    return nullptr;
  return out;
}

int bsz_batch_launch(bsz_batch* b) {
  return guard([&] {
    b->launches0 = b->ctx->dev->n_launches;
    b->runner->launch();
  });
}

int bsz_batch_finish(bsz_batch* b, bsz_stats* stats) {
  return guard([&] {
    b->runner->finish();
    if (uint32_t e = b->ctx->dev->take_error())
      throw bsz::RuntimeError(bsz::describe_device_error(e));
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->n_kernel_launches = b->ctx->dev->n_launches - b->launches0;
      stats->n_mallocs = b->ctx->dev->n_mallocs;
      stats->n_fused_launches = b->runner->launches;
      stats->n_fused_fallbacks = b->runner->fallbacks;
      stats->compile_ms = b->runner->compile_ms;
      stats->n_segments = 1;
    }
  });
}

int bsz_batch_ints(bsz_batch* b, int64_t instance, int64_t* values, int capacity) {
  int n = -1;
  guard([&] {
    const auto& v = b->runner->ints(instance);
    n = static_cast<int>(v.size());
    for (int i = 0; i < n && i < capacity; ++i) values[i] = v[i];
  });
  return n;
}

int64_t bsz_batch_items(bsz_batch* b) { return b->runner->n_items(); }

void bsz_batch_free(bsz_batch* b) {
  if (!b) return;
  b->runner.reset();
  for (auto* p : b->progs) prog_unref(p);
  delete b;
}

const char* bsz_run_case_json(bsz_ctx* ctx, const char* source, const char* bsdata_path,
                              const char* json_input, int flags) {
  g_json.clear();
  int rc = guard([&] {
    auto t0 = std::chrono::high_resolution_clock::now();
    auto prog = bsz::parse_program(source);
    double parse_ms =
        std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
    std::vector<bsz::CaseInput> cases;
    if (bsdata_path) cases = bsz::read_bsdata(bsdata_path);
    else cases.push_back(bsz::parse_json_case(json_input ? json_input : "{}"));
    bsz::DriverOptions o;
    o.warmup = flags & 1;
    o.mode = (flags >> 1) & 3;
    if (cases.size() == 1) {
      g_json = bsz::run_case_json(*ctx->dev, *prog, cases[0], o, parse_ms);
    } else {
      g_json = "[";
      for (size_t i = 0; i < cases.size(); ++i) {
        std::string one = bsz::run_case_json(*ctx->dev, *prog, cases[i], o, parse_ms);
        one.pop_back();
        one += ",\"name\":" + bsz::json_quote(cases[i].name) + "}";
        if (i) g_json += ",";
        g_json += one;
      }
      g_json += "]";
    }
  });
  return rc ? nullptr : g_json.c_str();
}

// ---- per-op data plane --------------------------------------------------
namespace {
// The logical length of an op on n words: 0 means the full storage width
// (64 n bits, the C++ binaries' convention); otherwise 1 .. 64 n.
uint64_t checked_mask(const char* op, int64_t bitlength, uint64_t n) {
  if (bitlength < 0 || (bitlength > 0 && static_cast<uint64_t>(bitlength) > 64 * n))
    throw std::invalid_argument(std::string(op) + ": bitlength " + std::to_string(bitlength) +
                                " outside [0, 64 * n_words] for n_words = " + std::to_string(n));
  return bsz::mask_for_bits(bitlength);
}
}  // namespace

int bsz_op_not(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, uint64_t n, int64_t bitlength) {
  return guard([&] { bsz::launch_not(*ctx->dev, dst, a, n, checked_mask("bsz_op_not", bitlength, n)); });
}
int bsz_op_and(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b, uint64_t n) {
  return guard([&] { bsz::launch_bitwise(*ctx->dev, bsz::kAnd, dst, a, b, n); });
}
int bsz_op_or(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b, uint64_t n) {
  return guard([&] { bsz::launch_bitwise(*ctx->dev, bsz::kOr, dst, a, b, n); });
}
int bsz_op_xor(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b, uint64_t n) {
  return guard([&] { bsz::launch_bitwise(*ctx->dev, bsz::kXor, dst, a, b, n); });
}
int bsz_op_andnot(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b, uint64_t n) {
  return guard([&] { bsz::launch_bitwise(*ctx->dev, bsz::kAndNot, dst, a, b, n); });
}
int bsz_op_add(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, const uint64_t* b, uint64_t n,
               int64_t bitlength) {
  return guard([&] {
    bsz::launch_add(*ctx->dev, dst, a, b, n, checked_mask("bsz_op_add", bitlength, n));
  });
}
int bsz_op_shl(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, uint64_t k, uint64_t n,
               int64_t bitlength) {
  return guard([&] {
    bsz::launch_shl(*ctx->dev, dst, a, static_cast<int64_t>(std::min<uint64_t>(k, uint64_t(1) << 62)), n,
                    checked_mask("bsz_op_shl", bitlength, n));
  });
}
int bsz_op_shr(bsz_ctx* ctx, uint64_t* dst, const uint64_t* a, uint64_t k, uint64_t n, int tail) {
  return guard([&] {
    bsz::launch_shr(*ctx->dev, dst, a, static_cast<int64_t>(std::min<uint64_t>(k, uint64_t(1) << 62)), n,
                    tail ? ~uint64_t(0) : 0);
  });
}
int bsz_op_popcount(bsz_ctx* ctx, const uint64_t* a, uint64_t n, uint64_t* result) {
  return guard([&] {
    bsz::Device& dev = *ctx->dev;
    auto* slot = static_cast<unsigned long long*>(dev.scratch(256));
    BSZ_CUDA(cudaMemsetAsync(slot, 0, 8, dev.stream()));
    bsz::launch_popcount(dev, a, n, slot);
    BSZ_CUDA(cudaMemcpyAsync(result, slot, 8, cudaMemcpyDeviceToHost, dev.stream()));
    dev.sync();
  });
}
int bsz_s2p(bsz_ctx* ctx, const uint8_t* bytes, int64_t n_bytes, uint64_t* const* basis) {
  return guard([&] {
    if (n_bytes < 0) throw bsz::RuntimeError("bsz_s2p: negative byte count");
    if (n_bytes > 0 && (!bytes || !basis)) throw bsz::RuntimeError("bsz_s2p: null pointer");
    bsz::launch_s2p(*ctx->dev, bytes, n_bytes, basis);
  });
}

void bsz_debug_add_lookback_hook(int64_t silent_tile, int spin_limit) {
  bsz::set_add_lookback_test_hook(silent_tile, spin_limit);
}

int bsz_op_is_nonzero(bsz_ctx* ctx, const uint64_t* a, uint64_t n, int* result) {
  return guard([&] {
    bsz::Device& dev = *ctx->dev;
    auto* flag = static_cast<unsigned int*>(dev.scratch(256));
    BSZ_CUDA(cudaMemsetAsync(flag, 0, 4, dev.stream()));
    bsz::launch_any(dev, a, n, flag);
    unsigned int h = 0;
    BSZ_CUDA(cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, dev.stream()));
    dev.sync();
    *result = h != 0;
  });
}

}  // extern "C"
