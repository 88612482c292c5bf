// Host I/O implementation (see io.h).
#include "io.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <cerrno>
#include <chrono>
#include <unordered_map>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <thread>

#include "device.h"
#include "engine.h"
#include "frontend.h"

namespace bsz {

// ------------------------------------------------------------------ JSON ---
namespace {

struct JParser {
  const char* p;
  const char* e;
  [[noreturn]] void fail(const char* what) {
    throw std::runtime_error(std::string("JSON parse error: ") + what);
  }
  void ws() {
    while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  JVal value() {
    ws();
    if (p >= e) fail("unexpected end");
    JVal v;
    char c = *p;
    if (c == '{') {
      v.type = JVal::Obj;
      ++p;
      ws();
      if (p < e && *p == '}') { ++p; return v; }
      while (true) {
        ws();
        if (p >= e || *p != '"') fail("expected key");
        std::string k = str();
        ws();
        if (p >= e || *p != ':') fail("expected ':'");
        ++p;
        v.o.emplace_back(std::move(k), value());
        ws();
        if (p < e && *p == ',') { ++p; continue; }
        if (p < e && *p == '}') { ++p; break; }
        fail("expected ',' or '}'");
      }
      return v;
    }
    if (c == '[') {
      v.type = JVal::Arr;
      ++p;
      ws();
      if (p < e && *p == ']') { ++p; return v; }
      while (true) {
        v.a.push_back(value());
        ws();
        if (p < e && *p == ',') { ++p; continue; }
        if (p < e && *p == ']') { ++p; break; }
        fail("expected ',' or ']'");
      }
      return v;
    }
    if (c == '"') {
      v.type = JVal::Str;
      v.s = str();
      return v;
    }
    if (e - p >= 4 && !std::strncmp(p, "true", 4)) { p += 4; v.type = JVal::Bool; v.b = true; return v; }
    if (e - p >= 5 && !std::strncmp(p, "false", 5)) { p += 5; v.type = JVal::Bool; return v; }
    if (e - p >= 4 && !std::strncmp(p, "null", 4)) { p += 4; return v; }
    const char* s = p;
    bool real = false;
    if (p < e && (*p == '-' || *p == '+')) ++p;
    while (p < e && ((*p >= '0' && *p <= '9') || *p == '.' || *p == 'e' || *p == 'E' ||
                     *p == '-' || *p == '+')) {
      if (*p == '.' || *p == 'e' || *p == 'E') real = true;
      ++p;
    }
    if (p == s) fail("unexpected character");
    std::string num(s, p);
    if (!real) {
      errno = 0;
      char* end = nullptr;
      long long x = std::strtoll(num.c_str(), &end, 10);
      if (errno == 0) { v.type = JVal::Int; v.i = x; return v; }
    }
    v.type = JVal::Real;
    v.d = std::strtod(num.c_str(), nullptr);
    return v;
  }
  std::string str() {
    ++p;   // opening quote
    std::string out;
    while (p < e && *p != '"') {
      if (*p == '\\') {
        ++p;
        if (p >= e) fail("bad escape");
        char c = *p++;
        switch (c) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (e - p < 4) fail("bad \\u escape");
            unsigned cp = std::stoul(std::string(p, p + 4), nullptr, 16);
            p += 4;
            if (cp < 0x80) out += static_cast<char>(cp);
            else if (cp < 0x800) { out += static_cast<char>(0xC0 | (cp >> 6)); out += static_cast<char>(0x80 | (cp & 0x3F)); }
            else { out += static_cast<char>(0xE0 | (cp >> 12)); out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F)); out += static_cast<char>(0x80 | (cp & 0x3F)); }
            break;
          }
          default: out += c;
        }
      } else {
        out += *p++;
      }
    }
    if (p >= e) fail("unterminated string");
    ++p;
    return out;
  }
};

}  // namespace

JVal json_parse(const char* p, size_t n) {
  JParser jp{p, p + n};
  JVal v = jp.value();
  return v;
}

std::string json_quote(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    switch (c) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\n': o += "\\n"; break;
      case '\t': o += "\\t"; break;
      case '\r': o += "\\r"; break;
      default:
        if (static_cast<unsigned char>(c) < 0x20) {
          char buf[8];
          std::snprintf(buf, sizeof buf, "\\u%04x", c);
          o += buf;
        } else {
          o += c;
        }
    }
  }
  return o + "\"";
}

// ------------------------------------------------------------------- hex ---

void hex_to_words(const std::string& hex, std::vector<uint64_t>& w, uint8_t& tail) {
  size_t i = 0;
  bool neg = false;
  if (i < hex.size() && hex[i] == '-') { neg = true; ++i; }
  if (i + 1 < hex.size() && hex[i] == '0' && (hex[i + 1] == 'x' || hex[i + 1] == 'X')) i += 2;
  if (i < hex.size() && hex[i] == '-') { neg = !neg; ++i; }
  std::fill(w.begin(), w.end(), 0);
  size_t end = hex.size();
  size_t nib = 0;
  for (size_t j = end; j > i; --j) {
    char c = hex[j - 1];
    uint64_t v;
    if (c >= '0' && c <= '9') v = c - '0';
    else if (c >= 'a' && c <= 'f') v = c - 'a' + 10;
    else if (c >= 'A' && c <= 'F') v = c - 'A' + 10;
    else continue;
    size_t wi = nib / 16;
    if (wi < w.size()) w[wi] |= v << (4 * (nib % 16));
    ++nib;
  }
  tail = 0;
  if (neg) {
    uint64_t carry = 1;
    for (auto& x : w) {
      uint64_t y = ~x + carry;
      carry = (carry && y == 0) ? 1 : 0;
      x = y;
    }
    // -(m) with m != 0 has all higher bits set; -0 == 0
    bool zero = true;
    for (size_t j = i; j < hex.size(); ++j)
      if (hex[j] != '0') { zero = false; break; }
    tail = zero ? 0 : 1;
  }
}

uint64_t StreamVal::word(size_t i) const {
  if (!view) return i < words.size() ? words[i] : 0;
  if (i * 8 >= view_bytes) return 0;
  uint64_t x = 0;
  std::memcpy(&x, view + i * 8, std::min<size_t>(8, view_bytes - i * 8));
  return x;
}

void StreamVal::materialize() {
  if (!view) return;
  words.assign(view_words, 0);
  std::memcpy(words.data(), view, view_bytes);
  view = nullptr;
  view_bytes = view_words = 0;
  hold.reset();
}

void words_to_hex(const uint64_t* w, size_t n, std::string& out) {
  static const char* digits = "0123456789abcdef";
  size_t top = n;
  while (top > 0 && w[top - 1] == 0) --top;
  if (top == 0) { out += "0x0"; return; }
  out += "0x";
  size_t start = out.size();
  uint64_t t = w[top - 1];
  int nd = 0;
  for (uint64_t x = t; x; x >>= 4) ++nd;
  out.resize(start + nd + 16 * (top - 1));
  char* o = &out[start];
  for (int k = nd - 1; k >= 0; --k) *o++ = digits[(t >> (4 * k)) & 15];
  // full words: 16 digits each, most significant word first, two digits per
  // byte from a 256-entry table; long outputs are split across threads
  static const std::array<uint16_t, 256> pairs = [] {
    std::array<uint16_t, 256> p{};
    for (int b = 0; b < 256; ++b)
      p[b] = static_cast<uint16_t>(static_cast<uint8_t>(digits[b >> 4]) |
                                   (static_cast<uint16_t>(static_cast<uint8_t>(digits[b & 15])) << 8));
    return p;
  }();
  const size_t full = top - 1;
  auto encode = [&](size_t lo, size_t hi) {   // output words [lo, hi) in print order
    for (size_t j = lo; j < hi; ++j) {
      const uint64_t x = w[full - 1 - j];
      char* d = o + 16 * j;
      for (int b = 7; b >= 0; --b) {
        const uint16_t pr = pairs[(x >> (8 * b)) & 0xff];
        std::memcpy(d + 2 * (7 - b), &pr, 2);
      }
    }
  };
  const size_t kPerThread = size_t(1) << 18;   // 2 MiB of words
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>({static_cast<size_t>(hw), size_t(16), full / kPerThread});
  if (nt <= 1) {
    encode(0, full);
    return;
  }
  std::vector<std::thread> th;
  const size_t per = (full + nt - 1) / nt;
  for (size_t t0 = 0; t0 < full; t0 += per) th.emplace_back(encode, t0, std::min(full, t0 + per));
  for (auto& t2 : th) t2.join();
}

// ---------------------------------------------------------------- bsdata ---
namespace {

size_t words_for(int64_t bitlength) {
  return bitlength > 0 ? static_cast<size_t>((bitlength + 63) / 64) : 1;
}

// The mapping every view of the file being decoded points into.
thread_local std::shared_ptr<const void> t_hold;

StreamVal from_bytes(const uint8_t* bin, size_t bin_len, size_t off, size_t nbytes, size_t nw) {
  StreamVal v;
  if (off + nbytes > bin_len) {   // out-of-range reference: zero (bsdata_reader.h:87-89)
    v.words.assign(nw, 0);
    return v;
  }
  v.view = bin + off;
  v.view_bytes = std::min(nbytes, nw * 8);
  v.view_words = nw;
  v.hold = t_hold;
  return v;
}

StreamVal from_json(const JVal& j, size_t nw) {
  StreamVal v;
  v.words.assign(nw, 0);
  if (j.type == JVal::Str) {
    hex_to_words(j.s, v.words, v.tail);
  } else if (j.type == JVal::Int) {
    if (j.i >= 0) {
      v.words[0] = static_cast<uint64_t>(j.i);
    } else {
      for (auto& x : v.words) x = ~uint64_t(0);
      v.words[0] = static_cast<uint64_t>(j.i);
      v.tail = 1;
    }
  } else if (j.type == JVal::Bool) {
    v.words[0] = j.b ? 1 : 0;
  }
  return v;
}

int64_t as_int(const JVal& j) {
  if (j.type == JVal::Int) return j.i;
  if (j.type == JVal::Real) return static_cast<int64_t>(j.d);
  if (j.type == JVal::Bool) return j.b;
  if (j.type == JVal::Str) return std::stoll(j.s, nullptr, 0);
  return 0;
}

void decode_section(const JVal& sec, const uint8_t* bin, size_t bin_len, size_t nw, CaseInput& c) {
  for (auto& kv : sec.o) {
    const std::string& k = kv.first;
    const JVal& v = kv.second;
    if (v.type == JVal::Obj) {
      if (const JVal* r = v.get("_bin")) {
        c.inputs[k] = from_bytes(bin, bin_len, as_int(r->a.at(0)), as_int(r->a.at(1)), nw);
      } else if (const JVal* r = v.get("_array_bin")) {
        int64_t count = as_int(r->a.at(0)), off = as_int(r->a.at(1)), stride = as_int(r->a.at(2));
        auto& arr = c.arrays[k];
        for (int64_t i = 0; i < count; ++i)
          arr[i] = from_bytes(bin, bin_len, off + i * stride, stride, nw);
      } else if (const JVal* r = v.get("_broadcast_pack")) {
        int64_t count = as_int(r->a.at(0)), off = as_int(r->a.at(1));
        std::vector<uint8_t> ones(count, 0);
        for (int64_t i = 0; i < count; ++i) {
          size_t byte = off + (i >> 3);
          ones[i] = byte < bin_len ? ((bin[byte] >> (i & 7)) & 1) : 0;
        }
        c.broadcast[k] = std::move(ones);
      } else {
        auto& arr = c.arrays[k];   // dict-style array {index: value}
        for (auto& e : v.o) {
          const JVal& x = e.second;
          if (x.type == JVal::Obj && x.get("_bin")) {
            const JVal* r = x.get("_bin");
            arr[std::stoll(e.first)] = from_bytes(bin, bin_len, as_int(r->a.at(0)), as_int(r->a.at(1)), nw);
          } else {
            arr[std::stoll(e.first)] = from_json(x, nw);
          }
        }
      }
    } else if (v.type == JVal::Arr) {
      auto& arr = c.arrays[k];
      for (size_t i = 0; i < v.a.size(); ++i) arr[static_cast<int64_t>(i)] = from_json(v.a[i], nw);
    } else {
      c.inputs[k] = from_json(v, nw);
    }
  }
}

CaseInput parse_case(const JVal& h, const uint8_t* bin, size_t bin_len) {
  CaseInput c;
  const JVal* bl = h.get("bitlength");
  if (!bl) bl = h.get("n_vectors");
  c.bitlength = bl ? as_int(*bl) : 0;
  size_t nw = words_for(c.bitlength);
  if (const JVal* p = h.get("params"))
    for (auto& kv : p->o) c.params.push_back({kv.first, as_int(kv.second)});
  if (const JVal* s = h.get("inputs")) decode_section(*s, bin, bin_len, nw, c);
  if (const JVal* s = h.get("input_arrays")) {
    CaseInput tmp;
    decode_section(*s, bin, bin_len, nw, tmp);
    for (auto& kv : tmp.arrays) c.arrays[kv.first] = std::move(kv.second);
    for (auto& kv : tmp.broadcast) c.broadcast[kv.first] = std::move(kv.second);
    for (auto& kv : tmp.inputs) c.inputs[kv.first] = std::move(kv.second);
  }
  if (const JVal* it = h.get("iterations")) c.iterations = static_cast<int>(as_int(*it));
  if (const JVal* fb = h.get("feedback"))
    for (auto& kv : fb->o) c.feedback.push_back({kv.first, kv.second.s});
  return c;
}

}  // namespace

namespace {

// A read-only private mapping of a whole file (unmapped when the last view
// into it goes away).
struct Mapping {
  void* p = MAP_FAILED;
  size_t n = 0;
  ~Mapping() {
    if (p != MAP_FAILED && n) munmap(p, n);
  }
};

}  // namespace

std::vector<CaseInput> read_bsdata(const std::string& path) {
  const int fd = open(path.c_str(), O_RDONLY);
  if (fd < 0) throw std::runtime_error("Cannot open bsdata file: " + path);
  struct stat st;
  if (fstat(fd, &st) != 0) {
    close(fd);
    throw std::runtime_error("Cannot stat bsdata file: " + path);
  }
  auto map = std::make_shared<Mapping>();
  map->n = static_cast<size_t>(st.st_size);
  if (map->n) map->p = mmap(nullptr, map->n, PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (map->n && map->p == MAP_FAILED) throw std::runtime_error("Cannot map bsdata file: " + path);
  const uint8_t* raw = map->n ? static_cast<const uint8_t*>(map->p) : nullptr;
  const uint8_t* sep = raw ? static_cast<const uint8_t*>(std::memchr(raw, 0, map->n)) : nullptr;
  if (!sep) throw std::runtime_error("Invalid bsdata file (no NUL separator): " + path);
  size_t hlen = static_cast<size_t>(sep - raw);
  JVal h = json_parse(reinterpret_cast<const char*>(raw), hlen);
  const uint8_t* bin = raw + hlen + 1;
  size_t bin_len = map->n - hlen - 1;
  t_hold = map;
  std::vector<CaseInput> cases;
  const JVal* multi = h.get("cases");
  if (!multi) multi = h.get("layers");
  try {
    if (multi) {
      for (auto& e : multi->a) cases.push_back(parse_case(e, bin, bin_len));
    } else {
      cases.push_back(parse_case(h, bin, bin_len));
    }
  } catch (...) {
    t_hold.reset();
    throw;
  }
  t_hold.reset();
  if (cases.size() == 1) {
    cases[0].name = path;
  } else {
    for (size_t i = 0; i < cases.size(); ++i) cases[i].name = path + "[" + std::to_string(i) + "]";
  }
  return cases;
}

CaseInput parse_json_case(const std::string& text) {
  JVal h = json_parse(text.data(), text.size());
  if (h.type != JVal::Obj) throw std::runtime_error("JSON parse error: input is not an object");
  return parse_case(h, nullptr, 0);
}

// ---------------------------------------------------------------- driver ---
namespace {

BufRef upload(Device& dev, const StreamVal& v, int64_t nw) {
  BufRef b = dev.alloc_stream(nw);
  size_t have = std::min<size_t>(v.n_words(), static_cast<size_t>(nw));
  if (have && v.view) {
    // whole words straight from the mapping; a partial last word and the
    // zero words after the stored bytes are filled from a padded copy
    const size_t bytes = std::min(v.view_bytes, have * 8);
    const size_t whole = bytes / 8;
    dev.h2d(b->p, v.view, whole * 8);
    if (whole < have) {
      std::vector<uint64_t> rest(have - whole, 0);
      std::memcpy(rest.data(), v.view + whole * 8, bytes - whole * 8);
      BSZ_CUDA(cudaMemcpyAsync(b->p + whole, rest.data(), rest.size() * 8, cudaMemcpyHostToDevice, dev.stream()));
      BSZ_CUDA(cudaStreamSynchronize(dev.stream()));   // `rest` is a local
    }
  } else if (have) {
    dev.h2d(b->p, v.words.data(), have * 8);
  }
  if (static_cast<int64_t>(have) < nw) {
    uint64_t fill = v.tail ? ~uint64_t(0) : 0;
    launch_fill(dev, b->p + have, nw - static_cast<int64_t>(have), fill, fill);
  }
  return b;
}

bool is_clean(const StreamVal& v, int64_t N, int64_t nw) {
  if (v.tail) return false;
  int64_t lw = (N + 63) / 64;
  if (lw <= 0) return true;
  const size_t n = v.n_words();
  if (static_cast<int64_t>(n) >= lw) {
    uint64_t hi = v.word(static_cast<size_t>(lw - 1)) & ~mask_for_bits(N);
    if (hi) return false;
  }
  for (size_t i = static_cast<size_t>(lw); i < n && static_cast<int64_t>(i) < nw; ++i)
    if (v.word(i)) return false;
  return true;
}

void download(Device& dev, const BufRef& b, int64_t nw, std::vector<uint64_t>& out) {
  out.resize(nw);
  dev.d2h(out.data(), b->p, static_cast<size_t>(nw) * 8);
}

}  // namespace

static const char* const kModeNames[4] = {"b200-plain", "b200-fused", "b200-auto", "b200-vm"};

std::string run_case_json(Device& dev, const Program& prog, CaseInput& c, const DriverOptions& o,
                          double parse_ms) {
  using clk = std::chrono::high_resolution_clock;
  std::unordered_map<std::string, int64_t> pmap(c.params.begin(), c.params.end());
  int64_t static_ops = count_static_ops(prog, pmap);
  int64_t nw = c.bitlength > 0 ? (c.bitlength + 63) / 64 : 1;
  if (c.bitlength <= 0)
    for (auto& kv : c.inputs) nw = std::max<int64_t>(nw, static_cast<int64_t>(kv.second.n_words()));
  const int64_t N = c.bitlength > 0 ? c.bitlength : 64 * nw;

  ExecOptions eo;
  eo.mode = static_cast<ExecMode>(o.mode & 3);

  struct OutRec {
    std::map<std::string, std::pair<std::vector<uint64_t>, uint8_t>> streams;
    std::map<std::string, std::map<int64_t, std::vector<uint64_t>>> arrays;
    std::map<std::string, int64_t> ints;
  };

  auto one_run = [&](std::map<std::string, StreamVal>& inputs, OutRec& rec, double& kernel_ms,
                     Executor** keep) -> std::unique_ptr<Executor> {
    cudaEvent_t e0, e1;
    BSZ_CUDA(cudaEventCreate(&e0));
    BSZ_CUDA(cudaEventCreate(&e1));
    BSZ_CUDA(cudaEventRecord(e0, dev.stream()));
    auto ex = std::make_unique<Executor>(dev, prog, N, eo);
    for (auto& kv : c.params) ex->set_param(prog.find(kv.first), kv.second);
    for (int id : prog.inputs) {
      const std::string& name = prog.names[id];
      auto it = inputs.find(name);
      if (it != inputs.end()) {
        ex->bind_input(id, upload(dev, it->second, nw), it->second.tail, is_clean(it->second, N, nw));
        continue;
      }
      auto bc = c.broadcast.find(name);
      if (bc != c.broadcast.end()) { ex->bind_broadcast(id, bc->second); continue; }
      auto ar = c.arrays.find(name);
      if (ar != c.arrays.end()) {
        for (auto& e : ar->second)
          ex->bind_input_array(id, e.first, upload(dev, e.second, nw), e.second.tail,
                               is_clean(e.second, N, nw));
      }
    }
    ex->run();
    for (int id : prog.outputs) {
      const std::string& name = prog.names[id];
      if (ex->has_stream(id)) {
        auto& slot = rec.streams[name];
        download(dev, ex->stream_value(id), nw, slot.first);
        slot.second = ex->stream_tail(id);
      }
      if (ex->has_array(id)) {
        auto& arr = rec.arrays[name];
        for (int64_t idx : ex->array_indices(id)) download(dev, ex->array_value(id, idx), nw, arr[idx]);
      }
    }
    for (int id : prog.output_ints) {
      int64_t v;
      if (ex->int_value(id, &v)) rec.ints[prog.names[id]] = v;
    }
    BSZ_CUDA(cudaEventRecord(e1, dev.stream()));
    BSZ_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    BSZ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    kernel_ms += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    (void)keep;
    return ex;
  };

  double warm_ms = 0;
  if (o.warmup) {
    auto t0 = clk::now();
    OutRec rec;
    double km = 0;
    auto inputs = c.inputs;
    one_run(inputs, rec, km, nullptr);
    warm_ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  }
  OutRec rec;
  double exec_ms = 0, kernel_ms = 0, compile_ms = 0;
  int64_t launches = 0, op_count = 0, max_live = 0, n_vars = 0;
  const int64_t launches0 = dev.n_launches;
  std::map<std::string, StreamVal> inputs = c.inputs;
  for (int it = 0; it < std::max(1, c.iterations); ++it) {
    rec = OutRec();
    auto t0 = clk::now();
    auto ex = one_run(inputs, rec, kernel_ms, nullptr);
    exec_ms += std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    op_count = ex->op_count;
    max_live = std::max(max_live, ex->max_live_buffers);
    compile_ms += ex->compile_ms;
    for (auto& fb : c.feedback) {
      auto s = rec.streams.find(fb.first);
      if (s != rec.streams.end()) {
        StreamVal v;
        v.words = s->second.first;
        v.tail = s->second.second;
        inputs[fb.second] = std::move(v);
      }
    }
  }
  launches = dev.n_launches - launches0;
  for (size_t id = 0; id < prog.names.size(); ++id)
    if (!prog.is_array[id]) ++n_vars;
  (void)n_vars;
  const int64_t dynamic_ops = op_count * std::max(1, c.iterations);

  // ---- JSON (key order of main.cu:146-206)
  std::string js;
  js.reserve(256);
  js += "{\"outputs\":{";
  bool first = true;
  const uint64_t lm = mask_for_bits(N);
  auto emit_stream = [&](std::vector<uint64_t>& w) {
    if (!w.empty()) w.back() &= lm;
    words_to_hex(w.data(), w.size(), js);
    js += '"';
  };
  for (int id : prog.outputs) {
    const std::string& name = prog.names[id];
    auto s = rec.streams.find(name);
    if (s != rec.streams.end()) {
      if (!first) js += ',';
      first = false;
      js += json_quote(name) + ":\"";
      emit_stream(s->second.first);
    }
    auto a = rec.arrays.find(name);
    if (a != rec.arrays.end()) {
      if (!first) js += ',';
      first = false;
      js += json_quote(name) + ":{";
      bool f2 = true;
      for (auto& e : a->second) {
        if (!f2) js += ',';
        f2 = false;
        js += "\"" + std::to_string(e.first) + "\":\"";
        emit_stream(e.second);
      }
      js += '}';
    }
  }
  for (int id : prog.output_ints) {
    auto it = rec.ints.find(prog.names[id]);
    if (it == rec.ints.end()) continue;
    if (!first) js += ',';
    first = false;
    js += json_quote(it->first) + ":" + std::to_string(it->second);
  }
  js += "}";
  int64_t scalar_names = 0;
  for (size_t id = 0; id < prog.names.size(); ++id)
    if (!prog.is_array[id]) ++scalar_names;
  char buf[1024];
  double gops = exec_ms > 0 ? static_cast<double>(dynamic_ops) * nw * 2.0 / (exec_ms * 1e-3) / 1e9 : 0.0;
  std::snprintf(buf, sizeof buf,
                ",\"op_count\":%lld,\"exec_ms\":%.6f,\"static_ops\":%lld,\"dynamic_ops\":%lld,"
                "\"n_words\":%lld,\"n_variables\":%lld,\"max_live\":%lld,"
                "\"n_kernel_launches\":%lld,\"n_mallocs\":%lld,\"peak_bytes\":%lld,"
                "\"reuse_bytes\":%lld,\"int32_gops\":%.6f,\"executor\":\"%s\","
                "\"timing\":{\"parse_ms\":%.6f,\"liveness_ms\":0.0,\"compile_ms\":%.6f,"
                "\"alloc_ms\":0.0,\"exec_ms\":%.6f,\"kernel_ms\":%.6f,\"warmup_ms\":%.6f,\"runs\":1}}",
                static_cast<long long>(dynamic_ops), exec_ms, static_cast<long long>(static_ops),
                static_cast<long long>(dynamic_ops), static_cast<long long>(nw),
                static_cast<long long>(scalar_names), static_cast<long long>(max_live),
                static_cast<long long>(launches), static_cast<long long>(dev.n_mallocs),
                static_cast<long long>(dev.bytes_peak),
                static_cast<long long>(max_live * nw * 8), gops,
                kModeNames[o.mode & 3], parse_ms, compile_ms, exec_ms, kernel_ms,
                warm_ms);
  js += buf;
  return js;
}

}  // namespace bsz
