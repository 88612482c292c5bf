// Host I/O: JSON, hex words, .bsdata files, and the whole-case driver that
// produces the bsim_cuda JSON result.
//
// Formats kept from the reference:
//  * .bsdata = UTF-8 JSON header, NUL, little-endian packed stream bytes;
//    "_bin": [offset, nbytes], "_array_bin": [count, offset, stride],
//    "_broadcast_pack": [count, offset, nbytes], multi-case {"cases": [...]}
//    (benchmark/bsdata.py:1-17, simulator/csim/src/bsdata_reader.h:31-299)
//  * stdin JSON input {"inputs", "params", "n_vectors"|"bitlength",
//    "input_arrays", "iterations", "feedback"} (benchmark/base.py:261-275)
//  * result JSON fields (simulator/csim/src/main.cu:146-206)
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace bsz {

struct JVal {
  enum Type : uint8_t { Null, Bool, Int, Real, Str, Arr, Obj } type = Null;
  bool b = false;
  int64_t i = 0;
  double d = 0;
  std::string s;
  std::vector<JVal> a;
  std::vector<std::pair<std::string, JVal>> o;
  const JVal* get(const std::string& k) const {
    for (auto& kv : o)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

JVal json_parse(const char* p, size_t n);
std::string json_quote(const std::string& s);

// Hex <-> words.  Hex strings are "0x..." (MSB first) with an optional
// leading '-'; a negative value becomes its two's complement over n words
// with tail bit 1.
void hex_to_words(const std::string& hex, std::vector<uint64_t>& words, uint8_t& tail);
void words_to_hex(const uint64_t* w, size_t n, std::string& out);   // appends "0x..."

// A stream input: owned words (JSON inputs, fed-back outputs), or a view of
// packed bytes inside a memory-mapped .bsdata file (no host copy; `hold`
// keeps the mapping alive).  Either way the value has n_words() words,
// zero past the stored bytes, and bits beyond them equal to `tail`.
struct StreamVal {
  std::vector<uint64_t> words;
  const uint8_t* view = nullptr;
  size_t view_bytes = 0;
  size_t view_words = 0;
  std::shared_ptr<const void> hold;
  uint8_t tail = 0;
  size_t n_words() const { return view ? view_words : words.size(); }
  uint64_t word(size_t i) const;
  void materialize();   // view -> words
};

struct CaseInput {
  std::string name;
  int64_t bitlength = 0;
  std::vector<std::pair<std::string, int64_t>> params;
  std::map<std::string, StreamVal> inputs;
  std::map<std::string, std::map<int64_t, StreamVal>> arrays;
  std::map<std::string, std::vector<uint8_t>> broadcast;
  int iterations = 1;
  std::vector<std::pair<std::string, std::string>> feedback;   // output -> input
};

// Reads every case of a .bsdata file.
std::vector<CaseInput> read_bsdata(const std::string& path);
// Parses the stdin JSON form.
CaseInput parse_json_case(const std::string& text);

class Device;
struct Program;

struct DriverOptions {
  bool warmup = false;
  int mode = 2;   // 0 plain, 1 fused, 2 auto, 3 vm (ExecMode)
};

// Runs one case end to end (H2D, execute, D2H) and returns the JSON object
// text of the bsim_cuda result for it.
std::string run_case_json(Device& dev, const Program& prog, CaseInput& c,
                          const DriverOptions& opt, double parse_ms);

}  // namespace bsz
