// bsim_cuda-compatible command line driver.
//
// Same contract as the reference binary (simulator/csim/src/main.cu:209-331):
//   bsim_cuda program.bs [--trace] [--word-bits=32|64] [--reuse-mem]
//             [--warmup] [--input file.bsdata ...] [--dump-input]
// Without --input a JSON case is read from stdin.  Prints one JSON object
// (an array with "name" per case for multi-case inputs) and exits 0; on error
// prints to stderr and exits 1 ("out of memory" is preserved in the message
// so the harness maps it to MemoryError, benchmark/base.py:219-223).
//
// Additional flag: --mode=plain|fused|auto|vm (default: $BSZ_MODE, else auto).
// --word-bits=32 is accepted; results do not depend on the word width, and
// the executor always computes on 64-bit words.
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

#include "device.h"
#include "frontend.h"
#include "io.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "Usage: bsim_cuda program.bs [--trace] [--word-bits=32|64] [--reuse-mem] "
                 "[--warmup] [--input file.bsdata ...] [--dump-input] [--mode=plain|fused|auto|vm]\n";
    return 1;
  }
  std::string bs_path = argv[1];
  bool dump_input = false;
  bsz::DriverOptions opt;
  auto mode_of = [](const std::string& m) {
    if (m == "plain") return 0;
    if (m == "fused") return 1;
    if (m == "vm") return 3;
    return 2;
  };
  const char* env_mode = std::getenv("BSZ_MODE");
  opt.mode = env_mode ? mode_of(env_mode) : 2;
  int word_bits = 64;
  std::vector<std::string> inputs;
  for (int i = 2; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "--trace" || a == "--reuse-mem") {
      // accepted for compatibility; the executor always plans buffer reuse
    } else if (a == "--warmup") {
      opt.warmup = true;
    } else if (a.rfind("--word-bits=", 0) == 0) {
      word_bits = std::atoi(a.c_str() + 12);
    } else if (a == "--input" && i + 1 < argc) {
      inputs.push_back(argv[++i]);
    } else if (a == "--dump-input") {
      dump_input = true;
    } else if (a.rfind("--mode=", 0) == 0) {
      opt.mode = mode_of(a.substr(7));
    }
  }
  if (word_bits != 32 && word_bits != 64) {
    std::cerr << "Error: --word-bits must be 32 or 64\n";
    return 1;
  }
  std::ifstream fs(bs_path);
  if (!fs) {
    std::cerr << "Error: cannot open " << bs_path << "\n";
    return 1;
  }
  std::stringstream ss;
  ss << fs.rdbuf();
  const std::string source = ss.str();

  std::vector<bsz::CaseInput> cases;
  try {
    if (!inputs.empty()) {
      for (auto& f : inputs) {
        auto cs = bsz::read_bsdata(f);
        for (auto& c : cs) cases.push_back(std::move(c));
      }
    } else {
      std::stringstream in;
      in << std::cin.rdbuf();
      cases.push_back(bsz::parse_json_case(in.str()));
    }
  } catch (const std::exception& e) {
    std::cerr << (inputs.empty() ? "JSON parse error: " : "Error reading bsdata: ") << e.what() << "\n";
    return 1;
  }

  if (dump_input) {
    std::string out = cases.size() > 1 ? "[" : "";
    for (size_t ci = 0; ci < cases.size(); ++ci) {
      auto& c = cases[ci];
      for (auto& kv : c.inputs) kv.second.materialize();
      for (auto& kv : c.arrays)
        for (auto& e : kv.second) e.second.materialize();
      if (ci) out += ",";
      out += "{\"bitlength\":" + std::to_string(c.bitlength) + ",\"inputs\":{";
      bool first = true;
      for (auto& kv : c.inputs) {
        if (!first) out += ",";
        first = false;
        out += bsz::json_quote(kv.first) + ":\"";
        bsz::words_to_hex(kv.second.words.data(), kv.second.words.size(), out);
        out += "\"";
      }
      out += "},\"params\":{";
      first = true;
      for (auto& kv : c.params) {
        if (!first) out += ",";
        first = false;
        out += bsz::json_quote(kv.first) + ":" + std::to_string(kv.second);
      }
      out += "},\"input_arrays\":{";
      first = true;
      for (auto& kv : c.arrays) {
        if (!first) out += ",";
        first = false;
        out += bsz::json_quote(kv.first) + ":{";
        bool f2 = true;
        for (auto& e : kv.second) {
          if (!f2) out += ",";
          f2 = false;
          out += "\"" + std::to_string(e.first) + "\":\"";
          bsz::words_to_hex(e.second.words.data(), e.second.words.size(), out);
          out += "\"";
        }
        out += "}";
      }
      out += "}}";
    }
    if (cases.size() > 1) out += "]";
    std::cout << out << "\n";
    return 0;
  }

  auto t0 = std::chrono::high_resolution_clock::now();
  std::unique_ptr<bsz::Program> prog;
  try {
    prog = bsz::parse_program(source);
  } catch (const std::exception& e) {
    std::cerr << "Parse error: " << e.what() << "\n";
    return 1;
  }
  double parse_ms =
      std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();

  try {
    bsz::Device dev(0);
    std::string out;
    if (cases.size() == 1) {
      out = bsz::run_case_json(dev, *prog, cases[0], opt, parse_ms);
    } else {
      out = "[";
      for (size_t i = 0; i < cases.size(); ++i) {
        std::string one = bsz::run_case_json(dev, *prog, cases[i], opt, parse_ms);
        one.pop_back();
        one += ",\"name\":" + bsz::json_quote(cases[i].name) + "}";
        if (i) out += ",";
        out += one;
      }
      out += "]";
    }
    std::fwrite(out.data(), 1, out.size(), stdout);
    std::fputc('\n', stdout);
  } catch (const std::exception& e) {
    std::cerr << "Error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
