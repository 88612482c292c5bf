// Front end for the bitstream DSL: tokenizer, AST, parser, 3-address check.
//
// Accepts the grammar of the reference front ends (simulator/csim/src/
// lexer.cpp:62-144, parser.cpp:36-457; DSL.md:300-360) and raises the same
// two error classes (ParseError for syntax, ThreeAddrError for the 3-address
// rule).  Names are interned to dense integer ids at parse time so that the
// executor never hashes strings while it walks the program.
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace bsz {

struct ParseError : std::runtime_error { using std::runtime_error::runtime_error; };
struct ThreeAddrError : std::runtime_error { using std::runtime_error::runtime_error; };

// ---------------------------------------------------------------- AST ----

struct IExpr;

// Stream expression.  In 3-address form operands are primaries
// (Var / Elem / Zero / Ones), but the parser builds the general tree first,
// exactly like the reference, and the validator rejects nesting afterwards.
struct SExpr {
  enum Kind : uint8_t { Var, Elem, Zero, Ones, Not, Bin, Shift } kind;
  char op = 0;            // Bin: '&' '|' '^' '+'   Shift: '<' (<<) or '>' (>>)
  int name = -1;          // Var / Elem: interned name id
  std::unique_ptr<IExpr> index;   // Elem: array index;  Shift: amount
  std::unique_ptr<SExpr> a, b;    // operands
};

struct IExpr {
  enum Kind : uint8_t { Lit, Var, Bin, Pop } kind;
  char op = 0;            // Bin: '+' '-' '*'
  int64_t value = 0;      // Lit
  int name = -1;          // Var
  std::unique_ptr<IExpr> a, b;
  std::unique_ptr<SExpr> arg;     // Pop
};

struct Stmt {
  enum Kind : uint8_t {
    LocalDecl,   // stream x (= e)?          name, e (may be null)
    ArrayDecl,   // stream x[n]               name, ie
    IntDecl,     // int x = ie                name, ie
    Assign,      // x = e                     name, e
    ArrayAssign, // x[ie] = e                 name, ie, e
    IntAssign,   // x = ie                    name, ie
    If,          // if (e) { body }           e, body
    While,       // while (e) { body }        e, body
    For          // for x in ie..ie2 { body } name, ie, ie2, body
  } kind;
  int name = -1;
  std::unique_ptr<SExpr> e;
  std::unique_ptr<IExpr> ie, ie2;
  std::vector<Stmt> body;
  int id = -1;            // dense statement id (liveness tables)
};

struct Program {
  std::vector<Stmt> stmts;
  std::vector<int> inputs, outputs, params, output_ints;   // name ids, in order
  std::vector<std::string> names;                          // id -> name
  std::vector<uint8_t> is_array;                           // id -> declared as array
  int n_stmt_ids = 0;
  // Executor caches of this program (stream liveness, walks of straight-line
  // runs), created on first use and freed with the program.
  mutable std::mutex exec_mu;
  mutable std::shared_ptr<void> exec_cache;

  int find(const std::string& s) const {
    auto it = index_.find(s);
    return it == index_.end() ? -1 : it->second;
  }
  int intern(const std::string& s) {
    auto it = index_.find(s);
    if (it != index_.end()) return it->second;
    int id = static_cast<int>(names.size());
    names.push_back(s);
    is_array.push_back(0);
    index_.emplace(s, id);
    return id;
  }

 private:
  std::unordered_map<std::string, int> index_;
};

// Parse + validate.  Throws ParseError / ThreeAddrError.
std::unique_ptr<Program> parse_program(const std::string& source);

// Static op count: counted loops multiply their body, if/while bodies count
// once, copies and constants count zero (the bsim_cuda ``static_ops`` field;
// reference: simulator/csim/src/ast_liveness.cpp:629-727).
int64_t count_static_ops(const Program& p,
                         const std::unordered_map<std::string, int64_t>& params);

}  // namespace bsz
