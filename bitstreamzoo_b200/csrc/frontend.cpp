// Tokenizer, recursive-descent parser and 3-address validator for the DSL.
// Grammar and precedence: DSL.md:300-360 and simulator/csim/src/parser.cpp:
// stream operators bind (tightest first) ~, << >>, &, +, ^, |; integer
// expressions use * over + -.
#include "frontend.h"

#include <cctype>

namespace bsz {
namespace {

enum class T : uint8_t {
  Input, Output, Param, Stream, Int, If, While, For, In, Zero, Ones, Popcount,
  Ident, Number, LBrace, RBrace, LParen, RParen, LBracket, RBracket,
  Assign, Tilde, Amp, Pipe, Caret, Shl, Shr, Plus, Minus, Star, DotDot, End
};

const char* tname(T t) {
  static const char* n[] = {
      "INPUT", "OUTPUT", "PARAM", "STREAM", "INT", "IF", "WHILE", "FOR", "IN", "ZERO",
      "ONES", "POPCOUNT", "IDENT", "INT_LIT", "LBRACE", "RBRACE", "LPAREN", "RPAREN",
      "LBRACKET", "RBRACKET", "ASSIGN", "TILDE", "AMP", "PIPE", "CARET", "LSHIFT",
      "RSHIFT", "PLUS", "MINUS", "STAR", "DOTDOT", "EOF"};
  return n[static_cast<int>(t)];
}

struct Tok {
  T t;
  std::string text;
  int line;
};

T keyword(const std::string& w) {
  static const std::unordered_map<std::string, T> kw = {
      {"input", T::Input}, {"output", T::Output}, {"param", T::Param},
      {"stream", T::Stream}, {"int", T::Int}, {"if", T::If}, {"while", T::While},
      {"for", T::For}, {"in", T::In}, {"ZERO", T::Zero}, {"ONES", T::Ones},
      {"popcount", T::Popcount}};
  auto it = kw.find(w);
  return it == kw.end() ? T::Ident : it->second;
}

std::vector<Tok> lex(const std::string& s) {
  std::vector<Tok> out;
  out.reserve(s.size() / 3 + 8);
  int line = 1;
  size_t i = 0, n = s.size();
  auto push = [&](T t, size_t len) {
    out.push_back({t, s.substr(i, len), line});
    i += len;
  };
  while (i < n) {
    char c = s[i];
    if (c == '\n') { ++line; ++i; continue; }
    if (c == ' ' || c == '\t' || c == '\r') { ++i; continue; }
    if (c == '/' && i + 1 < n && s[i + 1] == '/') {
      while (i < n && s[i] != '\n') ++i;
      continue;
    }
    char d = i + 1 < n ? s[i + 1] : '\0';
    if (c == '<' && d == '<') { push(T::Shl, 2); continue; }
    if (c == '>' && d == '>') { push(T::Shr, 2); continue; }
    if (c == '.' && d == '.') { push(T::DotDot, 2); continue; }
    switch (c) {
      case '{': push(T::LBrace, 1); continue;
      case '}': push(T::RBrace, 1); continue;
      case '(': push(T::LParen, 1); continue;
      case ')': push(T::RParen, 1); continue;
      case '[': push(T::LBracket, 1); continue;
      case ']': push(T::RBracket, 1); continue;
      case '=': push(T::Assign, 1); continue;
      case '~': push(T::Tilde, 1); continue;
      case '&': push(T::Amp, 1); continue;
      case '|': push(T::Pipe, 1); continue;
      case '^': push(T::Caret, 1); continue;
      case '+': push(T::Plus, 1); continue;
      case '-': push(T::Minus, 1); continue;
      case '*': push(T::Star, 1); continue;
      default: break;
    }
    if (std::isdigit(static_cast<unsigned char>(c))) {
      size_t j = i;
      while (j < n && std::isdigit(static_cast<unsigned char>(s[j]))) ++j;
      push(T::Number, j - i);
      continue;
    }
    if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
      size_t j = i;
      while (j < n && (std::isalnum(static_cast<unsigned char>(s[j])) || s[j] == '_')) ++j;
      std::string w = s.substr(i, j - i);
      push(keyword(w), j - i);
      continue;
    }
    throw ParseError("line " + std::to_string(line) + ": unexpected character '" +
                     std::string(1, c) + "'");
  }
  out.push_back({T::End, "", line});
  return out;
}

class Parser {
 public:
  Parser(std::vector<Tok> toks, Program& p) : t_(std::move(toks)), p_(p) {}

  void program() {
    while (!at(T::End)) {
      if (at(T::Input)) {
        take(); want(T::Stream);
        int id = name();
        if (at(T::LBracket)) { take(); int_expr(); want(T::RBracket); p_.is_array[id] = 1; }
        p_.inputs.push_back(id);
      } else if (at(T::Output)) {
        take();
        if (at(T::Int)) {
          take();
          int id = name();
          int_names_.push_back(id);
          p_.output_ints.push_back(id);
          Stmt s; s.kind = Stmt::IntDecl; s.name = id;
          s.ie = lit(0);
          p_.stmts.push_back(std::move(s));
        } else {
          want(T::Stream);
          int id = name();
          if (at(T::LBracket)) { take(); int_expr(); want(T::RBracket); p_.is_array[id] = 1; }
          p_.outputs.push_back(id);
        }
      } else if (at(T::Param)) {
        take(); want(T::Int);
        int id = name();
        int_names_.push_back(id);
        p_.params.push_back(id);
      } else {
        p_.stmts.push_back(statement(true));
      }
    }
  }

 private:
  std::vector<Tok> t_;
  size_t i_ = 0;
  Program& p_;
  std::vector<int> int_names_;   // ids declared int so far (parse order matters)

  bool at(T t) const { return t_[i_].t == t; }
  const Tok& peek() const { return t_[i_]; }
  Tok take() { return t_[i_++]; }
  [[noreturn]] void fail(const std::string& what) {
    const Tok& k = peek();
    throw ParseError("line " + std::to_string(k.line) + ": " + what + ", got " + tname(k.t) +
                     " ('" + k.text + "')");
  }
  void want(T t) {
    if (!at(t)) fail(std::string("expected ") + tname(t));
    take();
  }
  int name() {
    if (!at(T::Ident)) fail("expected IDENT");
    return p_.intern(take().text);
  }
  bool is_int_name(int id) const {
    for (int x : int_names_) if (x == id) return true;
    return false;
  }
  static std::unique_ptr<IExpr> lit(int64_t v) {
    auto e = std::make_unique<IExpr>();
    e->kind = IExpr::Lit;
    e->value = v;
    return e;
  }

  Stmt statement(bool top) {
    Stmt s;
    if (at(T::Stream)) {
      take();
      s.name = name();
      if (at(T::LBracket)) {
        take();
        s.kind = Stmt::ArrayDecl;
        s.ie = int_expr();
        want(T::RBracket);
        p_.is_array[s.name] = 1;
        return s;
      }
      s.kind = Stmt::LocalDecl;
      if (at(T::Assign)) { take(); s.e = stream_expr(); }
      return s;
    }
    if (at(T::Int)) {
      take();
      s.kind = Stmt::IntDecl;
      s.name = name();
      int_names_.push_back(s.name);
      want(T::Assign);
      s.ie = int_expr();
      return s;
    }
    if (at(T::If) || at(T::While)) {
      s.kind = take().t == T::If ? Stmt::If : Stmt::While;
      want(T::LParen);
      s.e = stream_expr();
      want(T::RParen);
      s.body = block();
      return s;
    }
    if (at(T::For)) {
      take();
      s.kind = Stmt::For;
      s.name = name();
      int_names_.push_back(s.name);
      want(T::In);
      s.ie = int_expr();
      want(T::DotDot);
      s.ie2 = int_expr();
      s.body = block();
      return s;
    }
    if (at(T::Ident)) {
      s.name = name();
      if (at(T::LBracket)) {
        take();
        s.kind = Stmt::ArrayAssign;
        s.ie = int_expr();
        want(T::RBracket);
        want(T::Assign);
        s.e = stream_expr();
        return s;
      }
      want(T::Assign);
      if (is_int_name(s.name)) {
        s.kind = Stmt::IntAssign;
        s.ie = int_expr();
      } else {
        s.kind = Stmt::Assign;
        s.e = stream_expr();
      }
      return s;
    }
    fail(top ? "unexpected token" : "unexpected token in block");
  }

  std::vector<Stmt> block() {
    want(T::LBrace);
    std::vector<Stmt> body;
    while (!at(T::RBrace)) {
      if (at(T::End)) fail("expected RBRACE");
      body.push_back(statement(false));
    }
    take();
    return body;
  }

  // stream precedence (loosest first): | ^ + & then shifts, then unary ~
  std::unique_ptr<SExpr> bin(char op, std::unique_ptr<SExpr> a, std::unique_ptr<SExpr> b) {
    auto e = std::make_unique<SExpr>();
    e->kind = SExpr::Bin;
    e->op = op;
    e->a = std::move(a);
    e->b = std::move(b);
    return e;
  }
  std::unique_ptr<SExpr> stream_expr() { return level(0); }
  std::unique_ptr<SExpr> level(int lv) {
    static const T toks[4] = {T::Pipe, T::Caret, T::Plus, T::Amp};
    static const char ops[4] = {'|', '^', '+', '&'};
    if (lv == 4) return shift_expr();
    auto left = level(lv + 1);
    while (at(toks[lv])) {
      take();
      left = bin(ops[lv], std::move(left), level(lv + 1));
    }
    return left;
  }
  std::unique_ptr<SExpr> shift_expr() {
    auto left = unary();
    while (at(T::Shl) || at(T::Shr)) {
      char op = take().t == T::Shl ? '<' : '>';
      auto e = std::make_unique<SExpr>();
      e->kind = SExpr::Shift;
      e->op = op;
      e->a = std::move(left);
      e->index = int_expr();
      left = std::move(e);
    }
    return left;
  }
  std::unique_ptr<SExpr> unary() {
    if (at(T::Tilde)) {
      take();
      auto e = std::make_unique<SExpr>();
      e->kind = SExpr::Not;
      e->a = unary();
      return e;
    }
    return primary();
  }
  std::unique_ptr<SExpr> primary() {
    auto e = std::make_unique<SExpr>();
    if (at(T::Zero)) { take(); e->kind = SExpr::Zero; return e; }
    if (at(T::Ones)) { take(); e->kind = SExpr::Ones; return e; }
    if (at(T::LParen)) {
      take();
      auto inner = stream_expr();
      want(T::RParen);
      return inner;
    }
    if (at(T::Ident)) {
      e->name = name();
      if (at(T::LBracket)) {
        take();
        e->kind = SExpr::Elem;
        e->index = int_expr();
        want(T::RBracket);
      } else {
        e->kind = SExpr::Var;
      }
      return e;
    }
    fail("expected stream expression");
  }

  std::unique_ptr<IExpr> ibin(char op, std::unique_ptr<IExpr> a, std::unique_ptr<IExpr> b) {
    auto e = std::make_unique<IExpr>();
    e->kind = IExpr::Bin;
    e->op = op;
    e->a = std::move(a);
    e->b = std::move(b);
    return e;
  }
  std::unique_ptr<IExpr> int_expr() {
    auto left = int_term();
    while (at(T::Plus) || at(T::Minus)) {
      char op = take().t == T::Plus ? '+' : '-';
      left = ibin(op, std::move(left), int_term());
    }
    return left;
  }
  std::unique_ptr<IExpr> int_term() {
    auto left = int_atom();
    while (at(T::Star)) {
      take();
      left = ibin('*', std::move(left), int_atom());
    }
    return left;
  }
  std::unique_ptr<IExpr> int_atom() {
    if (at(T::Number)) {
      const std::string txt = take().text;
      int64_t v = 0;
      for (char c : txt) {
        if (v > (INT64_MAX - 9) / 10) throw ParseError("integer literal out of range: " + txt);
        v = v * 10 + (c - '0');
      }
      return lit(v);
    }
    if (at(T::LParen)) {
      take();
      auto e = int_expr();
      want(T::RParen);
      return e;
    }
    if (at(T::Popcount)) {
      take();
      want(T::LParen);
      auto e = std::make_unique<IExpr>();
      e->kind = IExpr::Pop;
      e->arg = stream_expr();
      want(T::RParen);
      return e;
    }
    if (at(T::Ident)) {
      auto e = std::make_unique<IExpr>();
      e->kind = IExpr::Var;
      e->name = name();
      return e;
    }
    fail("expected integer expression");
  }
};

bool is_primary(const SExpr& e) {
  return e.kind == SExpr::Var || e.kind == SExpr::Elem || e.kind == SExpr::Zero ||
         e.kind == SExpr::Ones;
}

void check_rhs(const SExpr& e, const std::string& ctx) {
  if (is_primary(e)) return;
  switch (e.kind) {
    case SExpr::Not:
      if (!is_primary(*e.a)) throw ThreeAddrError(ctx + ": unary operand must be a primary");
      return;
    case SExpr::Bin:
      if (!is_primary(*e.a)) throw ThreeAddrError(ctx + ": binary left operand must be a primary");
      if (!is_primary(*e.b)) throw ThreeAddrError(ctx + ": binary right operand must be a primary");
      return;
    case SExpr::Shift:
      if (!is_primary(*e.a)) throw ThreeAddrError(ctx + ": shift operand must be a primary");
      return;
    default:
      throw ThreeAddrError(ctx + ": unknown expression type in stream RHS");
  }
}

void check_int(const IExpr& e, const std::string& ctx) {
  if (e.kind == IExpr::Pop && e.arg->kind != SExpr::Var)
    throw ThreeAddrError(ctx + ": popcount arg must be a variable");
}

// Popcount may also appear nested inside integer arithmetic, where the
// reference parser accepts any stream expression and the interpreter then
// requires a variable; enforce the variable rule there too.
void check_int_deep(const IExpr& e, const std::string& ctx) {
  if (e.kind == IExpr::Pop) {
    if (e.arg->kind != SExpr::Var) throw ThreeAddrError(ctx + ": popcount arg must be a variable");
  } else if (e.kind == IExpr::Bin) {
    check_int_deep(*e.a, ctx);
    check_int_deep(*e.b, ctx);
  }
}

void check_stmts(std::vector<Stmt>& v, const Program& p, const std::string& ctx, int& next_id) {
  for (auto& s : v) {
    s.id = next_id++;
    switch (s.kind) {
      case Stmt::LocalDecl:
        if (s.e) check_rhs(*s.e, ctx + ": stream " + p.names[s.name]);
        break;
      case Stmt::Assign: check_rhs(*s.e, ctx + ": " + p.names[s.name]); break;
      case Stmt::ArrayAssign: check_rhs(*s.e, ctx + ": " + p.names[s.name] + "[...]"); break;
      case Stmt::IntDecl:
      case Stmt::IntAssign:
        check_int(*s.ie, ctx + ": " + p.names[s.name]);
        check_int_deep(*s.ie, ctx + ": " + p.names[s.name]);
        break;
      case Stmt::If:
      case Stmt::While:
        if (s.e->kind != SExpr::Var)
          throw ThreeAddrError(ctx + (s.kind == Stmt::If ? ": if" : ": while") +
                               " condition must be a variable");
        check_stmts(s.body, p, ctx, next_id);
        break;
      case Stmt::For: check_stmts(s.body, p, ctx, next_id); break;
      default: break;
    }
  }
}

struct OpCounter {
  const Program& p;
  std::unordered_map<int, int64_t> env;

  int64_t ival(const IExpr& e) {
    switch (e.kind) {
      case IExpr::Lit: return e.value;
      case IExpr::Var: {
        auto it = env.find(e.name);
        return it == env.end() ? 0 : it->second;
      }
      case IExpr::Bin: {
        int64_t a = ival(*e.a), b = ival(*e.b);
        return e.op == '+' ? a + b : e.op == '-' ? a - b : a * b;
      }
      default: return 0;
    }
  }
  static bool compute(const SExpr* e) { return e && !is_primary(*e); }
  int64_t count(const std::vector<Stmt>& v) {
    int64_t total = 0;
    for (const auto& s : v) {
      switch (s.kind) {
        case Stmt::LocalDecl:
        case Stmt::Assign:
        case Stmt::ArrayAssign: total += compute(s.e.get()) ? 1 : 0; break;
        case Stmt::IntDecl:
        case Stmt::IntAssign: total += s.ie->kind == IExpr::Pop ? 1 : 0; break;
        case Stmt::For: {
          int64_t lo = ival(*s.ie), hi = ival(*s.ie2);
          if (hi > lo) {
            auto saved = env;
            env[s.name] = lo;
            total += count(s.body) * (hi - lo);
            env = std::move(saved);
          }
          break;
        }
        case Stmt::If:
        case Stmt::While: total += count(s.body); break;
        default: break;
      }
    }
    return total;
  }
};

}  // namespace

std::unique_ptr<Program> parse_program(const std::string& source) {
  auto p = std::make_unique<Program>();
  Parser parser(lex(source), *p);
  parser.program();
  std::string ctx = p->inputs.empty() ? "<program>" : p->names[p->inputs[0]];
  int next_id = 0;
  check_stmts(p->stmts, *p, ctx, next_id);
  p->n_stmt_ids = next_id;
  return p;
}

int64_t count_static_ops(const Program& p, const std::unordered_map<std::string, int64_t>& params) {
  OpCounter c{p, {}};
  for (const auto& kv : params) {
    int id = p.find(kv.first);
    if (id >= 0) c.env[id] = kv.second;
  }
  return c.count(p.stmts);
}

}  // namespace bsz
