// HVM-64 CPU ORACLE -- test infrastructure only, never the product.
//
// A C++ restatement of the reference evaluator (HigherOrderCO/hvm-64), used to
// check the CUDA reducer and as the timed CPU baseline.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
//
// The reference is Rust and cannot be built here (no cargo/rustc, git-only
// dependencies), so this file restates its algorithm.  Each part cites the
// reference file:line it follows.  Parity is pinned by tests/test_oracle.py
// against the reference's own snapshot files (tests/snapshots/run@*.snap),
// tests/lists.rs, tests/cli.rs and host/src/calc_labels.rs:196-234.
//
// Layout:  num (num/src/num.rs) -> ast + parser + printer (ast/src/*.rs)
//          -> runtime (runtime/src/*.rs) -> host (host/src/*.rs)
//          -> CLI (src/main.rs) and a small C ABI for the Python tests.
#include <algorithm>
#include <atomic>
#include <barrier>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <set>
#include <memory>
#include <optional>
#include <pthread.h>
#include <random>
#include <stdexcept>
#include <string>
#include <sys/mman.h>
#include <thread>
#include <unordered_map>
#include <vector>

namespace hvo {

using u8 = uint8_t;
using u16 = uint16_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i32 = int32_t;
using i64 = int64_t;

struct Panic : std::runtime_error {
  int code;
  Panic(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
enum { E_OK = 0, E_OOM = 1, E_BAD_PAIR = 2, E_DIV0 = 3, E_TIMEOUT = 4, E_BAD_INPUT = 5 };

// ===========================================================================
// num  (num/src/num.rs)
// ===========================================================================

// NumTag: num/src/num.rs:14-42 (value order and textual forms)
enum NumTag : u8 {
  U24 = 0, I24, F24, Sym, Add, Sub, SubS, Mul, Div, DivS, Rem, RemS,
  And, Or, Xor, Shl, ShlS, Shr, ShrS, Eq, Ne, Lt, Gt, NUMTAG_COUNT
};
static const char* const NUMTAG_STR[NUMTAG_COUNT] = {
  "u24", "i24", "f24", " ", "+", "-", ":-", "*", "/", ":/", "%", ":%",
  "&", "|", "^", "<<", ":<<", ">>", ":>>", "=", "!", "<", ">"};

static inline bool tag_is_op(u8 t) { return t > Sym; }  // num.rs:46-48
static inline bool tag_is_ty(u8 t) { return t < Sym; }  // num.rs:51-53

// bi_enum! from_str_prefix (util/src/bi_enum.rs:44-47): first declared match.
static int numtag_from_prefix(const char* s) {
  for (int t = 0; t < NUMTAG_COUNT; t++)
    if (strncmp(s, NUMTAG_STR[t], strlen(NUMTAG_STR[t])) == 0) return t;
  return -1;
}

struct Num {
  u32 raw;
  // num.rs:61-63
  static Num make(u8 tag, u32 payload) { return Num{(payload << 8) | (u32(tag) << 3) | 3u}; }
  static Num u24(u32 v) { return make(U24, v); }            // num.rs:71
  static Num i24(i32 v) { return make(I24, u32(v)); }       // num.rs:76
  static Num sym(u8 t) { return make(Sym, t); }             // num.rs:93
  static Num invalid() { return u24(0); }                   // num.rs:58
  // num.rs:81-90: round the low 8 bits off, ties to even, keep NaN a NaN.
  static Num f24(float val) {
    u32 bits;
    memcpy(&bits, &val, 4);
    u32 shifted = bits >> 8;
    u32 lost = bits & 0xFF;
    u32 nan = std::isnan(val) ? 1u : 0u;
    shifted += (nan ^ 1u) & ((lost - ((lost >> 7) & ~shifted)) >> 7);
    shifted |= nan;
    return make(F24, shifted);
  }
  u8 tag() const { return (raw >> 3) & 0x1f; }             // num.rs:103
  u32 payload() const { return raw >> 8; }                 // num.rs:108
  u32 get_u24() const { return payload(); }
  i32 get_i24() const { return i32(raw) >> 8; }            // num.rs:118
  float get_f24() const {                                  // num.rs:123
    u32 b = raw & ~0xffu;
    float f;
    memcpy(&f, &b, 4);
    return f;
  }
  u8 get_sym() const { return u8(get_u24()); }
};

// Rust `f as u32` / `f as i32`: saturating, NaN -> 0.
static inline u32 sat_u32(float f) {
  if (std::isnan(f) || f <= 0.0f) return 0;
  if (f >= 4294967296.0f) return 0xFFFFFFFFu;
  return u32(f);
}
static inline i32 sat_i32(float f) {
  if (std::isnan(f)) return 0;
  if (f <= -2147483648.0f) return INT32_MIN;
  if (f >= 2147483648.0f) return INT32_MAX;
  return i32(f);
}

// num.rs:133-161
static Num operate_unary(u8 op, Num num) {
  const u32 U24_MAX = (1u << 24) - 1;
  const i32 I24_MAX = (1 << 23) - 1, I24_MIN = -(1 << 23);
  switch (op) {
    case Sym: return num;
    case U24:
      switch (num.tag()) {
        case U24: return num;
        case I24: return Num::u24(num.get_u24());
        case F24: return Num::u24(std::min(sat_u32(num.get_f24()), U24_MAX));
        default: return Num::invalid();
      }
    case I24:
      switch (num.tag()) {
        case U24: return Num::i24(num.get_i24());
        case I24: return num;
        case F24: return Num::i24(std::clamp(sat_i32(num.get_f24()), I24_MIN, I24_MAX));
        default: return Num::invalid();
      }
    case F24:
      switch (num.tag()) {
        case U24: return Num::f24(float(num.get_u24()));
        case I24: return Num::f24(float(num.get_i24()));
        case F24: return num;
        default: return Num::invalid();
      }
    default: return Num::make(op, num.payload());
  }
}

static void div0() { throw Panic(E_DIV0, "attempt to divide by zero"); }

// num.rs:164-254.  `a` is always the op-tagged operand, `b` the typed one.
static Num operate_sym(Num a, Num b) {
  u8 at = a.tag(), bt = b.tag();
  if (at == Sym && bt == Sym) return Num::invalid();
  if (at == Sym) return operate_unary(a.get_sym(), b);
  if (bt == Sym) return operate_unary(b.get_sym(), a);
  bool ao = tag_is_op(at), bo = tag_is_op(bt);
  if (ao == bo) return Num::invalid();
  u8 op, ty;
  if (ao) { op = at; ty = bt; } else { op = bt; ty = at; std::swap(a, b); }
  if (ty == U24) {
    u32 x = a.get_u24(), y = b.get_u24();
    switch (op) {
      case Add: return Num::u24(x + y);
      case Sub: return Num::u24(x - y);
      case SubS: return Num::u24(y - x);
      case Mul: return Num::u24(x * y);
      case Div: if (y == 0) div0(); return Num::u24(x / y);
      case DivS: if (x == 0) div0(); return Num::u24(y / x);
      case Rem: if (y == 0) div0(); return Num::u24(x % y);
      case RemS: if (x == 0) div0(); return Num::u24(y % x);
      case Eq: return Num::u24(x == y);
      case Ne: return Num::u24(x != y);
      case Lt: return Num::u24(x < y);
      case Gt: return Num::u24(x > y);
      case And: return Num::u24(x & y);
      case Or: return Num::u24(x | y);
      case Xor: return Num::u24(x ^ y);
      case Shl: return Num::u24(x << (y & 31));
      case ShlS: return Num::u24(y << (x & 31));
      case Shr: return Num::u24(x >> (y & 31));
      case ShrS: return Num::u24(y >> (x & 31));
      default: return Num::invalid();
    }
  } else if (ty == I24) {
    i32 x = a.get_i24(), y = b.get_i24();
    auto wdiv = [](i32 p, i32 q) -> i32 {
      if (q == 0) div0();
      if (p == INT32_MIN && q == -1) return INT32_MIN;
      return p / q;
    };
    auto wrem = [](i32 p, i32 q) -> i32 {
      if (q == 0) div0();
      if (q == -1) return 0;
      return p % q;
    };
    switch (op) {
      case Add: return Num::i24(i32(u32(x) + u32(y)));
      case Sub: return Num::i24(i32(u32(x) - u32(y)));
      case SubS: return Num::i24(i32(u32(y) - u32(x)));
      case Mul: return Num::i24(i32(u32(x) * u32(y)));
      case Div: return Num::i24(wdiv(x, y));
      case DivS: return Num::i24(wdiv(y, x));
      case Rem: return Num::i24(wrem(x, y));
      case RemS: return Num::i24(wrem(y, x));
      case Eq: return Num::u24(x == y);
      case Ne: return Num::u24(x != y);
      case Lt: return Num::u24(x < y);
      case Gt: return Num::u24(x > y);
      case And: return Num::i24(x & y);
      case Or: return Num::i24(x | y);
      case Xor: return Num::i24(x ^ y);
      case Shl: return Num::i24(i32(u32(x) << (u32(y) & 31)));
      case ShlS: return Num::i24(i32(u32(y) << (u32(x) & 31)));
      case Shr: return Num::i24(x >> (u32(y) & 31));
      case ShrS: return Num::i24(y >> (u32(x) & 31));
      default: return Num::invalid();
    }
  } else if (ty == F24) {
    float x = a.get_f24(), y = b.get_f24();
    switch (op) {
      case Add: return Num::f24(x + y);
      case Sub: return Num::f24(x - y);
      case SubS: return Num::f24(y - x);
      case Mul: return Num::f24(x * y);
      case Div: return Num::f24(x / y);
      case DivS: return Num::f24(y / x);
      case Rem: return Num::f24(std::fmod(x, y));
      case RemS: return Num::f24(std::fmod(y, x));
      case Eq: return Num::u24(x == y);
      case Ne: return Num::u24(x != y);
      case Lt: return Num::u24(x < y);
      case Gt: return Num::u24(x > y);
      case And: return Num::f24(std::atan2(x, y));            // parity unpinned (libm)
      case Or: return Num::f24(std::log(y) / std::log(x));    // parity unpinned (libm)
      case Xor: return Num::f24(std::pow(x, y));              // parity unpinned (libm)
      default: return Num::invalid();
    }
  }
  return Num::invalid();
}

// num.rs:257-263
static Num operate_binary(Num a, u8 op, Num b) {
  if (op == Sym) return operate_sym(a, b);
  return operate_sym(operate_sym(a, Num::sym(op)), b);
}

// Rust `{:?}` for f32 (shortest round-trip digits; exponent form outside
// [1e-4, 1e16)).
static std::string rust_debug_f32(float v) {
  if (v == 0.0f) return std::signbit(v) ? "-0.0" : "0.0";
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
  std::string s(buf, r.ptr);
  bool neg = s[0] == '-';
  if (neg) s = s.substr(1);
  size_t epos = s.find('e');
  std::string mant = s.substr(0, epos);
  int exp10 = atoi(s.c_str() + epos + 1);
  std::string digits;
  for (char c : mant)
    if (c != '.') digits += c;
  float av = std::fabs(v);
  std::string out;
  if (av >= 1e-4f && av < 1e16f) {
    int n = int(digits.size());
    int point = exp10 + 1;  // digits before the decimal point
    if (point <= 0) {
      out = "0." + std::string(-point, '0') + digits;
    } else if (point < n) {
      out = digits.substr(0, point) + "." + digits.substr(point);
    } else {
      out = digits + std::string(point - n, '0') + ".0";
    }
  } else {
    out = digits.substr(0, 1);
    if (digits.size() > 1) out += "." + digits.substr(1);
    out += "e" + std::to_string(exp10);
  }
  return neg ? "-" + out : out;
}

// num.rs:287-305
static std::string num_to_string(Num n) {
  switch (n.tag()) {
    case Sym: {
      u8 s = n.get_sym();
      return std::string("[") + (s < NUMTAG_COUNT ? NUMTAG_STR[s] : "?") + "]";
    }
    case U24: return std::to_string(n.get_u24());
    case I24: {
      i32 v = n.get_i24();
      return (v >= 0 ? "+" : "") + std::to_string(v);
    }
    case F24: {
      float f = n.get_f24();
      if (std::isinf(f)) return f > 0 ? "+inf" : "-inf";
      if (std::isnan(f)) return "+NaN";
      return rust_debug_f32(f);
    }
    default: {
      u8 t = n.tag();
      return std::string("[") + (t < NUMTAG_COUNT ? NUMTAG_STR[t] : "?") + std::to_string(n.payload()) + "]";
    }
  }
}

// ===========================================================================
// ast  (ast/src/ast.rs, ast/src/parser.rs)
// ===========================================================================

enum TreeKind : u8 { T_ERA, T_NUM, T_REF, T_CTR, T_OP, T_SWITCH, T_VAR };

// ast.rs:57-96.  Trees live in an arena (no recursive destructors).
struct Tree {
  TreeKind kind = T_ERA;
  u16 lab = 0;
  Num num{0};
  std::string name;  // Ref / Var
  Tree* p1 = nullptr;
  Tree* p2 = nullptr;
};

struct Arena {
  std::deque<Tree> nodes;
  Tree* make(TreeKind k) {
    nodes.emplace_back();
    nodes.back().kind = k;
    return &nodes.back();
  }
};

// ast.rs:43-46
struct AstNet {
  Tree* root = nullptr;
  std::vector<std::pair<Tree*, Tree*>> redexes;
};

// ast.rs:29-31 (BTreeMap: names in byte order)
struct Book {
  std::shared_ptr<Arena> arena = std::make_shared<Arena>();
  std::map<std::string, AstNet> nets;
};

// create_var / var_to_num: util/src/create_var.rs:5-34
static std::string create_var(size_t id) {
  std::string txt;
  id += 1;
  while (id > 0) {
    id -= 1;
    txt.push_back(char('a' + id % 26));
    id /= 26;
  }
  std::reverse(txt.begin(), txt.end());
  return txt;
}
static std::optional<size_t> var_to_num(const std::string& s) {
  size_t n = 0;
  for (char c : s) {
    if (c < 'a') return std::nullopt;
    size_t i = size_t(c - 'a');
    if (i > size_t('z')) return std::nullopt;
    n = n * 26 + i + 1;
  }
  if (n == 0) return std::nullopt;
  return n - 1;
}

// TSPL-style recursive-descent parser: ast/src/parser.rs:300-451.  Trivia is
// ASCII whitespace and `//` line comments (the TSPL crate's skip_trivia).
struct Parser {
  const std::string& in;
  size_t i = 0;
  Arena& arena;
  Parser(const std::string& s, Arena& a) : in(s), arena(a) {}

  [[noreturn]] void expected(const std::string& what) {
    throw Panic(E_BAD_INPUT, "expected " + what + " at index " + std::to_string(i));
  }
  int peek() { return i < in.size() ? (unsigned char)in[i] : -1; }
  int advance() { return i < in.size() ? (unsigned char)in[i++] : -1; }
  void skip_trivia() {
    while (i < in.size()) {
      char c = in[i];
      if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f') { i++; continue; }
      if (c == '/' && in.compare(i, 2, "//") == 0) {
        while (i < in.size() && in[i] != '\n') i++;
        if (i < in.size()) i++;
        continue;
      }
      break;
    }
  }
  bool try_consume(const char* text) {
    skip_trivia();
    size_t n = strlen(text);
    if (in.compare(i, n, text) == 0) { i += n; return true; }
    return false;
  }
  void consume(const char* text) {
    if (!try_consume(text)) expected(std::string("'") + text + "'");
  }
  template <class F> std::string take_while(F f) {
    size_t s = i;
    while (i < in.size() && f(in[i])) i++;
    return in.substr(s, i - s);
  }
  static bool is_alnum(char c) { return isalnum((unsigned char)c) != 0; }
  u64 parse_u64() {
    skip_trivia();
    int radix = 10;
    if (in.compare(i, 2, "0x") == 0) { i += 2; radix = 16; }
    else if (in.compare(i, 2, "0b") == 0) { i += 2; radix = 2; }
    std::string s = take_while([&](char c) {
      if (c == '_') return true;
      if (radix == 16) return isxdigit((unsigned char)c) != 0;
      if (radix == 2) return c == '0' || c == '1';
      return isdigit((unsigned char)c) != 0;
    });
    std::string d;
    for (char c : s) if (c != '_') d += c;
    if (d.empty()) expected("numeric digit");
    return strtoull(d.c_str(), nullptr, radix);
  }
  // parser.rs:394-400
  std::string parse_name() {
    std::string n = take_while([](char c) { return is_alnum(c) || c == '_' || c == '.' || c == '$'; });
    if (n.empty()) expected("name");
    return n;
  }
  // parser.rs:442-450
  static u64 parse_int(const std::string& s) {
    auto bad = [&]() -> u64 { throw Panic(E_BAD_INPUT, "invalid number " + s); };
    std::string t = s;
    int radix = 10;
    if (t.rfind("0x", 0) == 0) { radix = 16; t = t.substr(2); }
    else if (t.rfind("0b", 0) == 0) { radix = 2; t = t.substr(2); }
    else if (!t.empty() && t[0] == '+') t = t.substr(1);  // u64::from_str accepts '+'
    if (t.empty()) return bad();
    u64 v = 0;
    for (char c : t) {
      int d;
      if (c >= '0' && c <= '9') d = c - '0';
      else if (c >= 'a' && c <= 'f') d = c - 'a' + 10;
      else if (c >= 'A' && c <= 'F') d = c - 'A' + 10;
      else return bad();
      if (d >= radix) return bad();
      if (v > (UINT64_MAX - u64(d)) / u64(radix)) return bad();
      v = v * u64(radix) + u64(d);
    }
    return v;
  }
  static float parse_float(const std::string& s) {
    std::string t = s;
    bool neg = false;
    if (!t.empty() && (t[0] == '+' || t[0] == '-')) { neg = t[0] == '-'; t = t.substr(1); }
    std::string low;
    for (char c : t) low += char(tolower((unsigned char)c));
    if (low == "inf" || low == "infinity") return neg ? -INFINITY : INFINITY;
    if (low == "nan") return neg ? -NAN : NAN;
    // Rust's decimal grammar: digits [. digits] [e[+-]digits]
    size_t k = 0;
    bool any = false;
    while (k < t.size() && isdigit((unsigned char)t[k])) { k++; any = true; }
    if (k < t.size() && t[k] == '.') { k++; while (k < t.size() && isdigit((unsigned char)t[k])) { k++; any = true; } }
    if (!any) throw Panic(E_BAD_INPUT, "invalid float " + s);
    if (k < t.size() && (t[k] == 'e' || t[k] == 'E')) {
      k++;
      if (k < t.size() && (t[k] == '+' || t[k] == '-')) k++;
      size_t e0 = k;
      while (k < t.size() && isdigit((unsigned char)t[k])) k++;
      if (k == e0) throw Panic(E_BAD_INPUT, "invalid float " + s);
    }
    if (k != t.size()) throw Panic(E_BAD_INPUT, "invalid float " + s);
    float f = strtof(t.c_str(), nullptr);
    return neg ? -f : f;
  }
  // parser.rs:428-440
  Num parse_num_lit() {
    std::string n = take_while([](char c) { return is_alnum(c) || c == '+' || c == '-' || c == '.'; });
    if (n.find('.') != std::string::npos || n.find("inf") != std::string::npos || n.find("NaN") != std::string::npos)
      return Num::f24(parse_float(n));
    if (!n.empty() && (n[0] == '+' || n[0] == '-')) {
      i32 v = i32(parse_int(n.substr(1)));
      return Num::i24(n[0] == '-' ? i32(0u - u32(v)) : v);
    }
    return Num::u24(u32(parse_int(n)));
  }
  // parser.rs:402-426
  Num parse_num() {
    skip_trivia();
    if (peek() != '[') return parse_num_lit();
    consume("[");
    int op = numtag_from_prefix(in.c_str() + i);
    if (op < 0) expected("operator");
    i += strlen(NUMTAG_STR[op]);
    skip_trivia();
    if (tag_is_ty(u8(op)) || peek() == ']') {
      consume("]");
      return Num::sym(u8(op));
    }
    Num lhs = parse_num_lit();
    consume("]");
    return operate_unary(u8(op), lhs);
  }
  // parser.rs:328-391
  Tree* parse_tree() {
    skip_trivia();
    int c = peek();
    if (c == '*') { advance(); return arena.make(T_ERA); }
    if (c == '(' || c == '{' || c == '#') {
      advance();
      u16 tag = 0;
      int ch = c;
      if (c == '#') {
        tag = u16(parse_u64());
        skip_trivia();
        ch = advance();
      }
      const char* close;
      u16 kind;
      if (ch == '(') { close = ")"; kind = 0; }
      else if (ch == '{') { close = "}"; kind = 1; }
      else expected("`(` or `{`");
      Tree* t = arena.make(T_CTR);
      t->lab = u16(tag * 2 + kind);
      skip_trivia();
      t->p1 = parse_tree();
      t->p2 = parse_tree();
      consume(close);
      return t;
    }
    if (c == '@') {
      advance();
      skip_trivia();
      Tree* t = arena.make(T_REF);
      t->name = parse_name();
      return t;
    }
    if (c == '$') {
      consume("$(");
      Tree* t = arena.make(T_OP);
      t->p1 = parse_tree();
      t->p2 = parse_tree();
      consume(")");
      return t;
    }
    if (c == '?') {
      consume("?(");
      Tree* t = arena.make(T_SWITCH);
      t->p1 = parse_tree();
      t->p2 = parse_tree();
      consume(")");
      return t;
    }
    if ((c >= '0' && c <= '9') || c == '+' || c == '-' || c == '[') {
      Tree* t = arena.make(T_NUM);
      t->num = parse_num();
      return t;
    }
    Tree* t = arena.make(T_VAR);
    t->name = parse_name();
    return t;
  }
  // parser.rs:316-326
  AstNet parse_net() {
    AstNet net;
    net.root = parse_tree();
    while (try_consume("&")) {
      Tree* a = parse_tree();
      consume("~");
      Tree* b = parse_tree();
      net.redexes.push_back({a, b});
    }
    return net;
  }
  // parser.rs:302-313
  void parse_book(Book& book) {
    while (try_consume("@")) {
      std::string name = parse_name();
      consume("=");
      book.nets[name] = parse_net();
    }
  }
  // parser.rs:455-462
  void eof() {
    if (i != in.size()) throw Panic(E_BAD_INPUT, "Unable to parse the whole input. Is this not an hvm64 file?");
  }
};

static Book parse_book(const std::string& text) {
  Book b;
  Parser p(text, *b.arena);
  p.parse_book(b);
  p.eof();
  return b;
}
static AstNet parse_net(const std::string& text, Arena& arena) {
  Parser p(text, arena);
  AstNet n = p.parse_net();
  p.eof();
  return n;
}
static Tree* parse_tree(const std::string& text, Arena& arena) {
  Parser p(text, arena);
  Tree* t = p.parse_tree();
  p.eof();
  return t;
}

// ast.rs:246-263
static void print_tree(std::string& o, const Tree* t) {
  switch (t->kind) {
    case T_ERA: o += "*"; return;
    case T_CTR: {
      u16 lab = t->lab;
      if (lab == 0) o += "(";
      else if (lab == 1) o += "{";
      else if (lab % 2 == 0) { o += "#" + std::to_string(lab / 2) + "("; }
      else { o += "#" + std::to_string(lab / 2) + "{"; }
      print_tree(o, t->p1);
      o += " ";
      print_tree(o, t->p2);
      o += (lab % 2 == 0) ? ")" : "}";
      return;
    }
    case T_VAR: o += t->name; return;
    case T_REF: o += "@" + t->name; return;
    case T_NUM: o += num_to_string(t->num); return;
    case T_OP: o += "$("; print_tree(o, t->p1); o += " "; print_tree(o, t->p2); o += ")"; return;
    case T_SWITCH: o += "?("; print_tree(o, t->p1); o += " "; print_tree(o, t->p2); o += ")"; return;
  }
}
// ast.rs:234-244
static std::string net_to_string(const AstNet& n) {
  std::string o;
  print_tree(o, n.root);
  for (auto& r : n.redexes) {
    o += "\n  & ";
    print_tree(o, r.first);
    o += " ~ ";
    print_tree(o, r.second);
  }
  return o;
}
// ast.rs:221-232
static std::string book_to_string(const Book& b) {
  std::string o;
  bool first = true;
  for (auto& [name, net] : b.nets) {
    if (!first) o += "\n\n";
    first = false;
    o += "@" + name + " = " + net_to_string(net);
  }
  return o;
}

static void tree_no_conflicts(const Tree* t, size_t& fresh) {  // ast.rs:169-176
  if (t->kind == T_VAR) {
    if (auto v = var_to_num(t->name)) fresh = std::max(fresh, *v);
  }
  if (t->p1) tree_no_conflicts(t->p1, fresh);
  if (t->p2) tree_no_conflicts(t->p2, fresh);
}
// ast.rs:112-123
static void apply_tree(AstNet& net, Tree* arg, Arena& arena) {
  size_t fresh = 0;
  tree_no_conflicts(net.root, fresh);
  for (auto& r : net.redexes) { tree_no_conflicts(r.first, fresh); tree_no_conflicts(r.second, fresh); }
  tree_no_conflicts(arg, fresh);
  std::string fresh_str = create_var(fresh + 1);
  Tree* fun = net.root;
  Tree* app = arena.make(T_CTR);
  app->lab = 0;
  app->p1 = arg;
  app->p2 = arena.make(T_VAR);
  app->p2->name = fresh_str;
  net.root = arena.make(T_VAR);
  net.root->name = fresh_str;
  net.redexes.push_back({fun, app});
}

// ===========================================================================
// runtime  (runtime/src/*.rs)
// ===========================================================================

using Lab = u16;
enum Tag : u8 { Red = 0, Var = 1, Ref = 2, NumT = 3, Op = 5, Switch = 6, Ctr = 7 };  // port.rs:22-86

// port.rs:105-116
static constexpr u64 P_ERA = 2;
static constexpr u64 P_FREE = 0x8000000000000000ull;
static constexpr u64 P_LOCK = 0xFFFFFFFFFFFFFFF0ull;
static constexpr u64 P_GONE = 0xFFFFFFFFFFFFFFFFull;

static inline u64 port_new(u8 tag, Lab lab, u64 addr) { return (u64(lab) << 48) | addr | tag; }  // port.rs:120
static inline u8 ptag(u64 p) { return p & 7; }
static inline Lab plab(u64 p) { return Lab(p >> 48); }
static inline u64 paddr(u64 p) { return p & 0x0000FFFFFFFFFFF8ull; }  // port.rs:173
static inline bool is_principal(u64 p) { return ptag(p) >= Ref; }    // port.rs:197
static inline bool is_skippable(u64 p) {                             // port.rs:205
  return ptag(p) == NumT || (ptag(p) == Ref && plab(p) != 0xFFFF);
}
static inline u64 port_var(u64 addr) { return port_new(Var, 0, addr); }
static inline u64 port_red(u64 addr) { return port_new(Red, 0, addr); }
static inline u64 other_half(u64 a) { return a ^ 8; }      // addr.rs:272
static inline u64 left_half(u64 a) { return a & ~u64(8); } // addr.rs:265

static inline std::atomic<u64>& at(u64 addr) { return *reinterpret_cast<std::atomic<u64>*>(addr); }
// wire.rs:318-350
static inline u64 w_load(u64 w) { return at(w).load(std::memory_order_relaxed); }
static inline void w_set(u64 w, u64 p) { at(w).store(p, std::memory_order_relaxed); }
static inline bool w_cas(u64 w, u64 expected, u64 value, u64* got) {
  u64 e = expected;
  bool ok = at(w).compare_exchange_strong(e, value, std::memory_order_relaxed, std::memory_order_relaxed);
  if (got) *got = e;
  return ok;
}
static inline u64 w_swap(u64 w, u64 v) { return at(w).exchange(v, std::memory_order_relaxed); }
static inline u64 w_lock(u64 w) {
  for (;;) {
    u64 got = w_swap(w, P_LOCK);
    if (got != P_LOCK) return got;
  }
}

struct Rewrites {  // runtime.rs:72-94
  u64 anni = 0, comm = 0, eras = 0, dref = 0, oper = 0;
  u64 total() const { return anni + comm + eras + dref + oper; }
};

// def.rs:7-62
struct LabSet {
  Lab min_safe = 0;
  std::vector<u64> bits;
  void add(Lab lab) {
    min_safe = std::max<Lab>(min_safe, Lab(lab + 1));
    size_t idx = lab >> 6;
    if (idx >= bits.size()) bits.resize(idx + 1, 0);
    bits[idx] |= u64(1) << (lab & 63);
  }
  bool has(Lab lab) const {
    if (lab >= min_safe) return false;
    size_t idx = lab >> 6;
    return idx < bits.size() && ((bits[idx] >> (lab & 63)) & 1);
  }
  void unite(const LabSet& o) {
    min_safe = std::max(min_safe, o.min_safe);
    for (size_t k = 0; k < std::min(bits.size(), o.bits.size()); k++) bits[k] |= o.bits[k];
    if (o.bits.size() > bits.size()) bits.insert(bits.end(), o.bits.begin() + bits.size(), o.bits.end());
  }
  static LabSet all() {
    LabSet s;
    s.min_safe = 0xFFFF;
    s.bits.assign(1024, ~u64(0));
    return s;
  }
};

// instruction.rs:34-72
enum InstrKind : u8 { I_CONST, I_LINK, I_LINKCONST, I_CTR, I_OP, I_OPNUM, I_SWITCH, I_WIRES };
struct Instruction {
  InstrKind k;
  Lab lab = 0;  // Ctr label / Op op
  u32 a = 0, b = 0, c = 0, d = 0;
  u64 port = 0;  // Const / LinkConst port, OpNum rhs raw
};

struct Net;
// D_INERT: transform/src/pre_reduce.rs:89-102 (InertDef), the stand-in for a
// reference missing from a Book being pre-reduced; its calls are captured.
enum DefKind : u8 { D_INTERPRETED, D_EXPAND, D_INERT };
// def.rs:86-95; aligned so that Ref ports can address it.
struct alignas(32) Def {
  LabSet labs;
  DefKind kind = D_INTERPRETED;
  std::vector<Instruction> instr;  // InterpretedDef (def.rs:194-199)
  size_t trgs = 1;
  u64 expand_out = 0;  // ExpandDef (net.rs:72-74)
};
static inline u64 port_ref(const Def* d) { return port_new(Ref, d->labs.min_safe, u64(uintptr_t(d))); }  // port.rs:138
static inline Def* port_def(u64 p) { return reinterpret_cast<Def*>(uintptr_t(paddr(p))); }

// Heap: allocator.rs:10-54.  Backed by an anonymous no-reserve mapping.
struct Heap {
  u64 base = 0;
  size_t nodes = 0;  // number of 16-byte nodes
  explicit Heap(size_t bytes) {
    nodes = bytes / 16;
    if (nodes == 0) throw Panic(E_OOM, "memory allocation failed");
    void* p = mmap(nullptr, nodes * 16, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) throw Panic(E_OOM, "memory allocation failed");
    // Transparent huge pages keep first-touch faults off the timed path.
    madvise(p, nodes * 16, MADV_HUGEPAGE);
    base = u64(uintptr_t(p));
  }
  ~Heap() { munmap(reinterpret_cast<void*>(uintptr_t(base)), nodes * 16); }
  Heap(const Heap&) = delete;
};

struct RedexQueue {  // linker.rs:307-344
  std::vector<std::pair<u64, u64>> fast, slow;
  size_t len() const { return fast.size() + slow.size(); }
  bool empty() const { return fast.empty() && slow.empty(); }
  bool pop(std::pair<u64, u64>& r) {
    if (!fast.empty()) { r = fast.back(); fast.pop_back(); return true; }
    if (!slow.empty()) { r = slow.back(); slow.pop_back(); return true; }
    return false;
  }
};

// linker.rs:347-351
static inline bool redex_would_shrink(u64 a, u64 b) {
  return (a == P_ERA || b == P_ERA) || (ptag(a) == Ctr && ptag(b) == Ctr && plab(a) == plab(b)) ||
         (!(ptag(a) == Ref || ptag(b) == Ref) && (ptag(a) == NumT || ptag(b) == NumT));
}

// Trg: linker.rs:228-281 (a wire is a Port with the Red tag holding the address)
static inline u64 trg_port(u64 p) { return p; }
static inline u64 trg_wire(u64 w) { return w; }
static inline bool trg_is_wire(u64 t) { return ptag(t) == Red; }
static inline u64 trg_target(u64 t) { return trg_is_wire(t) ? w_load(t) : t; }

// Order knob for the count-stability study: 0 = the reference's LIFO
// (fast-before-slow), 1 = FIFO, 2 = seeded random pick.
struct Net {
  // allocator.rs:57-62
  u64 heap_base;
  size_t heap_nodes;
  size_t next = 0;
  u64 head = 0;
  // linker.rs:10-14
  Rewrites rwts;
  RedexQueue redexes;
  // net.rs:7-13
  size_t tid = 0, tids = 1;
  std::vector<u64> trgs;
  u64 root = 0;
  int order = 0;
  std::mt19937_64 rng{12345};
  size_t fifo_pos_fast = 0, fifo_pos_slow = 0;
  std::vector<std::pair<u64, u64>>* captured = nullptr;  // InertDef calls (pre-reduce)

  Net(u64 base, size_t nodes) : heap_base(base), heap_nodes(nodes), trgs(1 << 16) {}

  // ---- allocator.rs:73-110
  void half_free(u64 addr) {
    w_set(addr, P_FREE);
    if (w_load(other_half(addr)) == P_FREE) {
      u64 l = left_half(addr);
      if (w_cas(l, P_FREE, head, nullptr)) head = l;
    }
  }
  u64 alloc() {
    u64 addr;
    if (head != 0) {
      addr = head;
      head = w_load(head);
    } else {
      size_t index = next++;
      if (index >= heap_nodes) throw Panic(E_OOM, "OOM");
      addr = heap_base + index * 16;
    }
    w_set(addr, P_LOCK);
    w_set(other_half(addr), P_LOCK);
    return addr;
  }
  void free_wire(u64 w) { half_free(w); }
  void free_trg(u64 t) { if (trg_is_wire(t)) free_wire(t); }

  // ---- node.rs:160-189
  struct Created { u64 p0, p1, p2; };
  Created create_node(u8 tag, Lab lab) {
    u64 a = alloc();
    return {port_new(tag, lab, a), port_var(a), port_var(other_half(a))};
  }
  std::pair<u64, u64> create_wire() {
    u64 a = alloc();
    half_free(other_half(a));
    return {a, port_var(a)};
  }
  u64 create_wire_to(u64 port) {
    u64 a = alloc();
    half_free(other_half(a));
    link_port_port(port, port_var(a));
    return a;
  }

  // ---- linker.rs:25-127
  void link_port_port(u64 a, u64 b) {
    if (is_principal(a) && is_principal(b)) redux(a, b);
    else { half_link_port_port(a, b); half_link_port_port(b, a); }
  }
  void link_wire_wire(u64 aw, u64 bw) {
    u64 ap = w_lock(aw);
    u64 bp = w_lock(bw);
    if (is_principal(ap) && is_principal(bp)) {
      free_wire(aw);
      free_wire(bw);
      redux(ap, bp);
    } else {
      half_link_wire_port(ap, aw, bp);
      half_link_wire_port(bp, bw, ap);
    }
  }
  void link_wire_port(u64 aw, u64 bp) {
    u64 ap = w_lock(aw);
    if (is_principal(ap) && is_principal(bp)) {
      free_wire(aw);
      redux(ap, bp);
    } else {
      half_link_wire_port(ap, aw, bp);
      half_link_port_port(bp, ap);
    }
  }
  void redux(u64 a, u64 b) {
    if (is_skippable(a) && is_skippable(b)) rwts.eras++;
    else if (redex_would_shrink(a, b)) redexes.fast.push_back({a, b});
    else redexes.slow.push_back({a, b});
  }
  void half_link_port_port(u64 a, u64 b) {
    if (ptag(a) == Var) w_set(paddr(a), b);
  }
  void half_link_wire_port(u64 ap, u64 aw, u64 bp) {
    if (ptag(ap) == Var) {
      u64 got;
      if (w_cas(paddr(ap), port_var(aw), bp, &got)) {
        free_wire(aw);
      } else {
        if (ptag(bp) == Var) {
          w_set(aw, port_red(paddr(bp)));
        } else if (is_principal(bp)) {
          w_set(aw, bp);
          resolve_redirect_pri(ap, aw, bp);
        } else {
          throw Panic(E_BAD_PAIR, "unreachable in half_link_wire_port");
        }
      }
    } else {
      free_wire(aw);
    }
  }
  // linker.rs:130-203
  void resolve_redirect_pri(u64 ap, u64 aw, u64 bp) {
    for (;;) {
      u64 tw = paddr(ap);
      u64 tp = w_load(tw);
      if (tp == P_LOCK) continue;
      if (ptag(tp) == Red) {
        free_wire(tw);
        ap = tp;
        continue;
      }
      if (ptag(tp) == Var) {
        if (w_cas(tw, tp, bp, nullptr)) {
          tw = paddr(tp);
          tp = w_load(tw);
          while (tp != P_LOCK && ptag(tp) == Red) {
            free_wire(tw);
            tw = paddr(tp);
            tp = w_load(tw);
          }
          return;
        }
        continue;
      }
      if (is_principal(tp) || tp == P_GONE) {
        u64 xw = aw < tw ? aw : tw;
        u64 yw = aw < tw ? tw : aw;
        u64 xp = w_swap(xw, P_GONE);
        if (xp != P_GONE) {
          u64 yp = w_swap(yw, P_GONE);
          redux(xp, yp);
          return;
        } else {
          free_wire(xw);
          while (!w_cas(yw, P_GONE, P_LOCK, nullptr)) {}
          free_wire(yw);
          return;
        }
      }
      throw Panic(E_BAD_PAIR, "unreachable in resolve_redirect_pri");
    }
  }
  // linker.rs:287-304
  void link_trg_port(u64 a, u64 b) {
    if (trg_is_wire(a)) link_wire_port(a, b);
    else link_port_port(a, b);
  }
  void link_trg(u64 a, u64 b) {
    bool aw = trg_is_wire(a), bw = trg_is_wire(b);
    if (aw && bw) link_wire_wire(a, b);
    else if (aw) link_wire_port(a, b);
    else if (bw) link_wire_port(b, a);
    else link_port_port(a, b);
  }

  // ---- interact.rs:6-44
  void interact(u64 a, u64 b) {
    u8 at = ptag(a), bt = ptag(b);
    if (at == Var || at == Red || bt == Var || bt == Red) throw Panic(E_BAD_PAIR, "not an active pair");
    bool a_nil = at == Ref || at == NumT, b_nil = bt == Ref || bt == NumT;
    if (at == Ref && (bt == Ref || bt == NumT) && !is_skippable(a)) return call(a, b);
    if ((at == Ref || at == NumT) && bt == Ref && !is_skippable(b)) return call(b, a);
    if (a_nil && b_nil) { rwts.eras++; return; }
    if (at == Ctr && bt == Switch && plab(a) != 0) return comm22(a, b);
    if (at == Switch && bt == Ctr && plab(b) != 0) return comm22(a, b);
    if ((at == Ctr && bt == Op) || (at == Op && bt == Ctr)) return comm22(a, b);
    if (at == Ctr && bt == Ctr && plab(a) != plab(b)) return comm22(a, b);
    if ((at == Switch && bt == Switch) || (at == Op && bt == Op) || (at == Ctr && bt == Ctr)) return anni2(a, b);
    if (at == Ref && bt == Ctr && plab(b) >= plab(a)) return comm02(a, b);
    if (at == Ctr && bt == Ref && plab(a) >= plab(b)) return comm02(b, a);
    if (at == NumT && bt == Ctr) return comm02(a, b);
    if (at == Ctr && bt == NumT) return comm02(b, a);
    if (at == Ref && a == P_ERA) return comm02(a, b);
    if (bt == Ref && b == P_ERA) return comm02(b, a);
    if (at == Ref) return call(a, b);
    if (bt == Ref) return call(b, a);
    if (at == Op && bt == NumT) return op_num(a, b);
    if (at == NumT && bt == Op) return op_num(b, a);
    if (at == Switch && bt == NumT) return switch_num(a, b);
    if (at == NumT && bt == Switch) return switch_num(b, a);
    throw Panic(E_BAD_PAIR, "unimplemented interaction");
  }
  // interact.rs:72-79
  void anni2(u64 a, u64 b) {
    rwts.anni++;
    u64 a1 = paddr(a), a2 = other_half(a1), b1 = paddr(b), b2 = other_half(b1);
    link_wire_wire(a1, b1);
    link_wire_wire(a2, b2);
  }
  // interact.rs:118-141
  void comm22(u64 a, u64 b) {
    rwts.comm++;
    u64 a1 = paddr(a), a2 = other_half(a1), b1 = paddr(b), b2 = other_half(b1);
    Created A1 = create_node(ptag(a), plab(a));
    Created A2 = create_node(ptag(a), plab(a));
    Created B1 = create_node(ptag(b), plab(b));
    Created B2 = create_node(ptag(b), plab(b));
    link_port_port(A1.p1, B1.p1);
    link_port_port(A1.p2, B2.p1);
    link_port_port(A2.p1, B1.p2);
    link_port_port(A2.p2, B2.p2);
    link_wire_port(a1, B1.p0);
    link_wire_port(a2, B2.p0);
    link_wire_port(b1, A1.p0);
    link_wire_port(b2, A2.p0);
  }
  // interact.rs:162-168
  void comm02(u64 a, u64 b) {
    rwts.comm++;
    u64 b1 = paddr(b), b2 = other_half(b1);
    link_wire_port(b1, a);
    link_wire_port(b2, a);
  }
  // interact.rs:201-223
  void switch_num(u64 a, u64 b) {
    rwts.oper++;
    u64 a1 = paddr(a), a2 = other_half(a1);
    Num num{u32(b)};
    u32 n = num.tag() == U24 ? num.get_u24() : 0;
    if (n == 0) {
      Created x = create_node(Ctr, 0);
      link_port_port(x.p2, P_ERA);
      link_wire_port(a2, x.p1);
      link_wire_port(a1, x.p0);
    } else {
      Created x = create_node(Ctr, 0);
      Created y = create_node(Ctr, 0);
      link_port_port(x.p1, P_ERA);
      link_port_port(x.p2, y.p0);
      link_port_port(y.p1, u64(Num::u24(n - 1).raw));
      link_wire_port(a2, y.p2);
      link_wire_port(a1, x.p0);
    }
  }
  // interact.rs:251-270
  void op_num(u64 a, u64 b) {
    u8 op = u8(plab(a));
    u64 a1 = paddr(a), a2 = other_half(a1);
    u64 t1 = w_load(a1);
    if (ptag(t1) == NumT) {
      rwts.oper++;
      half_free(a1);
      Num out = operate_binary(Num{u32(b)}, op, Num{u32(t1)});
      link_wire_port(a2, u64(out.raw));
    } else {
      Created x = create_node(Op, Sym);
      link_port_port(x.p1, u64(operate_unary(op, Num{u32(b)}).raw));
      link_wire_port(a2, x.p2);
      link_wire_port(a1, x.p0);
    }
  }

  // ---- def.rs:177-189
  void call(u64 port, u64 trg) {
    Def* def = port_def(port);
    if (ptag(trg) == Ctr && !def->labs.has(plab(trg))) return comm02(port, trg);
    rwts.dref++;
    if (def->kind == D_EXPAND) expand_call(def, trg);
    else if (def->kind == D_INERT) {  // pre_reduce.rs:96-101
      if (!captured) throw Panic(E_BAD_INPUT, "inert definition called outside pre-reduce");
      captured->push_back({port_ref(def), trg});
    } else interpreted_call(def, trg);
  }

  // ---- instruction.rs:403-500
  std::pair<u64, u64> do_ctr(Lab lab, u64 trg) {
    u64 port = trg_target(trg);
    if (ptag(port) == Ctr && plab(port) == lab) {
      free_trg(trg);
      rwts.anni++;
      u64 p1 = paddr(port);
      return {trg_wire(p1), trg_wire(other_half(p1))};
    }
    Created n = create_node(Ctr, lab);
    link_trg_port(trg, n.p0);
    return {n.p1, n.p2};
  }
  std::pair<u64, u64> do_op(u8 op, u64 trg) {
    u64 port = trg_target(trg);
    if (ptag(port) == NumT) {
      free_trg(trg);
      Created n = create_node(Op, Sym);
      w_set(paddr(n.p1), u64(operate_unary(op, Num{u32(port)}).raw));
      return {n.p0, n.p2};
    } else if (port == P_ERA) {
      free_trg(trg);
      return {P_ERA, P_ERA};
    }
    Created n = create_node(Op, op);
    link_trg_port(trg, n.p0);
    return {n.p1, n.p2};
  }
  u64 do_op_num(u8 op, u64 trg, Num rhs) {
    u64 port = trg_target(trg);
    if (ptag(port) == NumT) {
      rwts.oper++;
      free_trg(trg);
      return u64(operate_binary(Num{u32(port)}, op, rhs).raw);
    } else if (port == P_ERA) {
      free_trg(trg);
      return P_ERA;
    }
    Created n = create_node(Op, op);
    link_trg_port(trg, n.p0);
    w_set(paddr(n.p1), u64(rhs.raw));
    return n.p2;
  }
  std::pair<u64, u64> do_switch(u64 trg) {
    u64 port = trg_target(trg);
    if (ptag(port) == NumT) {
      rwts.oper++;
      free_trg(trg);
      Num num{u32(port)};
      u32 n = num.tag() == U24 ? num.get_u24() : 0;
      Created c1 = create_node(Ctr, 0);
      if (n == 0) {
        link_port_port(c1.p2, P_ERA);
        return {c1.p0, trg_wire(create_wire_to(c1.p1))};
      } else {
        Created c2 = create_node(Ctr, 0);
        link_port_port(c1.p1, P_ERA);
        link_port_port(c1.p2, c2.p0);
        link_port_port(c2.p1, u64(Num::u24(n - 1).raw));
        return {c1.p0, trg_wire(create_wire_to(c2.p2))};
      }
    } else if (port == P_ERA) {
      rwts.eras++;
      free_trg(trg);
      return {P_ERA, P_ERA};
    }
    Created m = create_node(Switch, 0);
    link_trg_port(trg, m.p0);
    return {m.p1, m.p2};
  }

  // ---- def.rs:217-289
  void interpreted_call(Def* def, u64 trg) {
    if (def->trgs >= trgs.size()) trgs.resize(def->trgs);
    u64* t = trgs.data();
    t[0] = trg_port(trg);
    for (const Instruction& i : def->instr) {
      switch (i.k) {
        case I_CONST: t[i.a] = trg_port(i.port); break;
        case I_LINK: link_trg(t[i.a], t[i.b]); break;
        case I_LINKCONST: link_trg_port(t[i.a], i.port); break;
        case I_CTR: { auto [x, y] = do_ctr(i.lab, t[i.a]); t[i.b] = x; t[i.c] = y; break; }
        case I_OP: { auto [x, y] = do_op(u8(i.lab), t[i.a]); t[i.b] = x; t[i.c] = y; break; }
        case I_OPNUM: t[i.c] = do_op_num(u8(i.lab), t[i.a], Num{u32(i.port)}); break;
        case I_SWITCH: { auto [x, y] = do_switch(t[i.a]); t[i.b] = x; t[i.c] = y; break; }
        case I_WIRES: {
          u64 a = alloc(), b = other_half(a);
          t[i.a] = port_var(a); t[i.b] = trg_wire(a); t[i.c] = port_var(b); t[i.d] = trg_wire(b);
          break;
        }
      }
    }
  }

  // ---- net.rs:63-108 (ExpandDef)
  static u64 new_expand(u64 out) {
    Def* d = new Def();
    d->labs = LabSet::all();
    d->kind = D_EXPAND;
    d->expand_out = out;
    return port_ref(d);
  }
  void expand() {
    auto [new_root, out_port] = create_wire();
    u64 old_root = root;
    root = new_root;
    link_wire_port(old_root, new_expand(out_port));
  }
  void expand_call(Def* def, u64 port) {
    if (ptag(port) == Ref && port != P_ERA) {
      Def* other = port_def(port);
      if (other->kind == D_EXPAND) {
        u64 a = def->expand_out, b = other->expand_out;
        delete def;
        delete other;
        return link_port_port(a, b);
      }
      return call(port, port_ref(def));
    }
    u64 out = def->expand_out;
    delete def;
    switch (ptag(port)) {
      case Red: throw Panic(E_BAD_PAIR, "unreachable in ExpandDef");
      case Ref: case NumT: case Var: return link_port_port(out, port);
      default: {
        u64 o1 = paddr(port), o2 = other_half(o1);
        Created n = create_node(ptag(port), plab(port));
        link_port_port(out, n.p0);
        link_wire_port(o1, new_expand(n.p1));
        link_wire_port(o2, new_expand(n.p2));
      }
    }
  }

  // ---- net.rs:36-60
  bool pop_redex(std::pair<u64, u64>& r) {
    if (order == 0) return redexes.pop(r);
    auto take = [&](std::vector<std::pair<u64, u64>>& v) {
      size_t k = order == 1 ? 0 : size_t(rng() % v.size());
      r = v[k];
      v[k] = v.back();
      v.pop_back();
    };
    if (!redexes.fast.empty()) { take(redexes.fast); return true; }
    if (!redexes.slow.empty()) { take(redexes.slow); return true; }
    return false;
  }
  bool reduce(size_t limit) {
    size_t count = 0;
    std::pair<u64, u64> r;
    while (pop_redex(r)) {
      interact(r.first, r.second);
      if (++count >= limit) return false;
    }
    return true;
  }
  void normal() {
    expand();
    while (!redexes.empty()) reduce(SIZE_MAX);
  }
  void boot(Def* def) { call(port_ref(def), port_var(root)); }  // net.rs:30-32
};

// net.rs:19-23
static std::unique_ptr<Net> net_new(Heap& h) {
  auto n = std::make_unique<Net>(h.base, h.nodes);
  n->root = n->alloc();
  return n;
}

// ---- parallel.rs:12-160
static void parallel_normal(Net& self, size_t tids_req) {
  self.expand();
  const size_t SHARE_LIMIT = 1 << 12;
  const size_t LOCAL_LIMIT = 1 << 18;
  size_t cores = tids_req ? tids_req : std::max(1u, std::thread::hardware_concurrency());
  size_t tlog2 = 0;
  while ((size_t(2) << tlog2) <= cores) tlog2++;
  size_t tids = size_t(1) << tlog2;

  std::atomic<u64> d_anni{0}, d_comm{0}, d_eras{0}, d_dref{0}, d_oper{0};
  std::vector<std::atomic<size_t>> rlens(tids);
  std::vector<std::atomic<u64>> share(SHARE_LIMIT * tids * 2);
  std::atomic<size_t> total{0};
  std::barrier<> barry{ptrdiff_t(tids)};

  // fork (parallel.rs:12-32)
  std::vector<std::pair<u64, u64>> all;
  all.insert(all.end(), self.redexes.fast.begin(), self.redexes.fast.end());
  all.insert(all.end(), self.redexes.slow.begin(), self.redexes.slow.end());
  self.redexes.fast.clear();
  self.redexes.slow.clear();
  size_t redexes_len = all.size(), taken = 0;
  std::vector<std::unique_ptr<Net>> nets;
  for (size_t tid = 0; tid < tids; tid++) {
    size_t heap_size = (self.heap_nodes / tids) & ~size_t(63);
    size_t heap_start = heap_size * tid;
    auto n = std::make_unique<Net>(self.heap_base + heap_start * 16, heap_size);
    n->root = self.root;
    n->next = self.next > heap_start ? self.next - heap_start : 0;
    n->head = 0;
    n->tid = tid;
    n->tids = tids;
    size_t count = redexes_len / (tids - tid);
    for (size_t k = 0; k < count && taken < redexes_len; k++, taken++) n->redux(all[taken].first, all[taken].second);
    nets.push_back(std::move(n));
  }

  std::atomic<int> failed{0};
  std::string fail_msg;
  int fail_code = 0;
  std::mutex fail_mu;

  auto worker = [&](size_t tid) {
    Net& net = *nets[tid];
    size_t tick = 0;
    auto count = [&]() -> size_t {
      barry.arrive_and_wait();
      total.store(0, std::memory_order_relaxed);
      barry.arrive_and_wait();
      rlens[tid].store(net.redexes.slow.size(), std::memory_order_relaxed);
      total.fetch_add(net.redexes.len(), std::memory_order_relaxed);
      barry.arrive_and_wait();
      return total.load(std::memory_order_relaxed);
    };
    auto split = [&](size_t plog2) {
      size_t side = (tid >> (plog2 - 1 - (tick % plog2))) & 1;
      size_t shift = (size_t(1) << (plog2 - 1)) >> (tick % plog2);
      size_t a_tid = tid;
      size_t b_tid = side == 1 ? a_tid - shift : a_tid + shift;
      size_t a_len = net.redexes.slow.size();
      size_t b_len = rlens[b_tid].load(std::memory_order_relaxed);
      size_t send = a_len > b_len ? (a_len - b_len) / 2 : 0;
      size_t recv = b_len > a_len ? (b_len - a_len) / 2 : 0;
      send = std::min(send, SHARE_LIMIT);
      recv = std::min(recv, SHARE_LIMIT);
      for (size_t i = 0; i < send; i++) {
        size_t init = a_len - send * 2;
        auto rdx0 = net.redexes.slow[init + i * 2];
        auto rdx1 = net.redexes.slow[init + i * 2 + 1];
        size_t t = (b_tid * SHARE_LIMIT + i) * 2;
        net.redexes.slow[init + i] = rdx0;
        share[t].store(rdx1.first, std::memory_order_relaxed);
        share[t + 1].store(rdx1.second, std::memory_order_relaxed);
      }
      net.redexes.slow.resize(a_len - send);
      barry.arrive_and_wait();
      for (size_t i = 0; i < recv; i++) {
        size_t t = (a_tid * SHARE_LIMIT + i) * 2;
        net.redexes.slow.push_back({share[t].load(std::memory_order_relaxed), share[t + 1].load(std::memory_order_relaxed)});
      }
    };
    // A panic in one thread would deadlock the barrier; the reference aborts
    // the process (Cargo.toml panic = "abort").  Here the panic is recorded
    // and the process aborts after printing it, like the reference.
    try {
      for (;;) {
        for (;;) {
          net.reduce(LOCAL_LIMIT);
          if (count() == 0) break;
          if (tlog2 > 0) split(tlog2);
          tick++;
        }
        if (count() == 0) break;
      }
    } catch (Panic& p) {
      fprintf(stderr, "thread '%zu' panicked: %s\n", tid, p.what());
      fflush(stderr);
      abort();
    }
    d_anni += net.rwts.anni; d_comm += net.rwts.comm; d_eras += net.rwts.eras;
    d_dref += net.rwts.dref; d_oper += net.rwts.oper;
  };
  if (tids == 1) {
    worker(0);
  } else {
    std::vector<std::thread> ths;
    for (size_t t = 0; t < tids; t++) ths.emplace_back(worker, t);
    for (auto& t : ths) t.join();
  }
  (void)failed; (void)fail_code;
  self.rwts.anni += d_anni; self.rwts.comm += d_comm; self.rwts.eras += d_eras;
  self.rwts.dref += d_dref; self.rwts.oper += d_oper;
}

// ===========================================================================
// host  (host/src/*.rs)
// ===========================================================================

// calc_labels.rs:78-194
struct LabelCalc {
  const Book& book;
  std::function<LabSet(const std::string&)> lookup;
  struct State { bool done; LabSet labs; size_t cycle; };
  std::map<std::string, State> labels;

  size_t visit_def(const std::string& key, std::optional<size_t> depth, LabSet* out) {
    auto it = labels.find(key);
    if (it == labels.end()) {
      labels[key] = State{false, {}, *depth};
      return calc_def(key, depth, out);
    }
    State& st = it->second;
    if (st.done) {
      if (out) out->unite(st.labs);
      return SIZE_MAX;
    }
    if (depth) return st.cycle;
    st = State{true, {}, 0};
    return calc_def(key, depth, out);
  }
  size_t calc_def(const std::string& key, std::optional<size_t> depth, LabSet* out) {
    LabSet labs;
    size_t head = visit_within_def(key, depth, &labs);
    if (out) out->unite(labs);
    if (depth && *depth > head) {
      labels[key] = State{false, {}, head};
    } else {
      labels[key] = State{true, labs, 0};
      if (depth && *depth == head) visit_within_def(key, std::nullopt, nullptr);
    }
    return head;
  }
  size_t visit_within_def(const std::string& key, std::optional<size_t> depth, LabSet* out) {
    const AstNet& def = book.nets.at(key);
    size_t head = visit_tree(def.root, depth, out);
    for (auto& r : def.redexes) {
      head = std::min(head, visit_tree(r.first, depth, out));
      head = std::min(head, visit_tree(r.second, depth, out));
    }
    return head;
  }
  size_t visit_tree(const Tree* t, std::optional<size_t> depth, LabSet* out) {
    if (t->kind == T_CTR && out) out->add(t->lab);
    if (t->kind == T_REF) {
      if (book.nets.count(t->name)) {
        std::optional<size_t> d = depth ? std::optional<size_t>(*depth + 1) : std::nullopt;
        return visit_def(t->name, d, out);
      }
      if (out) out->unite(lookup(t->name));
    }
    size_t r = SIZE_MAX;
    if (t->p1) r = std::min(r, visit_tree(t->p1, depth, out));
    if (t->p2) r = std::min(r, visit_tree(t->p2, depth, out));
    return r;
  }
};

static std::map<std::string, LabSet> calculate_label_sets(const Book& book,
                                                          std::function<LabSet(const std::string&)> lookup) {
  LabelCalc c{book, std::move(lookup), {}};
  for (auto& [name, _] : book.nets) c.visit_def(name, 0, nullptr);
  std::map<std::string, LabSet> out;
  for (auto& [name, st] : c.labels) {
    if (!st.done) throw Panic(E_BAD_INPUT, "label calculation did not converge");
    out[name] = st.labs;
  }
  return out;
}

// host.rs:17-85
struct Host {
  std::map<std::string, std::unique_ptr<Def>> defs;
  std::unordered_map<u64, std::string> back;
  Book book;  // keeps the trees alive

  void insert_def(const std::string& name, std::unique_ptr<Def> d) {
    back[paddr(port_ref(d.get()))] = name;
    defs[name] = std::move(d);
  }
  // host.rs:34-73.  With `inert_missing` (insert_book_with_default as
  // pre_reduce.rs:41 calls it) a reference the Book lacks becomes an inert def
  // with LabSet::ALL.
  void insert_book(const Book& b, bool inert_missing = false) {
    auto sets = calculate_label_sets(b, [&](const std::string& name) -> LabSet {
      auto it = defs.find(name);
      if (it != defs.end()) return it->second->labs;
      if (!inert_missing) throw Panic(E_BAD_INPUT, "Found reference \"" + name + "\", which is not in the book!");
      auto d = std::make_unique<Def>();
      d->labs = LabSet::all();
      d->kind = D_INERT;
      insert_def(name, std::move(d));
      return defs[name]->labs;
    });
    for (auto& [name, labs] : sets) {
      auto d = std::make_unique<Def>();
      d->labs = labs;
      insert_def(name, std::move(d));
    }
    for (auto& [name, net] : b.nets) encode_def(net, *defs[name]);
  }

  // ---- encode.rs (State + Encoder impls)
  template <class E> struct State {
    Host& host;
    E& enc;
    std::map<std::string, typename E::Trg> scope;
    void finish() {
      if (!scope.empty()) throw Panic(E_BAD_INPUT, "unbound variables: " + scope.begin()->first);
    }
    u64 ref_port(const std::string& name) {
      auto it = host.defs.find(name);
      if (it == host.defs.end()) throw Panic(E_BAD_INPUT, "Found reference \"" + name + "\", which is not in the book!");
      return port_ref(it->second.get());
    }
    void visit_net(const AstNet& net, typename E::Trg trg) {  // encode.rs:133-136
      visit_tree(net.root, trg);
      for (auto& r : net.redexes) visit_redex(r.first, r.second);
    }
    void visit_redex(const Tree* a, const Tree* b) {  // encode.rs:137-152
      u64 port;
      const Tree* tree;
      if (a->kind == T_ERA) { port = P_ERA; tree = b; }
      else if (b->kind == T_ERA) { port = P_ERA; tree = a; }
      else if (a->kind == T_REF) { port = ref_port(a->name); tree = b; }
      else if (b->kind == T_REF) { port = ref_port(b->name); tree = a; }
      else if (a->kind == T_NUM) { port = u64(a->num.raw); tree = b; }
      else if (b->kind == T_NUM) { port = u64(b->num.raw); tree = a; }
      else {
        auto [av, aw, bv, bw] = enc.wires();
        visit_tree(a, av);
        visit_tree(b, bv);
        enc.link(aw, bw);
        return;
      }
      auto trg = enc.make_const(port);
      visit_tree(tree, trg);
    }
    void visit_tree(const Tree* t, typename E::Trg trg) {  // encode.rs:153-189
      switch (t->kind) {
        case T_ERA: enc.link_const(trg, P_ERA); return;
        case T_NUM: enc.link_const(trg, u64(t->num.raw)); return;
        case T_REF: enc.link_const(trg, ref_port(t->name)); return;
        case T_CTR: {
          auto [l, r] = enc.ctr(t->lab, trg);
          visit_tree(t->p1, l);
          visit_tree(t->p2, r);
          return;
        }
        case T_OP: {
          u8 op = Sym;
          const Tree* rhs = t->p1;
          const Tree* out = t->p2;
          if (t->p1->kind == T_NUM && t->p2->kind == T_OP && t->p1->num.tag() == Sym) {
            op = t->p1->num.get_sym();
            rhs = t->p2->p1;
            out = t->p2->p2;
          }
          if (rhs->kind == T_NUM) {
            auto o = enc.op_num(op, trg, rhs->num);
            visit_tree(out, o);
          } else {
            auto [r, o] = enc.op(op, trg);
            visit_tree(rhs, r);
            visit_tree(out, o);
          }
          return;
        }
        case T_SWITCH: {
          auto [a, o] = enc.sw(trg);
          visit_tree(t->p1, a);
          visit_tree(t->p2, o);
          return;
        }
        case T_VAR: {
          auto it = scope.find(t->name);
          if (it != scope.end()) {
            auto other = it->second;
            scope.erase(it);
            enc.link(other, trg);
          } else {
            scope.emplace(t->name, trg);
          }
          return;
        }
      }
    }
  };

  // Encoder for InterpretedDef: encode.rs:204-248
  struct DefEncoder {
    using Trg = u32;
    Def& d;
    u32 new_trg() { return u32(d.trgs++); }
    void link_const(u32 trg, u64 port) { d.instr.push_back({I_LINKCONST, 0, trg, 0, 0, 0, port}); }
    void link(u32 a, u32 b) { d.instr.push_back({I_LINK, 0, a, b, 0, 0, 0}); }
    u32 make_const(u64 port) { u32 t = new_trg(); d.instr.push_back({I_CONST, 0, t, 0, 0, 0, port}); return t; }
    std::pair<u32, u32> ctr(Lab lab, u32 trg) { u32 p1 = new_trg(), p2 = new_trg(); d.instr.push_back({I_CTR, lab, trg, p1, p2, 0, 0}); return {p1, p2}; }
    std::pair<u32, u32> op(u8 op, u32 trg) { u32 r = new_trg(), o = new_trg(); d.instr.push_back({I_OP, op, trg, r, o, 0, 0}); return {r, o}; }
    u32 op_num(u8 op, u32 trg, Num rhs) { u32 o = new_trg(); d.instr.push_back({I_OPNUM, op, trg, 0, o, 0, u64(rhs.raw)}); return o; }
    std::pair<u32, u32> sw(u32 trg) { u32 a = new_trg(), o = new_trg(); d.instr.push_back({I_SWITCH, 0, trg, a, o, 0, 0}); return {a, o}; }
    std::tuple<u32, u32, u32, u32> wires() {
      u32 av = new_trg(), aw = new_trg(), bv = new_trg(), bw = new_trg();
      d.instr.push_back({I_WIRES, 0, av, aw, bv, bw, 0});
      return {av, aw, bv, bw};
    }
  };
  // Encoder for Net: encode.rs:250-277
  struct NetEncoder {
    using Trg = u64;
    Net& n;
    void link_const(u64 trg, u64 port) { n.link_trg_port(trg, port); }
    void link(u64 a, u64 b) { n.link_trg(a, b); }
    u64 make_const(u64 port) { return port; }
    std::pair<u64, u64> ctr(Lab lab, u64 trg) { return n.do_ctr(lab, trg); }
    std::pair<u64, u64> op(u8 op, u64 trg) { return n.do_op(op, trg); }
    u64 op_num(u8 op, u64 trg, Num rhs) { return n.do_op_num(op, trg, rhs); }
    std::pair<u64, u64> sw(u64 trg) { return n.do_switch(trg); }
    std::tuple<u64, u64, u64, u64> wires() {
      u64 a = n.alloc(), b = other_half(a);
      return {port_var(a), trg_wire(a), port_var(b), trg_wire(b)};
    }
  };

  void encode_def(const AstNet& net, Def& d) {  // encode.rs:98-104
    d.instr.clear();
    d.trgs = 1;
    DefEncoder e{d};
    State<DefEncoder> st{*this, e, {}};
    st.visit_net(net, 0);
    st.finish();
  }
  void encode_net(Net& n, u64 trg, const AstNet& net) {  // encode.rs:116-120
    NetEncoder e{n};
    State<NetEncoder> st{*this, e, {}};
    st.visit_net(net, trg);
    st.finish();
  }

  // ---- readback.rs:23-87.  With `resolve` set, Red redirect chains left by
  // concurrent linking are followed to the live endpoint (the reference's
  // readback marks this as a todo and only meets chain-free nets in its
  // snapshots); without it the key is the reference's min(wire, port).
  struct Readback {
    Host& host;
    Arena& arena;
    bool resolve;
    u64 heap_lo, heap_hi;
    std::map<u64, size_t> vars;
    size_t var_id = 0;
    Tree* read_wire(u64 w) { return read_port(w_load(w), w); }
    Tree* read_port(u64 port, u64 wire) {
      switch (ptag(port)) {
        case Var: case Red: {
          u64 end = paddr(port);
          // Follow only genuine redirects inside the heap: a vicious circle
          // can leave sentinels (FREE/LOCK) or free-list links here.
          auto in_heap = [&](u64 p) {
            return (p >> 48) == 0 && paddr(p) >= heap_lo && paddr(p) < heap_hi;
          };
          if (resolve && in_heap(port)) {
            for (size_t guard = 0; guard < (size_t(1) << 40); guard++) {
              u64 t = w_load(end);
              if (ptag(t) != Red || !in_heap(t)) break;
              end = paddr(t);
            }
          }
          u64 key = std::min(wire, end);
          Tree* t = arena.make(T_VAR);
          auto it = vars.find(key);
          if (it != vars.end()) { t->name = create_var(it->second); vars.erase(it); }
          else { vars[key] = var_id; t->name = create_var(var_id++); }
          return t;
        }
        case Ref: {
          if (port == P_ERA) return arena.make(T_ERA);
          Tree* t = arena.make(T_REF);
          auto it = host.back.find(paddr(port));
          t->name = it == host.back.end() ? std::string("<expand>") : it->second;
          return t;
        }
        case NumT: { Tree* t = arena.make(T_NUM); t->num = Num{u32(port)}; return t; }
        case Op: {
          u8 op = u8(plab(port));
          u64 p1 = paddr(port);
          Tree* node = arena.make(T_OP);
          node->p1 = read_wire(p1);
          node->p2 = read_wire(other_half(p1));
          if (op == Sym) return node;
          Tree* outer = arena.make(T_OP);
          outer->p1 = arena.make(T_NUM);
          outer->p1->num = Num::sym(op);
          outer->p2 = node;
          return outer;
        }
        case Ctr: {
          u64 p1 = paddr(port);
          Tree* t = arena.make(T_CTR);
          t->lab = plab(port);
          t->p1 = read_wire(p1);
          t->p2 = read_wire(other_half(p1));
          return t;
        }
        case Switch: {
          u64 p1 = paddr(port);
          Tree* t = arena.make(T_SWITCH);
          t->p1 = read_wire(p1);
          t->p2 = read_wire(other_half(p1));
          return t;
        }
      }
      throw Panic(E_BAD_PAIR, "bad port in readback");
    }
  };
  AstNet readback(Net& n, Arena& arena, bool resolve) {
    Readback r{*this, arena, resolve, n.heap_base, n.heap_base + u64(n.heap_nodes) * 16, {}, 0};
    AstNet out;
    out.root = r.read_wire(n.root);
    for (auto* q : {&n.redexes.fast, &n.redexes.slow})
      for (auto& [a, b] : *q) out.redexes.push_back({r.read_port(a, 0), r.read_port(b, 0)});
    return out;
  }
};

// Runs `f` on a thread with a large stack (the reference grows its stack with
// `stacker` for deep trees: util/src/maybe_grow.rs:3-5).
template <class F> static void with_big_stack(F f) {
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, size_t(4) << 30);
  struct Box { F* f; std::exception_ptr e; };
  Box box{&f, nullptr};
  pthread_t th;
  auto tramp = [](void* p) -> void* {
    Box* b = static_cast<Box*>(p);
    try { (*b->f)(); } catch (...) { b->e = std::current_exception(); }
    return nullptr;
  };
  if (pthread_create(&th, &attr, tramp, &box) != 0) { f(); return; }
  pthread_join(th, nullptr);
  pthread_attr_destroy(&attr);
  if (box.e) std::rethrow_exception(box.e);
}

static std::string pretty_num(u64 n) {  // util/src/pretty_num.rs:4
  std::string s = std::to_string(n), o;
  int lead = int(s.size()) % 3;
  for (size_t k = 0; k < s.size(); k++) {
    if (k != 0 && (int(k) - lead) % 3 == 0) o += '_';
    o += s[k];
  }
  return o;
}
static std::string rewrites_to_string(const Rewrites& r) {  // runtime.rs:131-141
  char buf[512];
  snprintf(buf, sizeof buf, "RWTS   : %15s\n- ANNI : %15s\n- COMM : %15s\n- ERAS : %15s\n- DREF : %15s\n- OPER : %15s\n",
           pretty_num(r.total()).c_str(), pretty_num(r.anni).c_str(), pretty_num(r.comm).c_str(),
           pretty_num(r.eras).c_str(), pretty_num(r.dref).c_str(), pretty_num(r.oper).c_str());
  return buf;
}

// util/src/parse_abbrev_number.rs:5-19
static u64 parse_abbrev_number(const std::string& arg) {
  if (arg.empty()) throw Panic(E_BAD_INPUT, "Mem size argument is empty");
  char last = char(tolower((unsigned char)arg.back()));
  u64 scale = 1;
  std::string base = arg;
  if (last == 'k') scale = 1ull << 10;
  else if (last == 'm') scale = 1ull << 20;
  else if (last == 'g') scale = 1ull << 30;
  else if (last == 't') scale = 1ull << 40;
  if (scale != 1) base = arg.substr(0, arg.size() - 1);
  return Parser::parse_int(base) * scale;
}

// Default heap for the oracle: a large no-reserve mapping (the reference
// tries 1 TiB and halves: allocator.rs:22-38).
static size_t default_heap_bytes() { return size_t(64) << 30; }

struct RunResult {
  std::string text;
  Rewrites rw;
  double seconds = 0;
};

// mode: 0 = Net::normal (single thread), 1 = parallel_normal,
//       2 = normal with FIFO redex order, 3 = normal with seeded random order.
static void run_normal(Net& net, int mode, int threads, u64 seed) {
  if (mode == 1) { parallel_normal(net, size_t(threads)); return; }
  net.order = mode == 2 ? 1 : mode == 3 ? 2 : 0;
  net.rng.seed(seed);
  net.normal();
}

// tests/tests.rs:28-35 (boot the entry def, normalise, read back)
static RunResult run_book(const std::string& text, const std::string& entry, int mode, int threads, u64 seed,
                          size_t heap_bytes, bool resolve) {
  RunResult rr;
  with_big_stack([&] {
    Host host;
    host.book = parse_book(text);
    host.insert_book(host.book);
    auto it = host.defs.find(entry);
    if (it == host.defs.end()) throw Panic(E_BAD_INPUT, "entry point not found: " + entry);
    Heap heap(heap_bytes ? heap_bytes : default_heap_bytes());
    auto net = net_new(heap);
    net->boot(it->second.get());
    auto t0 = std::chrono::steady_clock::now();
    run_normal(*net, mode, threads, seed);
    auto t1 = std::chrono::steady_clock::now();
    rr.seconds = std::chrono::duration<double>(t1 - t0).count();
    Arena arena;
    rr.text = net_to_string(host.readback(*net, arena, resolve));
    rr.rw = net->rwts;
  });
  return rr;
}

// src/main.rs:176-193 (encode an expression net, normalise, read back)
static RunResult run_expr(Host& host, const AstNet& expr, int mode, int threads, u64 seed, size_t heap_bytes,
                          bool resolve) {
  RunResult rr;
  Heap heap(heap_bytes ? heap_bytes : default_heap_bytes());
  auto net = net_new(heap);
  host.encode_net(*net, port_var(net->root), expr);
  auto t0 = std::chrono::steady_clock::now();
  run_normal(*net, mode, threads, seed);
  auto t1 = std::chrono::steady_clock::now();
  rr.seconds = std::chrono::duration<double>(t1 - t0).count();
  Arena arena;
  rr.text = net_to_string(host.readback(*net, arena, resolve));
  rr.rw = net->rwts;
  return rr;
}

// transform/src/pre_reduce.rs:38-74,136-164.  Every def of the Book not
// skipped is visited in byte order of names; a def first pre-reduces the defs
// its (original) net references, depth first (a def met again while still on
// the path is left as it is: the "Cycled" state).  Then it is booted in a
// fresh Net on the shared heap without the expansion agent and reduced with
// `Net::reduce(max_rwts)`; redexes captured by inert defs go back into the
// net's redex queue; the read-back net replaces the def's instructions at once
// (so later defs call the reduced version) and, at the end, its text in the
// Book.  Label sets stay those of the original Book.
struct PreReducer {
  Host& host;
  Heap& heap;
  const std::set<std::string>& skip;
  u64 max_rwts;
  Arena arena;
  std::vector<std::pair<u64, u64>> captured;
  std::map<std::string, int> seen;  // 0: on the path (Cycled), 1: reduced
  std::map<std::string, std::pair<AstNet, bool>> reduced;  // net, reached normal form
  Rewrites rw;

  void visit_tree(const Tree* t) {  // pre_reduce.rs:122-129
    if (t->kind == T_REF) pre_reduce(t->name);
    if (t->p1) visit_tree(t->p1);
    if (t->p2) visit_tree(t->p2);
  }
  void pre_reduce(const std::string& name) {  // pre_reduce.rs:137-164
    if (seen.count(name) || skip.count(name) || !host.book.nets.count(name)) return;
    seen[name] = 0;
    const AstNet& src = host.book.nets.at(name);
    visit_tree(src.root);
    for (auto& r : src.redexes) {
      visit_tree(r.first);
      visit_tree(r.second);
    }
    auto rt = net_new(heap);
    rt->captured = &captured;
    rt->boot(host.defs.at(name).get());
    bool normal = rt->reduce(max_rwts > u64(SIZE_MAX) ? SIZE_MAX : size_t(max_rwts));
    rw.anni += rt->rwts.anni; rw.comm += rt->rwts.comm; rw.eras += rt->rwts.eras;
    rw.dref += rt->rwts.dref; rw.oper += rt->rwts.oper;
    for (auto& [a, b] : captured) rt->redux(a, b);
    captured.clear();
    AstNet net = host.readback(*rt, arena, false);
    host.encode_def(net, *host.defs.at(name));
    seen[name] = 1;
    reduced[name] = {net, normal};
  }
};

struct PreReduceResult {
  std::string text;
  Rewrites rw;
  std::vector<std::string> not_normal;
};

static PreReduceResult pre_reduce_book(const std::string& text, const std::set<std::string>& skip, u64 max_rwts,
                                       size_t heap_bytes) {
  PreReduceResult out;
  with_big_stack([&] {
    Host host;
    host.book = parse_book(text);
    host.insert_book(host.book, true);
    Heap heap(heap_bytes ? heap_bytes : default_heap_bytes());
    PreReducer p{host, heap, skip, max_rwts, {}, {}, {}, {}, {}};
    for (auto& [name, _] : host.book.nets) p.pre_reduce(name);
    for (auto& [name, st] : p.reduced) {  // pre_reduce.rs:60-67
      host.book.nets[name] = st.first;
      if (!st.second) out.not_normal.push_back(name);
    }
    out.rw = p.rw;
    out.text = book_to_string(host.book);
  });
  return out;
}

}  // namespace hvo

// ===========================================================================
// C ABI for the Python tests (ctypes).  Every call returns 0 or an error code;
// text outputs are malloc'd and released with hvo_free.
// ===========================================================================
using namespace hvo;

static thread_local std::string g_err;
static char* dupstr(const std::string& s) {
  char* p = static_cast<char*>(malloc(s.size() + 1));
  memcpy(p, s.data(), s.size());
  p[s.size()] = 0;
  return p;
}
template <class F> static int guarded(F f) {
  try {
    f();
    return 0;
  } catch (Panic& p) {
    g_err = p.what();
    return p.code;
  } catch (std::exception& e) {
    g_err = e.what();
    return E_BAD_INPUT;
  }
}

extern "C" {

const char* hvo_last_error(void) { return g_err.c_str(); }
void hvo_free(char* p) { free(p); }

// Boot `entry` of the book and normalise it.  rw[0..5] = anni, comm, eras,
// dref, oper.
int hvo_run_book(const char* text, const char* entry, int mode, int threads, uint64_t seed, uint64_t heap_bytes,
                 int resolve, char** out_text, uint64_t* rw, double* seconds) {
  return guarded([&] {
    RunResult r = run_book(text, entry, mode, threads, seed, heap_bytes, resolve != 0);
    *out_text = dupstr(r.text);
    rw[0] = r.rw.anni; rw[1] = r.rw.comm; rw[2] = r.rw.eras; rw[3] = r.rw.dref; rw[4] = r.rw.oper;
    if (seconds) *seconds = r.seconds;
  });
}

// Encode an expression net against a book and normalise it
// (src/main.rs:176-193; tests/cli.rs:205-251).
int hvo_run_expr(const char* book_text, const char* expr_text, int mode, int threads, uint64_t heap_bytes,
                 int resolve, char** out_text, uint64_t* rw) {
  return guarded([&] {
    with_big_stack([&] {
      Host host;
      host.book = parse_book(book_text);
      host.insert_book(host.book);
      Arena arena;
      AstNet expr = parse_net(expr_text, arena);
      RunResult r = run_expr(host, expr, mode, threads, 0, heap_bytes, resolve != 0);
      *out_text = dupstr(r.text);
      rw[0] = r.rw.anni; rw[1] = r.rw.comm; rw[2] = r.rw.eras; rw[3] = r.rw.dref; rw[4] = r.rw.oper;
    });
  });
}

// tests/cli.rs:205-251: apply arguments to a net with Net::apply_tree, then
// encode, normal() and read back.  `args` is '\n'-separated.
int hvo_eval_with_args(const char* fun, const char* args, uint64_t heap_bytes, char** out_text) {
  return guarded([&] {
    with_big_stack([&] {
      Arena arena;
      AstNet net = parse_net(fun, arena);
      std::string a = args;
      size_t s = 0;
      while (s < a.size()) {
        size_t e = a.find('\n', s);
        if (e == std::string::npos) e = a.size();
        if (e > s) apply_tree(net, parse_tree(a.substr(s, e - s), arena), arena);
        s = e + 1;
      }
      Host host;
      RunResult r = run_expr(host, net, 0, 1, 0, heap_bytes, true);
      *out_text = dupstr(r.text);
    });
  });
}

// The label sets of every def (host/src/calc_labels.rs:78), one line each:
// "name min_safe lab lab ...".
int hvo_label_sets(const char* text, char** out_text) {
  return guarded([&] {
    with_big_stack([&] {
      Book b = parse_book(text);
      auto sets = calculate_label_sets(b, [](const std::string&) -> LabSet {
        throw Panic(E_BAD_INPUT, "unknown reference");
      });
      std::string o;
      for (auto& [name, ls] : sets) {
        o += name + " " + std::to_string(ls.min_safe);
        for (u32 l = 0; l < 65536; l++)
          if (ls.has(Lab(l))) o += " " + std::to_string(l);
        o += "\n";
      }
      *out_text = dupstr(o);
    });
  });
}

// tests/lists.rs:8-27: `book[def].apply_tree(arg)`, returning the new book
// text (printed with ast/src/ast.rs Display, which parses back identically).
int hvo_book_apply(const char* text, const char* def_name, const char* arg_tree, char** out_text) {
  return guarded([&] {
    with_big_stack([&] {
      Book b = parse_book(text);
      auto it = b.nets.find(def_name);
      if (it == b.nets.end()) throw Panic(E_BAD_INPUT, std::string("no def ") + def_name);
      apply_tree(it->second, parse_tree(arg_tree, *b.arena), *b.arena);
      *out_text = dupstr(book_to_string(b));
    });
  });
}

// Parse and re-print a book (ast/src/parser.rs + ast/src/ast.rs Display).
int hvo_book_roundtrip(const char* text, char** out_text) {
  return guarded([&] {
    with_big_stack([&] { *out_text = dupstr(book_to_string(parse_book(text))); });
  });
}

// Book::pre_reduce (transform/src/pre_reduce.rs:27-74): `skip` holds the
// '\n'-separated names not to pre-reduce.  Returns the pre-reduced Book's text
// (ast.rs Display), rw[0..5] and the '\n'-separated names of the defs whose
// reduction stopped at `max_rwts`.
int hvo_pre_reduce(const char* text, const char* skip, uint64_t max_rwts, uint64_t heap_bytes, char** out_text,
                   uint64_t* rw, char** out_not_normal) {
  return guarded([&] {
    std::set<std::string> sk;
    std::string a = skip ? skip : "";
    size_t s = 0;
    while (s < a.size()) {
      size_t e = a.find('\n', s);
      if (e == std::string::npos) e = a.size();
      if (e > s) sk.insert(a.substr(s, e - s));
      s = e + 1;
    }
    PreReduceResult r = pre_reduce_book(text, sk, max_rwts, heap_bytes);
    *out_text = dupstr(r.text);
    rw[0] = r.rw.anni; rw[1] = r.rw.comm; rw[2] = r.rw.eras; rw[3] = r.rw.dref; rw[4] = r.rw.oper;
    std::string nn;
    for (auto& n : r.not_normal) nn += n + "\n";
    *out_not_normal = dupstr(nn);
  });
}

// num: operate_binary(a, op, b) -> raw; 3 on a panic (div by zero).
int hvo_num_binary(uint32_t a, uint32_t op, uint32_t b, uint32_t* out) {
  return guarded([&] { *out = operate_binary(Num{a}, u8(op), Num{b}).raw; });
}
uint32_t hvo_num_unary(uint32_t op, uint32_t a) { return operate_unary(u8(op), Num{a}).raw; }
int hvo_num_parse(const char* text, uint32_t* out) {
  return guarded([&] {
    Arena arena;
    Tree* t = parse_tree(text, arena);
    if (t->kind != T_NUM) throw Panic(E_BAD_INPUT, "not a number");
    *out = t->num.raw;
  });
}
int hvo_num_print(uint32_t raw, char** out_text) {
  return guarded([&] { *out_text = dupstr(num_to_string(Num{raw})); });
}
uint32_t hvo_num_f24(float v) { return Num::f24(v).raw; }

}  // extern "C"

// ===========================================================================
// CLI (src/main.rs:32-204; src/args.rs).  Supports `run` and `reduce`.
// ===========================================================================
#ifdef HVO_MAIN
static void usage() {
  fprintf(stderr, "usage: hvm64-oracle run FILE [ARGS..] [-e ENTRY] [-m MEM] [-1] [-s] [-t THREADS]\n"
                  "       hvm64-oracle reduce [FILES..] [-m MEM] [-1] [-s] [-t THREADS] -- EXPRS..\n");
}
int main(int argc, char** argv) {
  if (argc < 2) { usage(); return 2; }
  std::string mode = argv[1];
  std::vector<std::string> files, args, exprs;
  std::string entry = "main";
  size_t mem = 0;
  bool single = false, stats = false, after_dd = false;
  int threads = 0;
  for (int k = 2; k < argc; k++) {
    std::string a = argv[k];
    if (after_dd) { exprs.push_back(a); continue; }
    if (a == "--") { after_dd = true; continue; }
    if (a == "-1" || a == "--single") single = true;
    else if (a == "-s" || a == "--stats") stats = true;
    else if ((a == "-m" || a == "--memory") && k + 1 < argc) mem = parse_abbrev_number(argv[++k]);
    else if (a == "-e" && k + 1 < argc) entry = argv[++k];
    else if (a == "-t" && k + 1 < argc) threads = atoi(argv[++k]);
    else if (mode == "run" && files.empty()) files.push_back(a);
    else if (mode == "run") args.push_back(a);
    else files.push_back(a);
  }
  int rc = 0;
  try {
    with_big_stack([&] {
      Host host;
      Book book;
      std::vector<std::shared_ptr<Arena>> keep;  // every file's trees stay alive
      for (auto& f : files) {
        FILE* fp = fopen(f.c_str(), "rb");
        if (!fp) {
          fprintf(stderr, "Input file \"%s\" not found\n", f.c_str());
          exit(1);
        }
        std::string s;
        char buf[1 << 16];
        size_t n;
        while ((n = fread(buf, 1, sizeof buf, fp)) > 0) s.append(buf, n);
        fclose(fp);
        Book b = parse_book(s);
        for (auto& [k, v] : b.nets) book.nets[k] = v;
        keep.push_back(b.arena);
      }
      host.insert_book(book);
      std::vector<AstNet> nets;
      Arena arena;
      if (mode == "run") {
        AstNet net;
        net.root = arena.make(T_REF);
        net.root->name = entry;
        for (auto& a : args) {
          AstNet an = parse_net(a, arena);
          for (auto& r : an.redexes) net.redexes.push_back(r);
          apply_tree(net, an.root, arena);
        }
        nets.push_back(net);
      } else {
        for (auto& e : exprs) nets.push_back(parse_net(e, arena));
      }
      for (auto& n : nets) {
        RunResult r = run_expr(host, n, single ? 0 : 1, threads, 0, mem, true);
        printf("%s\n", r.text.c_str());
        fflush(stdout);
        if (stats) {
          fprintf(stderr, "%s", rewrites_to_string(r.rw).c_str());
          fprintf(stderr, "TIME   : %.3fs\n", r.seconds);
          double ms = std::floor(r.seconds * 1000.0);
          fprintf(stderr, "RPS    : %.3f M\n", double(r.rw.total()) / ms / 1000.0);
        }
      }
    });
  } catch (Panic& p) {
    fprintf(stderr, "error: %s\n", p.what());
    rc = 101;
  }
  return rc;
}
#endif
