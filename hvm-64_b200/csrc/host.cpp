// Host side of the B200 reducer (see host.hpp).
#include "host.hpp"

#include <pthread.h>

#include <algorithm>
#include <atomic>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <optional>
#include <set>
#include <unordered_map>

#include "hvm64.h"

namespace hvm {

Tree* Arena::make(TreeKind k) {
  nodes.emplace_back();
  nodes.back().kind = k;
  return &nodes.back();
}

// ===========================================================================
// Numbers: literal parsing helpers and Display (num/src/num.rs:287-305)
// ===========================================================================
static const char* const NUMTAG_STR[NT_COUNT] = {
  "u24", "i24", "f24", " ", "+", "-", ":-", "*", "/", ":/", "%", ":%",
  "&", "|", "^", "<<", ":<<", ">>", ":>>", "=", "!", "<", ">"};

// Rust `{:?}` for a finite non-zero-or-zero f32: shortest round-trip digits,
// exponent form when |v| < 1e-4 or |v| >= 1e16.
static std::string debug_f32(float v) {
  if (v == 0.0f) return std::signbit(v) ? "-0.0" : "0.0";
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, std::fabs(v), std::chars_format::scientific);
  std::string s(buf, r.ptr);
  size_t e = s.find('e');
  int exp10 = atoi(s.c_str() + e + 1);
  std::string digits;
  for (size_t k = 0; k < e; k++)
    if (s[k] != '.') digits += s[k];
  float av = std::fabs(v);
  std::string out;
  if (av >= 1e-4f && av < 1e16f) {
    int n = int(digits.size()), point = exp10 + 1;
    if (point <= 0) out = "0." + std::string(size_t(-point), '0') + digits;
    else if (point < n) out = digits.substr(0, size_t(point)) + "." + digits.substr(size_t(point));
    else out = digits + std::string(size_t(point - n), '0') + ".0";
  } else {
    out = digits.substr(0, 1);
    if (digits.size() > 1) out += "." + digits.substr(1);
    out += "e" + std::to_string(exp10);
  }
  return (v < 0 ? "-" : "") + out;
}

std::string num_to_string(uint32_t n) {
  uint32_t t = num_tag(n);
  switch (t) {
    case NT_SYM: {
      uint32_t s = num_payload(n) & 0xff;
      return std::string("[") + (s < NT_COUNT ? NUMTAG_STR[s] : "?") + "]";
    }
    case NT_U24: return std::to_string(num_payload(n));
    case NT_I24: {
      int32_t v = num_get_i24(n);
      return (v >= 0 ? "+" : "") + std::to_string(v);
    }
    case NT_F24: {
      float f = num_get_f24(n);
      if (std::isinf(f)) return f > 0 ? "+inf" : "-inf";
      if (std::isnan(f)) return "+NaN";
      return debug_f32(f);
    }
    default:
      return std::string("[") + (t < NT_COUNT ? NUMTAG_STR[t] : "?") + std::to_string(num_payload(n)) + "]";
  }
}

// ===========================================================================
// Parser (ast/src/parser.rs:300-483).  Trivia: ASCII whitespace and `//`
// comments.
// ===========================================================================
namespace {
struct Parser {
  const std::string& in;
  size_t i = 0;
  Arena& arena;
  Parser(const std::string& s, Arena& a) : in(s), arena(a) {}

  [[noreturn]] void fail(const std::string& what) {
    throw Error(HVM64_ERR_BAD_INPUT, "Parsing error: expected " + what + " at byte " + std::to_string(i));
  }
  int peek() const { return i < in.size() ? (unsigned char)in[i] : -1; }
  void skip_trivia() {
    while (i < in.size()) {
      char c = in[i];
      if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f') { i++; continue; }
      if (c == '/' && in.compare(i, 2, "//") == 0) {
        while (i < in.size() && in[i] != '\n') i++;
        if (i < in.size()) i++;
        continue;
      }
      return;
    }
  }
  bool eat(const char* text) {
    skip_trivia();
    size_t n = strlen(text);
    if (in.compare(i, n, text) == 0) { i += n; return true; }
    return false;
  }
  void need(const char* text) {
    if (!eat(text)) fail(std::string("'") + text + "'");
  }
  template <class F> std::string span(F f) {
    size_t s = i;
    while (i < in.size() && f(in[i])) i++;
    return in.substr(s, i - s);
  }
  static bool alnum(char c) { return isalnum((unsigned char)c) != 0; }

  std::string name() {
    std::string n = span([](char c) { return alnum(c) || c == '_' || c == '.' || c == '$'; });
    if (n.empty()) fail("name");
    return n;
  }
  static uint64_t integer(const std::string& s) {
    std::string t = s;
    int radix = 10;
    if (t.rfind("0x", 0) == 0) { radix = 16; t = t.substr(2); }
    else if (t.rfind("0b", 0) == 0) { radix = 2; t = t.substr(2); }
    else if (!t.empty() && t[0] == '+') t = t.substr(1);
    if (t.empty()) throw Error(HVM64_ERR_BAD_INPUT, "Parsing error: bad number '" + s + "'");
    uint64_t v = 0;
    for (char c : t) {
      int d = isdigit((unsigned char)c) ? c - '0' : (isxdigit((unsigned char)c) ? (tolower(c) - 'a' + 10) : 99);
      if (d >= radix || v > (UINT64_MAX - uint64_t(d)) / uint64_t(radix))
        throw Error(HVM64_ERR_BAD_INPUT, "Parsing error: bad number '" + s + "'");
      v = v * uint64_t(radix) + uint64_t(d);
    }
    return v;
  }
  static float real(const std::string& s) {
    std::string t = s;
    bool neg = false;
    if (!t.empty() && (t[0] == '+' || t[0] == '-')) { neg = t[0] == '-'; t = t.substr(1); }
    std::string low;
    for (char c : t) low += char(tolower((unsigned char)c));
    if (low == "inf" || low == "infinity") return neg ? -INFINITY : INFINITY;
    if (low == "nan") return neg ? -NAN : NAN;
    size_t k = 0;
    bool any = false;
    while (k < t.size() && isdigit((unsigned char)t[k])) { k++; any = true; }
    if (k < t.size() && t[k] == '.') {
      k++;
      while (k < t.size() && isdigit((unsigned char)t[k])) { k++; any = true; }
    }
    if (any && k < t.size() && (t[k] == 'e' || t[k] == 'E')) {
      size_t e0 = ++k;
      if (k < t.size() && (t[k] == '+' || t[k] == '-')) { k++; e0 = k; }
      while (k < t.size() && isdigit((unsigned char)t[k])) k++;
      if (k == e0) any = false;
    }
    if (!any || k != t.size()) throw Error(HVM64_ERR_BAD_INPUT, "Parsing error: bad float '" + s + "'");
    float f = strtof(t.c_str(), nullptr);
    return neg ? -f : f;
  }
  uint32_t num_lit() {
    std::string n = span([](char c) { return alnum(c) || c == '+' || c == '-' || c == '.'; });
    if (n.find('.') != std::string::npos || n.find("inf") != std::string::npos || n.find("NaN") != std::string::npos)
      return num_f24(real(n));
    if (!n.empty() && (n[0] == '+' || n[0] == '-')) {
      int32_t v = int32_t(uint32_t(integer(n.substr(1))));
      return num_i24(n[0] == '-' ? int32_t(0u - uint32_t(v)) : v);
    }
    return num_u24(uint32_t(integer(n)));
  }
  uint32_t number() {
    skip_trivia();
    if (peek() != '[') return num_lit();
    need("[");
    int op = -1;
    for (int t = 0; t < NT_COUNT && op < 0; t++)
      if (in.compare(i, strlen(NUMTAG_STR[t]), NUMTAG_STR[t]) == 0) op = t;
    if (op < 0) fail("operator");
    i += strlen(NUMTAG_STR[op]);
    skip_trivia();
    if (op < NT_SYM || peek() == ']') {
      need("]");
      return num_sym(uint32_t(op));
    }
    uint32_t lhs = num_lit();
    need("]");
    return num_unary(uint32_t(op), lhs);
  }
  uint64_t label_number() {
    skip_trivia();
    std::string d = span([](char c) { return isdigit((unsigned char)c) || c == '_'; });
    d.erase(std::remove(d.begin(), d.end(), '_'), d.end());
    if (d.empty()) fail("numeric digit");
    return integer(d);
  }
  Tree* tree() {
    skip_trivia();
    int c = peek();
    if (c == '*') { i++; return arena.make(K_ERA); }
    if (c == '(' || c == '{' || c == '#') {
      i++;
      uint16_t tag = 0;
      int ch = c;
      if (c == '#') {
        tag = uint16_t(label_number());
        skip_trivia();
        ch = peek();
        if (ch >= 0) i++;
      }
      uint16_t kind;
      const char* close;
      if (ch == '(') { kind = 0; close = ")"; }
      else if (ch == '{') { kind = 1; close = "}"; }
      else fail("`(` or `{`");
      Tree* t = arena.make(K_CTR);
      t->lab = uint16_t(tag * 2 + kind);
      t->p1 = tree();
      t->p2 = tree();
      need(close);
      return t;
    }
    if (c == '@') {
      i++;
      skip_trivia();
      Tree* t = arena.make(K_REF);
      t->name = name();
      return t;
    }
    if (c == '$' || c == '?') {
      need(c == '$' ? "$(" : "?(");
      Tree* t = arena.make(c == '$' ? K_OP : K_SWITCH);
      t->p1 = tree();
      t->p2 = tree();
      need(")");
      return t;
    }
    if ((c >= '0' && c <= '9') || c == '+' || c == '-' || c == '[') {
      Tree* t = arena.make(K_NUM);
      t->num = number();
      return t;
    }
    Tree* t = arena.make(K_VAR);
    t->name = name();
    return t;
  }
  AstNet net() {
    AstNet n;
    n.root = tree();
    while (eat("&")) {
      Tree* a = tree();
      need("~");
      n.redexes.push_back({a, tree()});
    }
    return n;
  }
  void end() {
    if (i != in.size()) throw Error(HVM64_ERR_BAD_INPUT, "Parsing error: unable to parse the whole input");
  }
};
}  // namespace

AstBook parse_book(const std::string& text) {
  AstBook b;
  Parser p(text, *b.arena);
  while (p.eat("@")) {
    std::string name = p.name();
    p.need("=");
    b.nets[name] = p.net();
  }
  p.end();
  return b;
}
AstNet parse_net(const std::string& text, Arena& arena) {
  Parser p(text, arena);
  AstNet n = p.net();
  p.end();
  return n;
}
Tree* parse_tree(const std::string& text, Arena& arena) {
  Parser p(text, arena);
  Tree* t = p.tree();
  p.end();
  return t;
}

// ast.rs:246-263
static void print_into(std::string& o, const Tree* t) {
  switch (t->kind) {
    case K_ERA: o += '*'; return;
    case K_VAR: o += t->name; return;
    case K_REF: o += '@'; o += t->name; return;
    case K_NUM: o += num_to_string(t->num); return;
    case K_CTR:
      if (t->lab >= 2) { o += '#'; o += std::to_string(t->lab / 2); }
      o += (t->lab & 1) ? '{' : '(';
      print_into(o, t->p1);
      o += ' ';
      print_into(o, t->p2);
      o += (t->lab & 1) ? '}' : ')';
      return;
    case K_OP: case K_SWITCH:
      o += t->kind == K_OP ? "$(" : "?(";
      print_into(o, t->p1);
      o += ' ';
      print_into(o, t->p2);
      o += ')';
      return;
  }
}
std::string print_tree(const Tree* t) {
  std::string o;
  print_into(o, t);
  return o;
}
std::string print_net(const AstNet& n) {
  std::string o;
  print_into(o, n.root);
  for (auto& r : n.redexes) {
    o += "\n  & ";
    print_into(o, r.first);
    o += " ~ ";
    print_into(o, r.second);
  }
  return o;
}

// util/src/create_var.rs:5-34
static std::string create_var(size_t id) {
  std::string t;
  for (id += 1; id > 0; id /= 26) {
    id -= 1;
    t.push_back(char('a' + id % 26));
  }
  std::reverse(t.begin(), t.end());
  return t;
}
static std::optional<size_t> var_to_num(const std::string& s) {
  size_t n = 0;
  for (char c : s) {
    if (c < 'a') return std::nullopt;
    size_t d = size_t(c - 'a');
    if (d > size_t('z')) return std::nullopt;
    n = n * 26 + d + 1;
  }
  if (n == 0) return std::nullopt;
  return n - 1;
}
static void max_var(const Tree* t, size_t& fresh) {
  if (t->kind == K_VAR)
    if (auto v = var_to_num(t->name)) fresh = std::max(fresh, *v);
  if (t->p1) max_var(t->p1, fresh);
  if (t->p2) max_var(t->p2, fresh);
}
// ast.rs:112-123
void apply_tree(AstNet& net, Tree* arg, Arena& arena) {
  size_t fresh = 0;
  max_var(net.root, fresh);
  for (auto& r : net.redexes) { max_var(r.first, fresh); max_var(r.second, fresh); }
  max_var(arg, fresh);
  std::string v = create_var(fresh + 1);
  Tree* app = arena.make(K_CTR);
  app->p1 = arg;
  app->p2 = arena.make(K_VAR);
  app->p2->name = v;
  Tree* fun = net.root;
  net.root = arena.make(K_VAR);
  net.root->name = v;
  net.redexes.push_back({fun, app});
}

// ===========================================================================
// Label sets (runtime/src/def.rs:19-49; host/src/calc_labels.rs:78-194)
// ===========================================================================
void LabSet::add(uint16_t lab) {
  min_safe = std::max<uint16_t>(min_safe, uint16_t(lab + 1));
  size_t w = lab >> 6;
  if (w >= bits.size()) bits.resize(w + 1, 0);
  bits[w] |= uint64_t(1) << (lab & 63);
}
bool LabSet::has(uint16_t lab) const {
  if (lab >= min_safe) return false;
  size_t w = lab >> 6;
  return w < bits.size() && ((bits[w] >> (lab & 63)) & 1);
}
LabSet LabSet::all() {
  LabSet s;
  s.min_safe = 0xFFFF;
  s.bits.assign(1024, ~uint64_t(0));
  return s;
}
void LabSet::unite(const LabSet& o) {
  min_safe = std::max(min_safe, o.min_safe);
  if (o.bits.size() > bits.size()) bits.resize(o.bits.size(), 0);
  for (size_t k = 0; k < o.bits.size(); k++) bits[k] |= o.bits[k];
}

namespace {
// Two-phase memoised traversal: a def met again at a smaller depth is part of
// a cycle whose head re-traverses once the head's set is known.
struct Labeler {
  const AstBook& book;
  struct St { bool done; LabSet labs; size_t head; };
  std::map<std::string, St> memo;
  std::set<std::string>* missing = nullptr;  // collects absent references (null: they are errors)

  size_t def(const std::string& key, std::optional<size_t> depth, LabSet* out) {
    auto it = memo.find(key);
    if (it == memo.end()) {
      memo[key] = St{false, {}, *depth};
      return calc(key, depth, out);
    }
    if (it->second.done) {
      if (out) out->unite(it->second.labs);
      return SIZE_MAX;
    }
    if (depth) return it->second.head;
    it->second = St{true, {}, 0};
    return calc(key, depth, out);
  }
  size_t calc(const std::string& key, std::optional<size_t> depth, LabSet* out) {
    LabSet labs;
    size_t head = within(key, depth, &labs);
    if (out) out->unite(labs);
    if (depth && *depth > head) {
      memo[key] = St{false, {}, head};
    } else {
      memo[key] = St{true, labs, 0};
      if (depth && *depth == head) within(key, std::nullopt, nullptr);
    }
    return head;
  }
  size_t within(const std::string& key, std::optional<size_t> depth, LabSet* out) {
    const AstNet& n = book.nets.at(key);
    size_t head = tree(n.root, depth, out);
    for (auto& r : n.redexes) {
      head = std::min(head, tree(r.first, depth, out));
      head = std::min(head, tree(r.second, depth, out));
    }
    return head;
  }
  size_t tree(const Tree* t, std::optional<size_t> depth, LabSet* out) {
    if (t->kind == K_CTR && out) out->add(t->lab);
    if (t->kind == K_REF) {
      if (book.nets.count(t->name))
        return def(t->name, depth ? std::optional<size_t>(*depth + 1) : std::nullopt, out);
      if (!missing)
        throw Error(HVM64_ERR_BAD_INPUT, "Found reference \"" + t->name + "\", which is not in the book!");
      missing->insert(t->name);
      if (out) out->unite(LabSet::all());
      return SIZE_MAX;
    }
    size_t h = SIZE_MAX;
    if (t->p1) h = std::min(h, tree(t->p1, depth, out));
    if (t->p2) h = std::min(h, tree(t->p2, depth, out));
    return h;
  }
};

// ===========================================================================
// Def encoding (host/src/encode.rs:123-248) + register renaming.
// ===========================================================================
struct RawInstr {
  InstrKind k;
  uint8_t op = 0;
  uint16_t lab = 0;
  uint32_t a = 0, b = 0, c = 0, d = 0;
  uint64_t port = 0;
};

struct Encoder {
  const Book& book;
  std::vector<RawInstr> out;
  uint32_t trgs = 1;
  std::map<std::string, uint32_t> scope;
  // Emit the smaller child of a binary node first.  A child's wire stays live
  // while its sibling's subtree is emitted, so a deeply one-sided literal tree
  // needs one live wire per level in the reference's order (first child
  // first) and a constant number this way.  Used only for Defs that would not
  // fit the device register file otherwise.
  bool small_first = false;
  std::unordered_map<const Tree*, size_t> sizes;

  size_t size(const Tree* t) {
    if (!t) return 0;
    auto it = sizes.find(t);
    if (it != sizes.end()) return it->second;
    size_t n = 1 + size(t->p1) + size(t->p2);
    sizes[t] = n;
    return n;
  }
  bool swap_children(const Tree* a, const Tree* b) { return small_first && size(b) < size(a); }

  uint32_t fresh() { return trgs++; }
  uint64_t ref(const std::string& n) {
    auto it = book.ids.find(n);
    if (it == book.ids.end()) throw Error(HVM64_ERR_BAD_INPUT, "Found reference \"" + n + "\", which is not in the book!");
    return ref_port(it->second, book.labs[it->second].min_safe);
  }
  void link_const(uint32_t t, uint64_t p) { out.push_back({I_LINKCONST, 0, 0, t, 0, 0, 0, p}); }
  void link(uint32_t a, uint32_t b) { out.push_back({I_LINK, 0, 0, a, b, 0, 0, 0}); }
  uint32_t constant(uint64_t p) {
    uint32_t t = fresh();
    out.push_back({I_CONST, 0, 0, t, 0, 0, 0, p});
    return t;
  }
  void net(const AstNet& n, uint32_t t) {
    tree(n.root, t);
    for (auto& r : n.redexes) redex(r.first, r.second);
  }
  void redex(const Tree* a, const Tree* b) {
    uint64_t port;
    const Tree* t;
    if (a->kind == K_ERA) { port = PORT_ERA; t = b; }
    else if (b->kind == K_ERA) { port = PORT_ERA; t = a; }
    else if (a->kind == K_REF) { port = ref(a->name); t = b; }
    else if (b->kind == K_REF) { port = ref(b->name); t = a; }
    else if (a->kind == K_NUM) { port = a->num; t = b; }
    else if (b->kind == K_NUM) { port = b->num; t = a; }
    else {
      uint32_t av = fresh(), aw = fresh(), bv = fresh(), bw = fresh();
      out.push_back({I_WIRES, 0, 0, av, aw, bv, bw, 0});
      tree(a, av);
      tree(b, bv);
      link(aw, bw);
      return;
    }
    tree(t, constant(port));
  }
  void tree(const Tree* t, uint32_t trg) {
    switch (t->kind) {
      case K_ERA: link_const(trg, PORT_ERA); return;
      case K_NUM: link_const(trg, t->num); return;
      case K_REF: link_const(trg, ref(t->name)); return;
      case K_CTR: {
        uint32_t p1 = fresh(), p2 = fresh();
        out.push_back({I_CTR, 0, t->lab, trg, p1, p2, 0, 0});
        if (swap_children(t->p1, t->p2)) {
          tree(t->p2, p2);
          tree(t->p1, p1);
        } else {
          tree(t->p1, p1);
          tree(t->p2, p2);
        }
        return;
      }
      case K_OP: {
        uint8_t op = NT_SYM;
        const Tree* rhs = t->p1;
        const Tree* o = t->p2;
        if (t->p1->kind == K_NUM && t->p2->kind == K_OP && num_tag(t->p1->num) == NT_SYM) {
          op = uint8_t(num_payload(t->p1->num));
          rhs = t->p2->p1;
          o = t->p2->p2;
        }
        if (rhs->kind == K_NUM) {
          uint32_t out_t = fresh();
          out.push_back({I_OPNUM, op, 0, trg, 0, out_t, 0, rhs->num});
          tree(o, out_t);
        } else {
          uint32_t r = fresh(), out_t = fresh();
          out.push_back({I_OP, op, 0, trg, r, out_t, 0, 0});
          if (swap_children(rhs, o)) {
            tree(o, out_t);
            tree(rhs, r);
          } else {
            tree(rhs, r);
            tree(o, out_t);
          }
        }
        return;
      }
      case K_SWITCH: {
        uint32_t arms = fresh(), o = fresh();
        out.push_back({I_SWITCH, 0, 0, trg, arms, o, 0, 0});
        if (swap_children(t->p1, t->p2)) {
          tree(t->p2, o);
          tree(t->p1, arms);
        } else {
          tree(t->p1, arms);
          tree(t->p2, o);
        }
        return;
      }
      case K_VAR: {
        auto it = scope.find(t->name);
        if (it == scope.end()) {
          scope.emplace(t->name, trg);
        } else {
          uint32_t other = it->second;
          scope.erase(it);
          link(other, trg);
        }
        return;
      }
    }
  }
};

// Linear-scan renaming: every TrgId is defined once and read once, so a
// register can be reused right after its single read.
static uint32_t rename(std::vector<RawInstr>& ins, uint32_t ntrgs) {
  std::vector<int64_t> reg(ntrgs, -1);
  std::vector<uint32_t> freelist;
  uint32_t nregs = 1;
  reg[0] = 0;
  auto use = [&](uint32_t& t) {
    if (t >= ntrgs || reg[t] < 0) throw Error(HVM64_ERR_BAD_INPUT, "internal: trg read before write");
    uint32_t r = uint32_t(reg[t]);
    reg[t] = -2;
    freelist.push_back(r);
    t = r;
  };
  auto def = [&](uint32_t& t) {
    uint32_t r;
    if (!freelist.empty()) { r = freelist.back(); freelist.pop_back(); }
    else r = nregs++;
    reg[t] = r;
    t = r;
  };
  for (RawInstr& i : ins) {
    switch (i.k) {
      case I_CONST: def(i.a); break;
      case I_LINK: use(i.a); use(i.b); break;
      case I_LINKCONST: use(i.a); break;
      case I_CTR: case I_OP: case I_SWITCH: use(i.a); def(i.b); def(i.c); break;
      case I_OPNUM: use(i.a); def(i.c); break;
      case I_WIRES: def(i.a); def(i.b); def(i.c); def(i.d); break;
    }
  }
  return nregs;
}

static void emit(Book& book, const std::vector<RawInstr>& raw, uint32_t nregs, DevDef& d) {
  if (nregs > MAX_REGS)
    throw Error(HVM64_ERR_BAD_INPUT, "definition needs " + std::to_string(nregs) + " live wires; the device limit is " +
                                         std::to_string(MAX_REGS));
  d.ins_off = uint32_t(book.instrs.size());
  d.ins_len = uint32_t(raw.size());
  d.nregs = nregs;
  uint32_t nodes = 0, links = 0;
  for (const RawInstr& r : raw) {
    DevInstr x{};
    x.k = r.k;
    x.op = r.op;
    x.lab = r.lab;
    x.a = uint8_t(r.a); x.b = uint8_t(r.b); x.c = uint8_t(r.c); x.d = uint8_t(r.d);
    x.port = r.port;
    book.instrs.push_back(x);
    nodes += r.k == I_SWITCH ? 3 : (r.k == I_CTR || r.k == I_OP || r.k == I_OPNUM || r.k == I_WIRES) ? 1 : 0;
    links += (r.k == I_LINK || r.k == I_LINKCONST) ? 1 : 0;
  }
  d.nodes = nodes;
  d.redexes = links + nodes;
}
}  // namespace

// Encodes a Def's net into device instructions: in the reference's order,
// or smaller-child-first when that order needs more than LOCAL_REGS
// registers and the other does not (else the order needing fewer).
static uint32_t encode_net(Book& book, const AstNet& net, DevDef& d) {
  std::vector<RawInstr> best;
  uint32_t best_regs = 0;
  for (int pass = 0; pass < 2; pass++) {
    Encoder e{book, {}, 1, {}};
    e.small_first = pass == 1;
    e.net(net, 0);
    if (!e.scope.empty()) throw Error(HVM64_ERR_BAD_INPUT, "unbound variables: " + e.scope.begin()->first);
    uint32_t nregs = rename(e.out, e.trgs);
    if (pass == 0 || nregs < best_regs) {
      best = std::move(e.out);
      best_regs = nregs;
    }
    if (best_regs <= LOCAL_REGS) break;
  }
  emit(book, best, best_regs, d);
  return best_regs;
}

void Book::load(const AstBook& b, bool inert_missing) {
  keep.push_back(b.arena);
  // Phase 1: ids and label sets (host.rs:54-65); phase 2: instructions.
  for (auto& [name, _] : b.nets) {
    ids[name] = uint32_t(names.size());
    names.push_back(name);
  }
  std::set<std::string> missing;
  Labeler L{b, {}, inert_missing ? &missing : nullptr};
  for (auto& [name, _] : b.nets) L.def(name, 0, nullptr);
  for (const std::string& name : missing) {
    ids[name] = uint32_t(names.size());
    names.push_back(name);
  }
  labs.resize(names.size());
  for (auto& [name, st] : L.memo) {
    if (!st.done) throw Error(HVM64_ERR_BAD_INPUT, "label analysis did not converge");
    labs[ids[name]] = st.labs;
  }
  defs.resize(names.size());
  for (const std::string& name : missing) {  // pre_reduce.rs:89-102 (InertDef)
    uint32_t id = ids[name];
    labs[id] = LabSet::all();
    DevDef d{};
    d.ins_off = uint32_t(instrs.size());
    d.ins_len = 1;
    d.nregs = 1;
    d.flags = DEF_INERT;
    d.min_safe = labs[id].min_safe;
    d.lab_off = uint32_t(labbits.size());
    d.lab_len = uint32_t(labs[id].bits.size());
    labbits.insert(labbits.end(), labs[id].bits.begin(), labs[id].bits.end());
    DevInstr x{};
    x.k = I_CAPTURE;
    x.port = ref_port(id, d.min_safe);
    instrs.push_back(x);
    defs[id] = d;
  }
  for (auto& [name, net] : b.nets) {
    uint32_t id = ids[name];
    DevDef d{};
    encode_net(*this, net, d);
    d.min_safe = labs[id].min_safe;
    d.lab_off = uint32_t(labbits.size());
    d.lab_len = uint32_t(labs[id].bits.size());
    labbits.insert(labbits.end(), labs[id].bits.begin(), labs[id].bits.end());
    defs[id] = d;
  }
}

void Book::replace_def(uint32_t id, const AstNet& net) {
  if (id >= defs.size()) throw Error(HVM64_ERR_BAD_INPUT, "no such definition");
  DevDef d = defs[id];
  encode_net(*this, net, d);
  d.flags = uint16_t(d.flags & ~DEF_INERT);
  defs[id] = d;
}

uint32_t Book::add_expr(const AstNet& net) {
  DevDef d{};
  encode_net(*this, net, d);
  d.min_safe = 0;
  d.lab_off = 0;
  d.lab_len = 0;
  d.flags = DEF_EXPR;  // expression program: no DREF is counted for it
  defs.push_back(d);
  return uint32_t(defs.size() - 1);
}

// ===========================================================================
// Readback (host/src/readback.rs:23-87)
// ===========================================================================
namespace {
struct Reader {
  const Book& book;
  const uint64_t* heap;
  uint64_t words;
  std::unordered_map<uint64_t, size_t> vars;
  size_t next_var = 0;
  std::string o;
  // Gathered (address, word) pairs.  The device walk visits words in the
  // order this reader loads them, so a cursor serves almost every load; the
  // address map is built only if a load ever misses it.
  const uint64_t* pairs = nullptr;
  size_t npairs = 0, cursor = 0;
  std::unordered_map<uint64_t, uint64_t> sparse;

  uint64_t load(uint64_t addr) {
    uint64_t w = addr >> 3;
    if (w >= words) throw Error(HVM64_ERR_BAD_INPUT, "readback: address outside the heap");
    if (pairs) {
      if (cursor < npairs && pairs[2 * cursor] == addr) return pairs[2 * cursor++ + 1];
      if (sparse.empty())
        for (size_t i = 0; i < npairs; i++) sparse[pairs[2 * i]] = pairs[2 * i + 1];
      auto it = sparse.find(addr);
      if (it == sparse.end()) throw Error(HVM64_ERR_BAD_INPUT, "readback: word not gathered");
      return it->second;
    }
    return heap[w];
  }
  bool live_addr(uint64_t p) const { return (p >> 48) == 0 && (p & ADDR_MASK) != 0 && ((p & ADDR_MASK) >> 3) < words; }
  void wire(uint64_t w) { port(load(w), w); }
  void port(uint64_t p, uint64_t from) {
    uint8_t tag = p & 7;
    switch (tag) {
      case T_VAR: case T_RED: {
        uint64_t end = p & ADDR_MASK;
        if (live_addr(p)) {
          // Follow redirects: a word holding Red(x) stands for x.
          for (uint64_t guard = 0; guard < words; guard++) {
            uint64_t t = load(end);
            if ((t & 7) != T_RED || !live_addr(t)) break;
            end = t & ADDR_MASK;
          }
        }
        uint64_t key = std::min(from, end);
        auto it = vars.find(key);
        if (it != vars.end()) {
          o += create_var(it->second);
          vars.erase(it);
        } else {
          vars.emplace(key, next_var);
          o += create_var(next_var++);
        }
        return;
      }
      case T_REF: {
        if (p == PORT_ERA) { o += '*'; return; }
        uint64_t addr = p & ADDR_MASK;
        uint64_t id = (addr >> 3) - 1;
        if ((addr & EXPAND_BIT) || id >= book.names.size()) { o += "@<expand>"; return; }
        o += '@';
        o += book.names[id];
        return;
      }
      case T_NUM: o += num_to_string(uint32_t(p)); return;
      case T_OP: {
        uint8_t op = uint8_t(p >> 48);
        uint64_t a = p & ADDR_MASK;
        if (op != NT_SYM) o += "$([" + std::string(NUMTAG_STR[op < NT_COUNT ? op : 0]) + "] ";
        o += "$(";
        wire(a);
        o += ' ';
        wire(a ^ 8);
        o += ')';
        if (op != NT_SYM) o += ')';
        return;
      }
      case T_CTR: {
        uint16_t lab = uint16_t(p >> 48);
        uint64_t a = p & ADDR_MASK;
        if (lab >= 2) { o += '#'; o += std::to_string(lab / 2); }
        o += (lab & 1) ? '{' : '(';
        wire(a);
        o += ' ';
        wire(a ^ 8);
        o += (lab & 1) ? '}' : ')';
        return;
      }
      case T_SWITCH: {
        uint64_t a = p & ADDR_MASK;
        o += "?(";
        wire(a);
        o += ' ';
        wire(a ^ 8);
        o += ')';
        return;
      }
      default: throw Error(HVM64_ERR_BAD_INPUT, "readback: bad port");
    }
  }
};
}  // namespace

std::string readback(const Book& book, const uint64_t* heap, uint64_t heap_words, uint64_t root) {
  Reader r{book, heap, heap_words, {}, 0, {}};
  r.wire(root);
  return r.o;
}

// ===========================================================================
// Ahead-of-time Def specialisation (src/compile.rs:110-161)
// ===========================================================================
uint64_t defs_hash(const Book& book, uint32_t n) {
  // FNV-1a over every field the generated code or its dispatch depends on
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&](uint64_t v) {
    for (int k = 0; k < 8; k++) {
      h ^= (v >> (8 * k)) & 0xff;
      h *= 0x100000001b3ull;
    }
  };
  mix(n);
  for (uint32_t id = 0; id < n && id < book.defs.size(); id++) {
    const DevDef& d = book.defs[id];
    mix(d.ins_len);
    mix(d.nregs);
    mix(d.min_safe);
    mix(d.flags);
    mix(d.nodes);
    mix(d.redexes);
    for (uint32_t k = 0; k < d.lab_len; k++) mix(book.labbits[d.lab_off + k]);
    for (uint32_t k = 0; k < d.ins_len; k++) {
      const DevInstr& x = book.instrs[d.ins_off + k];
      mix(uint64_t(x.k) | uint64_t(x.op) << 8 | uint64_t(x.lab) << 16 | uint64_t(x.a) << 32 | uint64_t(x.b) << 40 |
          uint64_t(x.c) << 48 | uint64_t(x.d) << 56);
      mix(x.port);
    }
  }
  return h;
}

std::string compile_defs_cuda(const Book& book) {
  const uint32_t n = book.def_count();
  char buf[256];
  std::string o;
  snprintf(buf, sizeof buf, "// Generated by hvm64 compile: %u definitions.\n#define HVM_GEN_NDEFS %uu\n"
           "#define HVM_GEN_HASH 0x%016llxull\n\n", n, n, (unsigned long long)defs_hash(book, n));
  o += buf;
  auto hex = [&](uint64_t v) {
    snprintf(buf, sizeof buf, "0x%llxull", (unsigned long long)v);
    return std::string(buf);
  };
  auto r = [](unsigned i) { return "r" + std::to_string(i); };
  // Which Defs get a function.  Long ones (literal data, such as an entry
  // point holding a whole input tree, called once) stay on the VM.  A Book of
  // many Defs (a batch: shared library Defs plus a few per net) compiles only
  // the Defs reachable from two or more of its entry points (Defs no other Def
  // references): compiling thousands of per-net Defs would take long and each
  // runs for one net.
  constexpr uint32_t MAX_INS = 128, ALL_BELOW = 512;
  std::vector<std::vector<uint32_t>> refs(n);
  std::vector<uint32_t> referrers(n, 0);
  for (uint32_t id = 0; id < n; id++) {
    const DevDef& d = book.defs[id];
    for (uint32_t k = 0; k < d.ins_len; k++) {
      const DevInstr& x = book.instrs[d.ins_off + k];
      if ((x.k == I_CONST || x.k == I_LINKCONST) && (x.port & 7) == T_REF && !(x.port & EXPAND_BIT)) {
        uint64_t t = ((x.port & ADDR_MASK) >> 3) - 1;
        if (t < n && t != id) {
          refs[id].push_back(uint32_t(t));
          referrers[t]++;
        }
      }
    }
  }
  std::vector<uint8_t> roots_reaching(n, 0);  // 0, 1 or 2 (two or more)
  if (n > ALL_BELOW) {
    std::vector<uint32_t> seen(n, ~0u), stack;
    for (uint32_t root = 0; root < n; root++) {
      if (referrers[root]) continue;
      stack.assign(1, root);
      seen[root] = root;
      while (!stack.empty()) {
        uint32_t v = stack.back();
        stack.pop_back();
        if (roots_reaching[v] < 2) roots_reaching[v]++;
        for (uint32_t t : refs[v])
          if (seen[t] != root) {
            seen[t] = root;
            stack.push_back(t);
          }
      }
    }
  }
  std::vector<uint32_t> done;
  for (uint32_t id = 0; id < n; id++) {
    const DevDef& d = book.defs[id];
    if (d.ins_len > MAX_INS || (n > ALL_BELOW && roots_reaching[id] < 2)) continue;
    done.push_back(id);
    o += "// @" + book.names[id] + "\n";
    o += "HVM_COLD void gen_def_" + std::to_string(id) + "(const Ctx& c, ull r0) {\n";
    if (d.nregs > 1) {
      o += "  ull";
      for (uint32_t k = 1; k < d.nregs; k++) o += (k > 1 ? ", " : " ") + r(k);
      o += ";\n";
    }
    for (uint32_t k = 0; k < d.ins_len; k++) {
      const DevInstr& x = book.instrs[d.ins_off + k];
      switch (x.k) {
        case I_CONST: o += "  " + r(x.a) + " = " + hex(x.port) + ";\n"; break;
        case I_LINK: o += "  count(c, EX_DLINKS); link_trg(c, " + r(x.a) + ", " + r(x.b) + ");\n"; break;
        case I_LINKCONST: o += "  count(c, EX_DLINKS); link_trg_port(c, " + r(x.a) + ", " + hex(x.port) + ");\n"; break;
        case I_CTR:
          o += "  do_ctr(c, " + std::to_string(x.lab) + "u, " + r(x.a) + ", " + r(x.b) + ", " + r(x.c) + ");\n";
          break;
        case I_OP:
          o += "  do_op(c, " + std::to_string(x.op) + "u, " + r(x.a) + ", " + r(x.b) + ", " + r(x.c) + ");\n";
          break;
        case I_OPNUM:
          o += "  " + r(x.c) + " = do_op_num(c, " + std::to_string(x.op) + "u, " + r(x.a) + ", " +
               std::to_string(uint32_t(x.port)) + "u);\n";
          break;
        case I_SWITCH: o += "  do_switch(c, " + r(x.a) + ", " + r(x.b) + ", " + r(x.c) + ");\n"; break;
        case I_WIRES:
          o += "  { ull n = alloc(c); " + r(x.a) + " = pvar(n); " + r(x.b) + " = n; " + r(x.c) + " = pvar(n ^ 8); " +
               r(x.d) + " = n ^ 8; }\n";
          break;
        case I_CAPTURE: o += "  capture(c, " + hex(x.port) + ", " + r(x.a) + ");\n"; break;
      }
    }
    o += "}\n";
  }
  o += "\n// The Def's function for Def `id` (false: none; the VM runs it).\n";
  o += "HVM_INL bool gen_call(const Ctx& c, unsigned id, ull t0) {\n  switch (id) {\n";
  for (uint32_t id : done)
    o += "    case " + std::to_string(id) + "u: gen_def_" + std::to_string(id) + "(c, t0); return true;\n";
  o += "  }\n  return false;\n}\n";
  return o;
}

// ===========================================================================
// Pre-reduce driver (transform/src/pre_reduce.rs:38-74,136-164)
// ===========================================================================
namespace {
struct PreReduceDfs {
  const AstBook& ast;
  Book& book;
  const std::set<std::string>& skip;
  uint64_t max_rwts;
  const std::function<PreReduceRun(uint32_t)>& run_one;
  std::map<std::string, int> seen;  // 0: on the path ("Cycled"), 1: done
  std::map<std::string, std::string> reduced;
  PreReduceOut out;

  void visit_tree(const Tree* t) {  // pre_reduce.rs:122-129
    if (t->kind == K_REF) visit(t->name);
    if (t->p1) visit_tree(t->p1);
    if (t->p2) visit_tree(t->p2);
  }
  void visit(const std::string& name) {  // pre_reduce.rs:137-164
    auto src = ast.nets.find(name);
    if (seen.count(name) || skip.count(name) || src == ast.nets.end()) return;
    seen[name] = 0;
    visit_tree(src->second.root);
    for (auto& rd : src->second.redexes) {
      visit_tree(rd.first);
      visit_tree(rd.second);
    }
    const uint32_t id = book.ids.at(name);
    PreReduceRun r = run_one(id);
    out.runs++;
    seen[name] = 1;
    if (r.status && r.status != HVM64_ERR_LIMIT)
      throw Error(r.status, "pre-reducing @" + name + ": " + r.error);
    // Net::reduce(limit) stops, reporting no normal form, once it has popped
    // `limit` redexes; it checks after each pop, so a reduction that pops
    // none is normal whatever the limit (net.rs:41-52).
    if (r.status == HVM64_ERR_LIMIT || (r.pops > 0 && r.pops >= max_rwts)) {
      // The reference keeps the net as it stood after max_rwts pops; a device
      // run does not stop at an exact pop, so the Def keeps its original net
      // (and adds no Rewrites).  Either way it is reported as not normal.
      out.not_normal.push_back(name);
      return;
    }
    for (int k = 0; k < 5; k++) out.rw[k] += r.rw[k];
    Arena arena;
    AstNet net = parse_net(r.text, arena);
    book.replace_def(id, net);
    reduced[name] = std::move(r.text);
  }
};
}  // namespace

std::string print_book(const AstBook& b) {
  std::string o;
  for (auto& [name, net] : b.nets) {
    if (!o.empty()) o += "\n\n";
    o += "@" + name + " = " + print_net(net);
  }
  return o;
}

PreReduceOut pre_reduce(const AstBook& ast, Book& book, const std::set<std::string>& skip, uint64_t max_rwts,
                        const std::function<PreReduceRun(uint32_t)>& run_one) {
  PreReduceDfs d{ast, book, skip, max_rwts, run_one, {}, {}, {}};
  for (auto& [name, _] : ast.nets) d.visit(name);
  for (auto& [name, net] : ast.nets) {  // pre_reduce.rs:60-67, then ast.rs:221-232
    if (!d.out.text.empty()) d.out.text += "\n\n";
    auto it = d.reduced.find(name);
    d.out.text += "@" + name + " = " + (it != d.reduced.end() ? it->second : print_net(net));
  }
  return std::move(d.out);
}

std::string readback_net(const Book& book, const uint64_t* heap, uint64_t heap_words, uint64_t root,
                         const uint64_t* redexes, size_t nredexes) {
  Reader r{book, heap, heap_words, {}, 0, {}};
  r.wire(root);
  for (size_t i = 0; i < nredexes; i++) {  // host/src/readback.rs:28-30
    r.o += "\n  & ";
    r.port(redexes[2 * i], 0);
    r.o += " ~ ";
    r.port(redexes[2 * i + 1], 0);
  }
  return r.o;
}

std::string readback_pairs(const Book& book, const uint64_t* pairs, size_t npairs, uint64_t heap_words,
                           uint64_t root) {
  Reader r{book, nullptr, heap_words, {}, 0, {}};
  r.pairs = pairs;
  r.npairs = npairs;
  r.wire(root);
  return r.o;
}

std::vector<ReadbackOut> readback_pairs_many(const Book& book, const uint64_t* pairs, const uint64_t* offsets,
                                             const unsigned* counts, const uint64_t* roots, size_t n,
                                             uint64_t heap_words, unsigned threads) {
  std::vector<ReadbackOut> out(n);
  std::atomic<size_t> next{0};
  struct Job {
    const Book* book;
    const uint64_t *pairs, *offsets, *roots;
    const unsigned* counts;
    size_t n;
    uint64_t heap_words;
    std::vector<ReadbackOut>* out;
    std::atomic<size_t>* next;
  } job{&book, pairs, offsets, roots, counts, n, heap_words, &out, &next};
  auto work = [](void* p) -> void* {
    Job* j = static_cast<Job*>(p);
    for (;;) {
      size_t i = j->next->fetch_add(1);
      if (i >= j->n) break;
      ReadbackOut& r = (*j->out)[i];
      if (j->counts[i] == ~0u) continue;  // not gathered: the caller reads it back another way
      try {
        r.text = readback_pairs(*j->book, j->pairs + 2 * j->offsets[i], j->counts[i], j->heap_words, j->roots[i]);
        r.ok = true;
      } catch (std::exception& e) {
        r.error = e.what();
      } catch (...) {
        r.error = "readback failed";
      }
    }
    return nullptr;
  };
  threads = std::max(1u, std::min<unsigned>(threads, unsigned(std::max<size_t>(n, 1))));
  std::vector<pthread_t> ts;
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, size_t(256) << 20);  // deep normal forms recurse
  for (unsigned t = 0; t < threads; t++) {
    pthread_t th;
    if (pthread_create(&th, &attr, work, &job) == 0) ts.push_back(th);
  }
  pthread_attr_destroy(&attr);
  if (ts.empty()) work(&job);  // no thread could start: do it here
  for (auto th : ts) pthread_join(th, nullptr);
  return out;
}

void with_big_stack(const std::function<void()>& f) {
  struct Box {
    const std::function<void()>* f;
    std::exception_ptr e;
  } box{&f, nullptr};
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, size_t(2) << 30);
  pthread_t th;
  auto tramp = [](void* p) -> void* {
    Box* b = static_cast<Box*>(p);
    try {
      (*b->f)();
    } catch (...) {
      b->e = std::current_exception();
    }
    return nullptr;
  };
  int rc = pthread_create(&th, &attr, tramp, &box);
  pthread_attr_destroy(&attr);
  if (rc != 0) {
    f();
    return;
  }
  pthread_join(th, nullptr);
  if (box.e) std::rethrow_exception(box.e);
}

}  // namespace hvm
