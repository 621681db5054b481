// Host side of the B200 reducer: the `.hvm` Book loader (ast/src/parser.rs),
// label sets (host/src/calc_labels.rs), Def encoding (host/src/encode.rs)
// into the flat device instruction table, and readback of a device heap image
// (host/src/readback.rs) into the text format (ast/src/ast.rs Display).
#pragma once
#include <stdint.h>

#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "num.h"

namespace hvm {

// ---- ports (runtime/src/port.rs:20-224), identical 64-bit layout ----------
// tag bits 0-2, address bits 3-47 (a byte offset into the device heap, so the
// other half of a node is addr ^ 8), label bits 48-63.  A Ref port's address
// is (def id + 1) << 3; an expansion agent's address has bit 47 set and names
// the heap word holding its output port.
enum PortTag : uint8_t { T_RED = 0, T_VAR = 1, T_REF = 2, T_NUM = 3, T_OP = 5, T_SWITCH = 6, T_CTR = 7 };
constexpr uint64_t PORT_ERA = 2;
constexpr uint64_t PORT_FREE = 0x8000000000000000ull;
constexpr uint64_t PORT_LOCK = 0xFFFFFFFFFFFFFFF0ull;
constexpr uint64_t PORT_GONE = 0xFFFFFFFFFFFFFFFFull;
constexpr uint64_t ADDR_MASK = 0x0000FFFFFFFFFFF8ull;
constexpr uint64_t EXPAND_BIT = 1ull << 47;

inline uint64_t port_new(uint8_t tag, uint16_t lab, uint64_t addr) { return (uint64_t(lab) << 48) | addr | tag; }
inline uint64_t ref_port(uint32_t def_id, uint16_t min_safe) { return port_new(T_REF, min_safe, uint64_t(def_id + 1) << 3); }

// ---- device instruction table -------------------------------------------
// One Def = a run of DevInstr (the reference's Instruction list,
// runtime/src/instruction.rs:34-72) over a small register file; TrgIds are
// renamed to registers by linear scan (each TrgId is written once and read
// once), register 0 being the Def's argument port.
// I_CAPTURE is the whole body of an inert Def (a reference a Book being
// pre-reduced lacks, transform/src/pre_reduce.rs:89-102): the call's redex
// (`port`, register a) is recorded for the host instead of expanded.
enum InstrKind : uint8_t { I_CONST, I_LINK, I_LINKCONST, I_CTR, I_OP, I_OPNUM, I_SWITCH, I_WIRES, I_CAPTURE };

struct DevInstr {  // 16 bytes
  uint8_t k;
  uint8_t op;    // NumTag for Op / OpNum
  uint16_t lab;  // Ctr label
  uint8_t a, b, c, d;  // registers
  uint64_t port;  // Const / LinkConst port, OpNum right operand (low 32 bits)
};

struct DevDef {  // 32 bytes
  uint32_t ins_off, ins_len;
  uint32_t nregs;
  uint32_t lab_off, lab_len;  // label bitset words in the shared table
  uint16_t min_safe;
  uint16_t flags;  // DEF_EXPR | DEF_INERT
  uint32_t nodes;  // upper bound on nodes one call allocates
  uint32_t redexes;
};
constexpr uint16_t DEF_EXPR = 1;   // an expression program: booting it counts no DREF
constexpr uint16_t DEF_INERT = 2;  // an inert Def (pre-reduce): its body is one I_CAPTURE
static_assert(sizeof(DevInstr) == 16, "DevInstr layout");
static_assert(sizeof(DevDef) == 32, "DevDef layout");

// A Def call's registers: up to LOCAL_REGS in the calling thread's local
// memory; more (up to MAX_REGS, the reach of a DevInstr's one-byte register
// indices) in a per-lane register file in device memory, which a run
// allocates only when its Book has such a Def.
constexpr uint32_t LOCAL_REGS = 48;
constexpr uint32_t MAX_REGS = 256;

struct LabSet {  // runtime/src/def.rs:7-62
  uint16_t min_safe = 0;
  std::vector<uint64_t> bits;
  void add(uint16_t lab);
  bool has(uint16_t lab) const;
  void unite(const LabSet& o);
  static LabSet all();  // LabSet::ALL (runtime/src/def.rs:17)
};

// ---- AST (ast/src/ast.rs) -------------------------------------------------
enum TreeKind : uint8_t { K_ERA, K_NUM, K_REF, K_CTR, K_OP, K_SWITCH, K_VAR };
struct Tree {
  TreeKind kind = K_ERA;
  uint16_t lab = 0;
  uint32_t num = 0;
  std::string name;
  Tree* p1 = nullptr;
  Tree* p2 = nullptr;
};
struct Arena {
  std::deque<Tree> nodes;
  Tree* make(TreeKind k);
};
struct AstNet {
  Tree* root = nullptr;
  std::vector<std::pair<Tree*, Tree*>> redexes;
};
struct AstBook {
  std::shared_ptr<Arena> arena = std::make_shared<Arena>();
  std::map<std::string, AstNet> nets;
};

struct Error : std::exception {
  int code;
  std::string msg;
  Error(int c, std::string m) : code(c), msg(std::move(m)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};

AstBook parse_book(const std::string& text);
AstNet parse_net(const std::string& text, Arena& arena);
Tree* parse_tree(const std::string& text, Arena& arena);
std::string print_tree(const Tree* t);
std::string print_net(const AstNet& n);
std::string print_book(const AstBook& b);  // ast.rs:221-232
std::string num_to_string(uint32_t n);
void apply_tree(AstNet& net, Tree* arg, Arena& arena);

// ---- a loaded Book: names, label sets and the device tables ---------------
struct Book {
  std::vector<std::string> names;  // def id -> name
  std::map<std::string, uint32_t> ids;
  std::vector<LabSet> labs;
  std::vector<DevDef> defs;  // Book defs first, then expression programs
  std::vector<DevInstr> instrs;
  std::vector<uint64_t> labbits;
  std::vector<std::shared_ptr<Arena>> keep;

  // Loads a Book (Host::insert_book, host/src/host.rs:34-73).  With
  // `inert_missing`, a reference the Book lacks becomes an inert Def with
  // LabSet::ALL (insert_book_with_default as transform/src/pre_reduce.rs:41
  // calls it) instead of an error.
  void load(const AstBook& b, bool inert_missing = false);
  // Replaces Def `id`'s instructions by the encoding of `net`, keeping its
  // label set (pre_reduce.rs:155-157: encode_def into the existing Def).
  void replace_def(uint32_t id, const AstNet& net);
  // Encodes an expression net as a program run against the root
  // (Host::encode_net, host/src/encode.rs:116-120).  Returns its def index.
  uint32_t add_expr(const AstNet& net);
  uint32_t def_count() const { return uint32_t(names.size()); }
  uint32_t max_nregs() const {
    uint32_t m = 0;
    for (const DevDef& d : defs) m = d.nregs > m ? d.nregs : m;
    return m;
  }
};

// Reads the net rooted at heap word `root` out of a heap image
// (Host::readback, host/src/readback.rs:23-87).  Redirect chains (Red ports
// left by concurrent linking) are followed to the live endpoint.
std::string readback(const Book& book, const uint64_t* heap, uint64_t heap_words, uint64_t root);
// The same followed by redexes (port pairs, ast.rs:234-244 layout), all
// sharing one variable naming: Host::readback of a net with redexes.
std::string readback_net(const Book& book, const uint64_t* heap, uint64_t heap_words, uint64_t root,
                         const uint64_t* redexes, size_t nredexes);
// Many nets' normal forms from gathered pairs at once, on `threads` host
// threads: net i's pairs start at pair offsets[i] and number counts[i]
// (~0u: not gathered, left empty).  A net that fails keeps its message.
struct ReadbackOut {
  bool ok = false;
  std::string text, error;
};
std::vector<ReadbackOut> readback_pairs_many(const Book& book, const uint64_t* pairs, const uint64_t* offsets,
                                             const unsigned* counts, const uint64_t* roots, size_t n,
                                             uint64_t heap_words, unsigned threads);
// The same from the (address, word) pairs a serving reducer gathered.
std::string readback_pairs(const Book& book, const uint64_t* pairs, size_t npairs, uint64_t heap_words,
                           uint64_t root);

// Book::pre_reduce (transform/src/pre_reduce.rs:38-74,136-164).  Each Def
// of `ast` not in `skip` is visited in byte order of names and first visits
// the Defs its original net references, depth first (a Def met again while
// still on that path is used as it is: the reference's "Cycled" state).  Then
// `run_one(id)` boots Def `id` of `book` alone, without the expansion agent,
// and reduces it; the net it reads back replaces the Def's instructions in
// `book` at once (so later Defs call the reduced version) and the Def's text
// in the result.  Label sets stay those of the original Book, as in the
// reference's Host.  `book` must have been loaded from `ast` with
// inert_missing.
struct PreReduceRun {
  int status = 0;         // HVM64_OK, HVM64_ERR_LIMIT (stopped early), or an error
  uint64_t pops = 0;      // redexes the reduction popped (Net::reduce's count)
  uint64_t rw[5] = {0};   // anni, comm, eras, dref, oper
  std::string text;       // the net read back (root, then its redexes)
  std::string error;
};
struct PreReduceOut {
  std::string text;       // the pre-reduced Book (ast.rs:221-232 Display)
  uint64_t rw[5] = {0};
  std::vector<std::string> not_normal;
  uint32_t runs = 0;
};
PreReduceOut pre_reduce(const AstBook& ast, Book& book, const std::set<std::string>& skip, uint64_t max_rwts,
                        const std::function<PreReduceRun(uint32_t)>& run_one);

// Ahead-of-time Def specialisation (the analogue of `hvm64 compile`,
// src/compile.rs:110-161): CUDA source with one straight-line function per
// Def of `book` (its instructions as direct calls on registers held in
// variables, instead of the device VM's loop over an instruction table) and
// the dispatch `gen_call`; included into the device runtime it replaces the
// VM for Books whose device tables hash to the same value.
std::string compile_defs_cuda(const Book& book);
// Hash of the device tables of Defs [0, n) (instructions, register counts,
// labels, flags): a compiled build runs its functions only for a Book whose
// hash matches the one it was generated from.
uint64_t defs_hash(const Book& book, uint32_t n);

// Runs f on a thread with a large stack (deep trees recurse; the reference
// grows its stack with `stacker`, util/src/maybe_grow.rs).
void with_big_stack(const std::function<void()>& f);

}  // namespace hvm
