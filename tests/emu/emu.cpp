// CPU emulation harness for the device runtime -- TESTS ONLY.
//
// Compiles the reducer's device code (hvm-64_b200/csrc/device.cuh) with the
// host platform layer (std::atomic_ref) and runs it on host threads: each
// thread plays one warp lane with a local LIFO redex stack, idle threads take
// shared work from a mutex-guarded queue, and nets end by the same
// holder-count rule as the CUDA kernel.  This exercises the allocator, the
// link/redirect protocol, the rules and the instruction VM under real
// concurrency without a GPU.  It is never a fallback for the CUDA path.
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <set>
#include <string>
#include <memory>
#include <thread>
#include <vector>

#include "device.cuh"

using namespace hvm;
using namespace hvm::dev;

namespace {
struct Emu {
  Params P{};
  Ctrl C{};
  std::vector<ull> heap;
  std::vector<NetState> nets;
  std::mutex mu;
  std::deque<std::pair<unsigned, std::vector<ull>>> queue;
};
thread_local Emu* g_emu = nullptr;

void flush(WarpSmem& W, NetState& ns) {
  for (int k = 0; k < NCOUNT; k++) {
    ull v = W.rw[k] + W.cnt[k * 32];
    if (v) atom_add(&ns.rw[k], v);
    W.rw[k] = 0;
    W.cnt[k * 32] = 0;
  }
}

// One host thread = one warp of one lane, with the kernel's per-warp state.
std::unique_ptr<WarpSmem> new_warp() {
  auto W = std::make_unique<WarpSmem>();
  memset(W.get(), 0, sizeof(WarpSmem));
  W->icache_def = ~0u;
  W->pool_cap = POOL;
  lane_init(W.get(), 0);
  return W;
}

void give(Emu* E, WarpSmem& W, unsigned& bot, unsigned cnt, int cur) {
  std::vector<ull> v;
  for (unsigned k = 0; k < cnt; k++) {
    unsigned i = (bot + k) & (SCAP - 1);
    v.push_back(W.stk[2 * i]);
    v.push_back(W.stk[2 * i + 1]);
  }
  bot += cnt;
  atom_add(reinterpret_cast<ull*>(&E->nets[cur].pending), 1ull);
  std::lock_guard<std::mutex> g(E->mu);
  E->queue.push_back({unsigned(cur), std::move(v)});
}

// One lane's share of work, like a reducer warp: a shared-memory stack plus
// an overflow stack.  The stack a step may push into is kept tiny (`ring`
// slots) so that pushes keep spilling into the overflow stack, whose own
// small capacity sends the rest to the shared queue -- the paths a reducer
// warp takes only under a burst of redexes.
void worker(Emu* E, unsigned share_min, unsigned ring, unsigned spill_cap, unsigned index) {
  g_emu = E;
  auto W = new_warp();
  // Every other lane has no reuse pool: its reclaimed nodes all go through
  // its free list and, in batches, the shared free stack.
  if (index & 1) W->pool_cap = 0;
  std::vector<ull> spill(2 * size_t(spill_cap) + 2), bigregs(32 * MAX_REGS);
  W->sp = spill_cap ? spill.data() : nullptr;
  W->bigregs = bigregs.data();
  W->sp_cap = spill_cap;
  W->sp_n = 0;
  Ctx c{W.get(), 0, 0};
  unsigned top = 0, bot = 0;
  int cur = -1;
  ull pops = 0;  // redexes this lane interacted (Net::reduce's count)
  for (;;) {
    if (ld_gpu32(&E->C.error)) break;
    if (W->sp_n && top - bot < 4) {  // refill from the overflow stack's newest
      unsigned m = std::min(W->sp_n, unsigned(SCAP - HEADROOM) - (top - bot));
      for (unsigned i = 0; i < m; i++) {
        unsigned k = (top + i) & (SCAP - 1);
        W->stk[2 * k] = W->sp[2 * (W->sp_n - m + i)];
        W->stk[2 * k + 1] = W->sp[2 * (W->sp_n - m + i) + 1];
      }
      top += m;
      W->sp_n -= m;
    }
    if (top == bot) {
      if (cur >= 0) {
        flush(*W, E->nets[cur]);
        long long old = (long long)atom_add(reinterpret_cast<ull*>(&E->nets[cur].pending), ~0ull);
        if (old == 1) atom_add(reinterpret_cast<ull*>(&E->C.nets_left), ~0ull);
        cur = -1;
      }
      std::vector<ull> got;
      {
        std::lock_guard<std::mutex> g(E->mu);
        if (!E->queue.empty()) {
          cur = int(E->queue.front().first);
          got = std::move(E->queue.front().second);
          E->queue.pop_front();
        }
      }
      if (cur < 0) {
        if (ld_gpu64s(&E->C.nets_left) <= 0) break;
        if (globaltimer() > E->C.deadline) {
          run_fail(c.net, HVM64_ERR_TIMEOUT, 1);
          break;
        }
        std::this_thread::yield();
        continue;
      }
      c.net = unsigned(cur);
      bot = 0;
      top = unsigned(got.size() / 2);
      for (size_t k = 0; k < got.size(); k++) W->stk[k] = got[k];
    }
    while (top - bot > unsigned(SCAP - HEADROOM)) give(E, *W, bot, 32, cur);
    unsigned i = (top - 1) & (SCAP - 1);
    ull a = W->stk[2 * i], b = W->stk[2 * i + 1];
    top -= 1;
    W->ring_cnt = 0;
    W->ring_base = top;
    W->ring_cap = std::min(unsigned(SCAP) - (top - bot), ring);
    interact(c, a, b);
    pops++;
    settle(c);
    {
      unsigned cnt = W->ring_cnt;
      top += std::min(cnt, W->ring_cap);
      W->sp_n += spilled_of(W.get(), cnt);
    }
    // merge reclaimed nodes into the pool
    int pn = std::max(W->pool_n, 0), fn = std::min(W->freed_n, POOL), mv = std::min(fn, POOL - pn);
    for (int k = 0; k < mv; k++) W->pool[pn + k] = W->freed[k];
    for (int k = mv; k < fn; k++) {
      free_list_push(c.net, &W->ovf[0], W->freed[k]);
    }
    W->pool_n = pn + mv;
    W->freed_n = 0;
    if (top - bot + W->sp_n >= share_min) {
      bool want;
      {
        std::lock_guard<std::mutex> g(E->mu);
        want = E->queue.size() < 4;
      }
      if (want && W->sp_n >= 8) {  // the overflow stack's newest first
        std::vector<ull> v(W->sp + 2 * (W->sp_n - 8), W->sp + 2 * W->sp_n);
        W->sp_n -= 8;
        atom_add(reinterpret_cast<ull*>(&E->nets[cur].pending), 1ull);
        std::lock_guard<std::mutex> g(E->mu);
        E->queue.push_back({unsigned(cur), std::move(v)});
      } else if (want && top - bot >= 2) {
        give(E, *W, bot, std::min(32u, (top - bot) / 2), cur);
      }
    }
  }
  if (cur >= 0) flush(*W, E->nets[cur]);
  atom_add(&E->C.stat_lanes, pops);
}

// Boots Def `prog` of `book` in a fresh emulated device and reduces it on
// `threads` host threads.  With `capture` (pre-reduce), the boot skips the
// expansion agent and inert Defs record their redexes there.
std::unique_ptr<Emu> emu_reduce(const Book& book, uint32_t prog, unsigned threads, unsigned ring,
                                unsigned spill_cap, unsigned share_min, uint64_t heap_bytes, uint64_t chunk,
                                std::vector<ull>* capture) {
  auto Ep = std::make_unique<Emu>();
  Emu& E = *Ep;
#ifdef HVM_EMU_CHECK_ALLOC
  static std::vector<std::atomic<unsigned>> node_out;
  node_out = std::vector<std::atomic<unsigned>>(heap_bytes / 16);
  g_node_out = node_out.data();
  g_alloc_faults = 0;
#endif
  E.heap.assign(heap_bytes / 8, 0);
  E.nets.assign(1, NetState{});
  E.nets[0].prog = int(prog);
  E.C.bump = 1;
  E.C.heap_nodes = heap_bytes / 16;
  E.C.heap_bytes = heap_bytes;
  E.C.chunk_nodes = chunk;
  E.C.reuse_mark = 0;  // free nodes shared between threads from the start
  E.C.spin_limit = 1ull << 26;
  E.C.deadline = globaltimer() + 120ull * 1000000000ull;
  E.P.heap = E.heap.data();
  E.P.heap_bytes = heap_bytes;
  E.P.ctrl = &E.C;
  E.P.nets = E.nets.data();
  E.P.nnets = 1;
  E.P.defs = book.defs.data();
  E.P.instrs = book.instrs.data();
  E.P.labbits = reinterpret_cast<const ull*>(book.labbits.data());
  E.P.ndefs = unsigned(book.defs.size());
  E.P.ovf_flush = OVF_FLUSH;
#ifdef HVM_GEN_INCLUDE
  E.P.gen = book.defs.size() >= HVM_GEN_NDEFS && defs_hash(book, HVM_GEN_NDEFS) == HVM_GEN_HASH;
#endif
  if (capture) {
    E.P.no_expand = 1;
    E.P.capture = capture->data();
    E.P.capture_cap = unsigned(capture->size() / 2);
  }
  g_P = E.P;
  // boot (the boot kernel's steps, one thread)
  g_emu = &E;
  {
    auto W = new_warp();
    std::vector<ull> boot_regs(32 * MAX_REGS);
    W->bigregs = boot_regs.data();
    W->ring_cap = 0;  // boot redexes go straight to the shared queue
    Ctx c{W.get(), 0, 0};
    ull root = alloc(c);
    if (!(book.defs[prog].flags & DEF_EXPR)) W->rw[RW_DREF]++;
    run_def(c, prog, pvar(root));
    settle(c);
    if (!g_P.no_expand) {
      root = expand(c, root);
      settle(c);
    }
    E.nets[0].root = root;
    flush(*W, E.nets[0]);
    if (E.nets[0].pending > 0) E.C.nets_left = 1;
  }
  std::vector<std::thread> th;
  for (unsigned t = 0; t < threads; t++) th.emplace_back(worker, &E, share_min, std::max(1u, ring), spill_cap, t);
  for (auto& t : th) t.join();
  return Ep;
}
}  // namespace

// The emulation ships an overflowing redex to the shared queue.
void hvm::dev::push_overflow(unsigned net, ull a, ull b) {
  Emu* E = g_emu;
  atom_add(reinterpret_cast<ull*>(&g_P.nets[net].pending), 1ull);
  std::lock_guard<std::mutex> g(E->mu);
  E->queue.push_back({net, std::vector<ull>{a, b}});
}

extern "C" int hvm64emu_run(const char* book_text, const char* entry, unsigned threads, unsigned ring,
                            unsigned spill_cap, unsigned share_min, uint64_t heap_bytes, uint64_t chunk,
                            char** out_text, uint64_t* rw, char* err, size_t errcap) {
  try {
    Book book;
    std::string src(book_text);
    with_big_stack([&] { book.load(parse_book(src)); });
    auto it = book.ids.find(entry);
    if (it == book.ids.end()) throw Error(HVM64_ERR_BAD_INPUT, "no entry");
    auto Ep = emu_reduce(book, it->second, threads, ring, spill_cap, share_min, heap_bytes, chunk, nullptr);
    Emu& E = *Ep;
    if (E.C.error) {
      snprintf(err, errcap, "device error %d info 0x%llx", E.C.error, (unsigned long long)E.C.error_info);
      return E.C.error;
    }
#ifdef HVM_EMU_CHECK_ALLOC
    if (g_alloc_faults.load()) {
      snprintf(err, errcap, "%llu nodes handed out twice or reclaimed twice",
               (unsigned long long)g_alloc_faults.load());
      return HVM64_ERR_BAD_ADDR;
    }
#endif
    for (int k = 0; k < 5; k++) rw[k] = E.nets[0].rw[k];
    std::string txt;
    with_big_stack([&] { txt = readback(book, reinterpret_cast<const uint64_t*>(E.heap.data()), E.heap.size(), E.nets[0].root); });
    // The device-side gather (the words readback loads, in its order) must
    // read back to the same text.
    {
      std::vector<ull> pairs(2 * 4096), stk(256);
      bool deep = false;
      unsigned n = gather_walk(0, E.nets[0].root, pairs.data(), 4096, stk.data(), 256, &deep);
      if (!deep && n > 4096) {
        pairs.assign(2 * size_t(n), 0);
        n = gather_walk(0, E.nets[0].root, pairs.data(), n, stk.data(), 256, &deep);
      }
      if (!deep) {
        // The batch gather's split walk (the top expanded by one thread, the
        // subtrees walked separately) must give the same pairs in the same order.
        {
          std::vector<ull> tw(GTOP), tv(GTOP), tsz(GTOP), sp(256);
          std::vector<unsigned> tref(GTOP), tc(GTASKS);
          std::vector<unsigned char> tkind(GTOP);
          GatherTop T{tw.data(), tv.data(), tsz.data(), tref.data(), tkind.data(), 0, 0};
          gather_top(0, E.nets[0].root, T);
          bool sdeep = false;
          for (unsigned k = 0; k < T.nt; k++)
            if (tkind[k] == GATHER_SUB) tc[tref[k]] = gather_walk(0, tw[k], nullptr, 0, sp.data(), 256, &sdeep);
          ull total = gather_sizes(T, tc.data());
          if (!sdeep) {
            if (total != n) throw Error(HVM64_ERR_BAD_INPUT, "split gather counts " + std::to_string(total) +
                                                                 " pairs, the walk " + std::to_string(n));
            std::vector<ull> split(2 * size_t(n) + 2, 0);
            gather_place(T, tc.data(), split.data());
            for (unsigned k = 0; k < T.nt; k++)
              if (tkind[k] == GATHER_SUB)
                gather_walk(0, tw[k], split.data() + 2 * tsz[k], tc[tref[k]], sp.data(), 256, &sdeep);
            for (size_t k = 0; k < 2 * size_t(n); k++)
              if (split[k] != pairs[k]) throw Error(HVM64_ERR_BAD_INPUT, "split gather differs at " + std::to_string(k));
          }
        }
        std::string g;
        with_big_stack([&] { g = readback_pairs(book, reinterpret_cast<const uint64_t*>(pairs.data()), n,
                                                E.heap.size(), E.nets[0].root); });
        if (g != txt) throw Error(HVM64_ERR_BAD_INPUT, "gathered readback differs: " + g.substr(0, 80));
        // out of order (the reader's address map instead of its cursor)
        for (size_t i = 0; i + 1 < n; i += 2) {
          std::swap(pairs[2 * i], pairs[2 * (i + 1)]);
          std::swap(pairs[2 * i + 1], pairs[2 * (i + 1) + 1]);
        }
        with_big_stack([&] { g = readback_pairs(book, reinterpret_cast<const uint64_t*>(pairs.data()), n,
                                                E.heap.size(), E.nets[0].root); });
        if (g != txt) throw Error(HVM64_ERR_BAD_INPUT, "shuffled gathered readback differs: " + g.substr(0, 80));
        // many nets at once on several host threads (here: the same net 8 times,
        // plus one not gathered)
        std::vector<uint64_t> offs(9, 0), roots(9, E.nets[0].root);
        std::vector<unsigned> counts(9, n);
        counts[4] = ~0u;
        auto many = readback_pairs_many(book, reinterpret_cast<const uint64_t*>(pairs.data()), offs.data(),
                                        counts.data(), roots.data(), 9, E.heap.size(), 4);
        for (size_t i = 0; i < 9; i++) {
          if (i == 4 ? (many[i].ok || !many[i].text.empty()) : (!many[i].ok || many[i].text != txt))
            throw Error(HVM64_ERR_BAD_INPUT, "parallel gathered readback differs at " + std::to_string(i));
        }
      }
    }
    *out_text = strdup(txt.c_str());
    return 0;
  } catch (Error& e) {
    snprintf(err, errcap, "%s", e.msg.c_str());
    return e.code;
  } catch (std::exception& e) {
    snprintf(err, errcap, "%s", e.what());
    return HVM64_ERR_BAD_INPUT;
  }
}

// Book::pre_reduce with every Def reduced by the emulated device (the same
// host driver, hvm::pre_reduce, that the CUDA library uses).  `skip` holds
// '\n'-separated names; rw[0..5]; not_normal gets one name per line.
extern "C" int hvm64emu_pre_reduce(const char* book_text, const char* skip, uint64_t max_rwts, unsigned threads,
                                   unsigned ring, unsigned spill_cap, uint64_t heap_bytes, uint64_t chunk,
                                   char** out_text, uint64_t* rw, char** not_normal, char* err, size_t errcap) {
  try {
    AstBook ast;
    Book book;
    std::string src(book_text);
    with_big_stack([&] {
      ast = parse_book(src);
      book.load(ast, true);
    });
    std::set<std::string> sk;
    std::string names = skip ? skip : "";
    for (size_t s0 = 0; s0 < names.size();) {
      size_t e = names.find('\n', s0);
      if (e == std::string::npos) e = names.size();
      if (e > s0) sk.insert(names.substr(s0, e - s0));
      s0 = e + 1;
    }
    PreReduceOut res;
    with_big_stack([&] {
      res = pre_reduce(ast, book, sk, max_rwts, [&](uint32_t id) {
        std::vector<ull> cap(2 * 4096);
        auto E = emu_reduce(book, id, threads, ring, spill_cap, 16, heap_bytes, chunk, &cap);
        PreReduceRun r;
        r.status = E->C.error;
        r.pops = E->C.stat_lanes;
        for (int k = 0; k < 5; k++) r.rw[k] = E->nets[0].rw[k];
        if (r.status) {
          r.error = "device error " + std::to_string(r.status);
          return r;
        }
        // captured redexes after the net's own, ones with an eraser first
        std::vector<uint64_t> pairs;
        uint64_t n = std::min<uint64_t>(E->C.captured, cap.size() / 2);
        for (int pass = 0; pass < 2; pass++)
          for (uint64_t k = 0; k < n; k++)
            if ((cap[2 * k + 1] == PORT_ERA) == (pass == 0)) {
              pairs.push_back(cap[2 * k]);
              pairs.push_back(cap[2 * k + 1]);
            }
        r.text = readback_net(book, reinterpret_cast<const uint64_t*>(E->heap.data()), E->heap.size(),
                              E->nets[0].root, pairs.data(), pairs.size() / 2);
        return r;
      });
    });
    for (int k = 0; k < 5; k++) rw[k] = res.rw[k];
    *out_text = strdup(res.text.c_str());
    std::string nn;
    for (auto& n : res.not_normal) nn += n + "\n";
    *not_normal = strdup(nn.c_str());
    return 0;
  } catch (Error& e) {
    snprintf(err, errcap, "%s", e.msg.c_str());
    return e.code;
  } catch (std::exception& e) {
    snprintf(err, errcap, "%s", e.what());
    return HVM64_ERR_BAD_INPUT;
  }
}

// 1 when this build carries compiled Def functions that match `book_text`
// (a build with -DHVM_GEN_INCLUDE), else 0.
extern "C" int hvm64emu_compiled_for(const char* book_text) {
#ifdef HVM_GEN_INCLUDE
  try {
    Book book;
    std::string src(book_text);
    with_big_stack([&] { book.load(parse_book(src)); });
    return book.defs.size() >= HVM_GEN_NDEFS && defs_hash(book, HVM_GEN_NDEFS) == HVM_GEN_HASH;
  } catch (...) {
    return 0;
  }
#else
  (void)book_text;
  return 0;
#endif
}
