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
#include <string>
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

void flush(Lane& L, NetState& ns) {
  for (int k = 0; k < NCOUNT; k++) {
    if (L.rw[k]) atom_add(&ns.rw[k], L.rw[k]);
    L.rw[k] = 0;
  }
}

void worker(Emu* E, unsigned budget, unsigned share_min) {
  g_emu = E;
  Lane L(E->P);
  std::vector<ull> st;
  int cur = -1;
  for (;;) {
    if (ld_gpu32(&E->C.error)) break;
    if (st.empty()) {
      if (cur >= 0) {
        flush(L, E->nets[cur]);
        long long old = (long long)atom_add(reinterpret_cast<ull*>(&E->nets[cur].pending), ~0ull);
        if (old == 1) atom_add(reinterpret_cast<ull*>(&E->C.nets_left), ~0ull);
        cur = -1;
      }
      bool got = false;
      {
        std::lock_guard<std::mutex> g(E->mu);
        if (!E->queue.empty()) {
          cur = int(E->queue.front().first);
          st = std::move(E->queue.front().second);
          E->queue.pop_front();
          got = true;
        }
      }
      if (!got) {
        if (ld_gpu64s(&E->C.nets_left) <= 0) break;
        if (globaltimer() > E->C.deadline) {
          L.fail(HVM64_ERR_TIMEOUT, 1);
          break;
        }
        std::this_thread::yield();
        continue;
      }
      L.net = unsigned(cur);
    }
    for (unsigned k = 0; k < budget && !st.empty(); k++) {
      ull b = st.back();
      st.pop_back();
      ull a = st.back();
      st.pop_back();
      L.interact(a, b);
      L.settle();
      for (int i = 0; i < L.pn; i++) {
        st.push_back(L.pb[2 * i]);
        st.push_back(L.pb[2 * i + 1]);
      }
      L.pn = 0;
    }
    // Share the oldest half when the queue runs dry.
    if (st.size() / 2 >= share_min) {
      std::lock_guard<std::mutex> g(E->mu);
      if (E->queue.size() < 4) {
        size_t half = (st.size() / 4) * 2;
        std::vector<ull> give(st.begin(), st.begin() + long(half));
        st.erase(st.begin(), st.begin() + long(half));
        atom_add(reinterpret_cast<ull*>(&E->nets[cur].pending), 1ull);
        E->queue.push_back({unsigned(cur), std::move(give)});
      }
    }
  }
  if (cur >= 0) flush(L, E->nets[cur]);
}
}  // namespace

// The emulation ships a full lane buffer to the shared queue.
void hvm::dev::Lane::overflow() {
  Emu* E = g_emu;
  atom_add(reinterpret_cast<ull*>(&P.nets[net].pending), 1ull);
  std::vector<ull> v(pb, pb + 2 * pn);
  {
    std::lock_guard<std::mutex> g(E->mu);
    E->queue.push_back({net, std::move(v)});
  }
  pn = 0;
}

extern "C" int hvm64emu_run(const char* book_text, const char* entry, unsigned threads, unsigned budget,
                            unsigned share_min, uint64_t heap_bytes, uint64_t chunk, char** out_text, uint64_t* rw,
                            char* err, size_t errcap) {
  try {
    Book book;
    std::string src(book_text);
    with_big_stack([&] { book.load(parse_book(src)); });
    auto it = book.ids.find(entry);
    if (it == book.ids.end()) throw Error(HVM64_ERR_BAD_INPUT, "no entry");
    Emu E;
    E.heap.assign(heap_bytes / 8, 0);
    E.nets.assign(1, NetState{});
    E.nets[0].prog = int(it->second);
    E.C.bump = 1;
    E.C.heap_nodes = heap_bytes / 16;
    E.C.heap_bytes = heap_bytes;
    E.C.chunk_nodes = chunk;
    E.C.spin_limit = 1ull << 26;
    E.C.deadline = globaltimer() + 120ull * 1000000000ull;
    E.P.heap = E.heap.data();
    E.P.ctrl = &E.C;
    E.P.nets = E.nets.data();
    E.P.nnets = 1;
    E.P.defs = book.defs.data();
    E.P.instrs = book.instrs.data();
    E.P.labbits = reinterpret_cast<const ull*>(book.labbits.data());
    E.P.ndefs = unsigned(book.defs.size());
    // boot (the boot kernel's steps, one thread)
    g_emu = &E;
    {
      Lane L(E.P);
      L.net = 0;
      ull root = L.alloc();
      if (!(book.defs[it->second].flags & 1)) L.rw[RW_DREF]++;
      L.run_def(it->second, pvar(root));
      L.settle();
      root = L.expand(root);
      L.settle();
      E.nets[0].root = root;
      if (L.pn) L.overflow();
      flush(L, E.nets[0]);
      if (E.nets[0].pending > 0) E.C.nets_left = 1;
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < threads; t++) th.emplace_back(worker, &E, budget, share_min);
    for (auto& t : th) t.join();
    if (E.C.error) {
      snprintf(err, errcap, "device error %d info 0x%llx", E.C.error, (unsigned long long)E.C.error_info);
      return E.C.error;
    }
    for (int k = 0; k < 5; k++) rw[k] = E.nets[0].rw[k];
    std::string txt;
    with_big_stack([&] { txt = readback(book, reinterpret_cast<const uint64_t*>(E.heap.data()), E.heap.size(), E.nets[0].root); });
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
