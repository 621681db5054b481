// Device runtime of the B200 interaction-net reducer.
//
// Heap: one HBM arena of 16-byte nodes (two 8-byte port words), addressed by
// byte offset, so a node's other half is `addr ^ 8` exactly as in the
// reference (runtime/src/addr.rs:36-50).  Node 0 is reserved (the free-list
// terminator and a scratch target for guarded accesses).
//
// Every heap access is a strong GPU-scope operation (ld/st.relaxed.gpu or an
// atomic), so no SM reads a stale L1 copy of a word another SM changed.  A
// freshly allocated node is filled with LOCK and fenced before its address
// can escape; readers treat LOCK as "not ready yet" and wait, which is the
// reference's own protocol (runtime/src/wire.rs:67-75).
//
// Every wait is bounded: after `spin_limit` polls, or when another lane has
// already failed, the wait gives up, the run's error word is set and all
// warps drain and exit.  Every heap address is bounds-checked; an address
// outside the arena sets HVM64_ERR_BAD_ADDR and is redirected to node 0, so a
// protocol fault can never become a memory fault.
#pragma once
#include <stdint.h>

#ifndef __CUDACC__
#include <atomic>
#include <chrono>
#include <thread>
#endif

#include "host.hpp"
#include "hvm64.h"
#include "num.h"

namespace hvm {
namespace dev {

typedef unsigned long long ull;

constexpr int WARPS = 4;            // warps per reducer block
constexpr int THREADS = WARPS * 32;
constexpr int SCAP = 512;           // per-warp shared-memory redex stack (power of two)
constexpr int HEADROOM = 192;       // stack slots kept free for the redexes of one step
constexpr int CHUNK = 32;           // redexes per global-queue slot
constexpr int POOL = 128;           // per-warp pool of free nodes ready for reuse
constexpr unsigned SMALL_REGS = 12; // Defs with at most this many registers use shared memory

constexpr ull P_ERA = 2;
constexpr ull P_FREE = 0x8000000000000000ull;
constexpr ull P_LOCK = 0xFFFFFFFFFFFFFFF0ull;
constexpr ull P_GONE = 0xFFFFFFFFFFFFFFFFull;
constexpr ull A_MASK = 0x0000FFFFFFFFFFF8ull;
constexpr ull X_BIT = 1ull << 47;  // expansion-agent Ref ports

enum : int { RW_ANNI = 0, RW_COMM, RW_ERAS, RW_DREF, RW_OPER };

// Global control block.  Hot counters sit on their own 128-byte lines.
struct Ctrl {
  ull bump;        // next never-used node index
  ull heap_nodes;
  ull heap_bytes;
  ull chunk_nodes;
  ull spin_limit;
  ull deadline;    // %globaltimer ns
  ull donate_min;
  ull lane_budget;
  ull q_mask;
  int error;
  int error_net;
  ull error_info;
  ull pad0[6];
  long long nets_left;
  ull pad1[15];
  long long hungry;
  ull pad2[15];
  ull q_head;
  ull pad3[15];
  ull q_tail;
  ull pad4[15];
  ull stat_donated, stat_spilled, stat_overflow, stat_taken;
  ull stat_steps, stat_lanes, stat_busy_cycles, stat_idle_cycles;
  ull timeout_ns;  // per launch: each warp's deadline is its start + timeout_ns
  ull stat_g_steps[8], stat_g_cycles[8];  // steps by number of distinct rule classes among lanes
};

constexpr int NCOUNT = 8;  // rw[5] then comm22, dref_nodes, dref_links
enum : int { EX_COMM22 = 5, EX_DNODES, EX_DLINKS };

struct NetState {  // 96 bytes
  ull root;            // byte offset of the root wire
  long long pending;   // warps holding this net's work + queued chunks
  ull rw[NCOUNT];
  int prog;            // DevDef index of the boot program
  int status;
};

struct Slot {  // 544 bytes: one chunk of up to 32 redexes of one net
  ull seq;
  unsigned net;
  unsigned count;
  ull pad[2];
  ull r[2 * CHUNK];
};

struct Params {
  ull* heap;
  ull heap_bytes;
  Ctrl* ctrl;
  NetState* nets;
  unsigned nnets;
  Slot* q;
  const DevDef* __restrict__ defs;
  const DevInstr* __restrict__ instrs;
  const ull* __restrict__ labbits;
  unsigned ndefs;
};

// ---- platform layer ------------------------------------------------------------
// The runtime below is written against these few operations.  Under nvcc
// they are strong GPU-scope PTX accesses and CUDA atomics; under a host
// compiler (the CPU emulation harness the tests build from this same file)
// they are std::atomic_ref operations, so the protocol logic can be exercised
// with many host threads.
#ifdef __CUDACC__
#define HVM_DEV __device__
#define HVM_INL __device__ __forceinline__
__device__ __forceinline__ ull ld_gpu(const ull* p) {
  ull v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_gpu(ull* p, ull v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int ld_gpu32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ ull globaltimer() {
  ull t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ ull atom_exch(ull* p, ull v) { return atomicExch(p, v); }
__device__ __forceinline__ ull atom_cas(ull* p, ull e, ull v) { return atomicCAS(p, e, v); }
__device__ __forceinline__ ull atom_add(ull* p, ull v) { return atomicAdd(p, v); }
__device__ __forceinline__ int atom_cas32(int* p, int e, int v) { return atomicCAS(p, e, v); }
__device__ __forceinline__ unsigned atom_add_u32(unsigned* p, unsigned v) { return atomicAdd(p, v); }
__device__ __forceinline__ int atom_add_i32(int* p, int v) { return atomicAdd(p, v); }
__device__ __forceinline__ void mem_fence() { __threadfence(); }
__device__ __forceinline__ void pause_brief() { __nanosleep(64); }
// LOCK-fill nodes [s, s+n) with 16-byte stores.
__device__ __forceinline__ void lock_fill(ull* H, ull s, ull n) {
  ulonglong2* c = reinterpret_cast<ulonglong2*>(H) + s;
  for (ull k = 0; k < n; k++) c[k] = make_ulonglong2(P_LOCK, P_LOCK);
}
#else
#define HVM_DEV
#define HVM_INL inline
#ifdef HVM_EMU_STRESS
// Test builds only: yield at random inside memory operations to widen race
// windows.
inline void emu_jitter() {
  thread_local unsigned x = 0x9E3779B9u ^ unsigned(std::hash<std::thread::id>{}(std::this_thread::get_id()));
  x ^= x << 13; x ^= x >> 17; x ^= x << 5;
  if ((x & 31) == 0) std::this_thread::yield();
}
#else
inline void emu_jitter() {}
#endif
inline ull ld_gpu(const ull* p) {
  emu_jitter();
  return std::atomic_ref<ull>(*const_cast<ull*>(p)).load(std::memory_order_acquire);
}
inline void st_gpu(ull* p, ull v) {
  emu_jitter();
  std::atomic_ref<ull>(*p).store(v, std::memory_order_release);
}
inline int ld_gpu32(const int* p) {
  return std::atomic_ref<int>(*const_cast<int*>(p)).load(std::memory_order_acquire);
}
inline ull globaltimer() {
  return ull(std::chrono::duration_cast<std::chrono::nanoseconds>(
                 std::chrono::steady_clock::now().time_since_epoch()).count());
}
inline ull atom_exch(ull* p, ull v) {
  emu_jitter();
  return std::atomic_ref<ull>(*p).exchange(v);
}
inline ull atom_cas(ull* p, ull e, ull v) {
  emu_jitter();
  std::atomic_ref<ull>(*p).compare_exchange_strong(e, v);
  return e;
}
inline ull atom_add(ull* p, ull v) { return std::atomic_ref<ull>(*p).fetch_add(v); }
inline int atom_cas32(int* p, int e, int v) {
  std::atomic_ref<int>(*p).compare_exchange_strong(e, v);
  return e;
}
inline unsigned atom_add_u32(unsigned* p, unsigned v) { return std::atomic_ref<unsigned>(*p).fetch_add(v); }
inline int atom_add_i32(int* p, int v) { return std::atomic_ref<int>(*p).fetch_add(v); }
inline void mem_fence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void pause_brief() { std::this_thread::yield(); }
inline void lock_fill(ull* H, ull s, ull n) {
  for (ull k = 0; k < 2 * n; k++) st_gpu(H + 2 * s + k, P_LOCK);
}
#endif
HVM_INL long long ld_gpu64s(const long long* p) {
  return (long long)ld_gpu(reinterpret_cast<const ull*>(p));
}

// ---- ports (runtime/src/port.rs) ---------------------------------------------
HVM_INL unsigned ptag(ull p) { return unsigned(p & 7); }
HVM_INL unsigned plab(ull p) { return unsigned(p >> 48); }
HVM_INL ull paddr(ull p) { return p & A_MASK; }
HVM_INL ull mkport(unsigned tag, unsigned lab, ull addr) { return (ull(lab) << 48) | addr | tag; }
HVM_INL ull pvar(ull a) { return a | T_VAR; }
HVM_INL ull pred(ull a) { return a | T_RED; }
HVM_INL bool principal(ull p) { return ptag(p) >= T_REF; }
HVM_INL bool skippable(ull p) {  // port.rs:205-207
  return ptag(p) == T_NUM || (ptag(p) == T_REF && plab(p) != 0xFFFF);
}
HVM_INL bool is_expand(ull p) { return ptag(p) == T_REF && (p & X_BIT) != 0; }
// Trg (runtime/src/linker.rs:228-281): a wire is its address with the Red tag.
HVM_INL bool trg_is_wire(ull t) { return ptag(t) == T_RED; }

// Rule class of a redex, following interact()'s dispatch: the Def index for
// a Def call (calls of one Def run the same instruction stream), else a small
// code per rule.  Warps pick redexes of one class per step to stay convergent.
HVM_INL unsigned redex_class(ull a, ull b) {
  unsigned at = unsigned(a & 7), bt = unsigned(b & 7);
  if (at == T_REF && !(a & X_BIT) && a != P_ERA) return 64 + unsigned((a & A_MASK) >> 3);
  if (bt == T_REF && !(b & X_BIT) && b != P_ERA) return 64 + unsigned((b & A_MASK) >> 3);
  if ((a & X_BIT) || (b & X_BIT)) return 1;
  if (at == bt) return 2 + at;  // annihilation (or nilary pair)
  return 16 + at * 8 + bt;      // commutation / native ops
}

// VM register files: a warp's shared-memory block laid out [register][lane],
// or a local array for the rare Def needing more than SMALL_REGS.
struct StridedRegs {
  ull* base;
  unsigned stride;
  HVM_INL ull& operator[](unsigned i) const { return base[i * stride]; }
};

// Per-warp shared state of the reducer (one per warp; the CPU emulation
// harness gives each host thread one too).
struct WarpSmem {
  ull stk[2 * SCAP];          // redex stack (ring of SCAP pairs)
  ull regs[SMALL_REGS * 32];  // VM registers, [register][lane]
  ull pool[POOL];             // free nodes ready for reuse
  ull freed[POOL];            // nodes reclaimed during the current step
  ull sel[64];                // the redexes chosen for the current step
  ull rw[NCOUNT];             // counters of the warp's current net
  ull st_steps, st_lanes, st_busy, st_idle;
  unsigned ring_cnt;
  int pool_n;
  int freed_n;
  unsigned pad;
};

HVM_INL void count(ull* c, ull v) { atom_add(c, v); }

struct Lane {
  const Params& P;
  WarpSmem* W;      // this lane's warp state (sinks, pools, counters, VM registers)
  ull ovf;          // overflow free list (left word links; right word LOCK)
  ull bnext;        // pre-LOCKed bump chunk [bnext, bend) in node indices
  ull bend;
  unsigned allocs;  // nodes allocated by this lane (for the DREF statistics)
  unsigned net;
  unsigned lane;
  unsigned ring_base;  // this step's pushes go to stack slots ring_base + k
  unsigned ring_cap;
  unsigned pool_cap;   // 0: no reuse pool (reclaimed nodes go to `ovf`)
  // Words freed alone by the current interaction (0 = empty slot).
  ull fw0, fw1, fw2, fw3;

  HVM_DEV Lane(const Params& p, WarpSmem* w, unsigned ln)
      : P(p), W(w), ovf(0), bnext(0), bend(0), allocs(0), net(0), lane(ln), ring_base(0), ring_cap(0),
        pool_cap(POOL), fw0(0), fw1(0), fw2(0), fw3(0) {}

  HVM_DEV void fail(int code, ull info) {
    if (atom_cas32(&P.ctrl->error, 0, code) == 0) {
      P.ctrl->error_info = info;
      P.ctrl->error_net = int(net);
    }
  }
  HVM_DEV bool failed() const { return ld_gpu32(&P.ctrl->error) != 0; }

  // One poll of a bounded wait; false = abandon the wait.
  HVM_DEV bool spin(unsigned& it) {
    ++it;
    if ((it & 63) == 0) {
      if (failed()) return false;
      if (it > P.ctrl->spin_limit) {
        fail(HVM64_ERR_TIMEOUT, 0);
        return false;
      }
      pause_brief();
    }
    return true;
  }

  HVM_DEV ull* at(ull a) {
    if (a >= P.heap_bytes) {
      fail(HVM64_ERR_BAD_ADDR, a);
      a = 0;
    }
    return P.heap + (a >> 3);
  }
  HVM_DEV ull load(ull a) { return ld_gpu(at(a)); }
  HVM_DEV void store(ull a, ull v) { st_gpu(at(a), v); }
  HVM_DEV ull swap(ull a, ull v) { return atom_exch(at(a), v); }
  HVM_DEV ull cas(ull a, ull e, ull v) { return atom_cas(at(a), e, v); }

  // wire.rs:342-350
  HVM_DEV ull relock(ull w) {
    unsigned it = 0;
    for (;;) {
      ull got = swap(w, P_LOCK);
      if (got != P_LOCK) return got;
      if (!spin(it)) return P_ERA;
    }
  }
  HVM_DEV ull lock_target(ull w) {
    ull got = swap(w, P_LOCK);
    return got != P_LOCK ? got : relock(w);
  }

  // ---- allocator -------------------------------------------------------------
  // The reference's allocator (runtime/src/allocator.rs:73-110) writes LOCK
  // into both words of every node it hands out and links a node into a
  // free list once both halves are FREE.  Here a node is LOCK-filled when it
  // becomes free (or when its bump chunk is taken) and that fill is fenced
  // before the node is handed out again, so alloc() itself touches no heap
  // memory.  A node whose two halves are both freed by the same interaction
  // is reclaimed without reading the other half; otherwise the reference's
  // store-FREE / read-other-half / CAS sequence decides which lane reclaims.
  HVM_DEV void recycle(ull node) {
    int k = pool_cap ? atom_add_i32(&W->freed_n, 1) : POOL;
    if (k < int(pool_cap)) {
      W->freed[k] = node;
    } else {
      store(node, ovf);  // right word already LOCK
      ovf = node;
    }
  }
  HVM_DEV bool fw_take(ull x) {
    if (fw0 == x) { fw0 = 0; return true; }
    if (fw1 == x) { fw1 = 0; return true; }
    if (fw2 == x) { fw2 = 0; return true; }
    if (fw3 == x) { fw3 = 0; return true; }
    return false;
  }
  HVM_DEV void fw_add(ull a) {
    if (!fw0) fw0 = a;
    else if (!fw1) fw1 = a;
    else if (!fw2) fw2 = a;
    else if (!fw3) fw3 = a;
    else {
      settle();
      fw0 = a;
    }
  }
  HVM_DEV void half_free(ull a) {
    if (a != 0 && fw_take(a ^ 8)) {  // both halves freed by this interaction: no one else can claim the node
      ull l = a & ~8ull;
      store(l, P_LOCK);
      store(l | 8, P_LOCK);
      recycle(l);
      return;
    }
    store(a, P_FREE);
    fw_add(a);
  }
  // A word freed alone: a node found fully free is claimed by CAS on its left
  // word, then kept only if its right word is still free -- between the load
  // and the CAS the node may have been reclaimed by the other half's owner,
  // reused, and half-freed again (ABA); then the left word is handed back.
  HVM_DEV void claim(ull w, ull other) {
    if (!w || other != P_FREE) return;
    ull l = w & ~8ull;
    if (cas(l, P_FREE, P_LOCK) != P_FREE) return;
    if (load(l | 8) == P_FREE) {
      store(l | 8, P_LOCK);
      recycle(l);
    } else {
      store(l, P_FREE);
    }
  }
  // End of an interaction: look at the other half of every word freed alone
  // (the loads are in flight together).
  HVM_DEV void settle() {
    ull o0 = fw0 ? load(fw0 ^ 8) : 0, o1 = fw1 ? load(fw1 ^ 8) : 0;
    ull o2 = fw2 ? load(fw2 ^ 8) : 0, o3 = fw3 ? load(fw3 ^ 8) : 0;
    claim(fw0, o0);
    claim(fw1, o1);
    claim(fw2, o2);
    claim(fw3, o3);
    fw0 = fw1 = fw2 = fw3 = 0;
  }
  HVM_DEV ull alloc() {
    allocs++;
    if (pool_cap) {
      int k = atom_add_i32(&W->pool_n, -1) - 1;
      if (k >= 0) return W->pool[k];
    }
    if (ovf != 0) {
      ull a = ovf;
      ovf = load(a);
      store(a, P_LOCK);
      mem_fence();
      return a;
    }
    if (bnext == bend) {
      ull n = P.ctrl->chunk_nodes;
      ull s = atom_add(&P.ctrl->bump, n);
      if (s + n > P.ctrl->heap_nodes) {
        fail(HVM64_ERR_OOM, s);
        return 0;
      }
      lock_fill(P.heap, s, n);
      mem_fence();  // LOCK is visible before any of these nodes escapes
      bnext = s;
      bend = s + n;
    }
    return (bnext++) << 4;
  }

  // ---- redex pushes ----------------------------------------------------------
  HVM_DEV void overflow_one(ull a, ull b);  // platform driver: ship one redex to shared work
  HVM_DEV void push(ull a, ull b) {
    unsigned k = ring_cap ? atom_add_u32(&W->ring_cnt, 1u) : 0u;
    if (k < ring_cap) {
      unsigned i = (ring_base + k) & unsigned(SCAP - 1);
      W->stk[2 * i] = a;
      W->stk[2 * i + 1] = b;
    } else {
      overflow_one(a, b);
    }
  }
  // linker.rs:70-85
  HVM_DEV void redux(ull a, ull b) {
    if (skippable(a) && skippable(b)) count(&W->rw[RW_ERAS], 1);
    else push(a, b);
  }

  // ---- linker (runtime/src/linker.rs:25-203) --------------------------------
  HVM_DEV void half_link_port_port(ull a, ull b) {
    if (ptag(a) == T_VAR) store(paddr(a), b);
  }
  HVM_DEV void link_port_port(ull a, ull b) {
    if (principal(a) && principal(b)) {
      redux(a, b);
    } else {
      half_link_port_port(a, b);
      half_link_port_port(b, a);
    }
  }
  HVM_DEV void link_wire_wire(ull aw, ull bw) {
    // Lock order as in the reference: a lane waiting on `aw` must not hold
    // `bw`, or a lane resolving a redirect through `bw` could wait on it.
    ull ap = lock_target(aw);
    ull bp = lock_target(bw);
    if (principal(ap) && principal(bp)) {
      half_free(aw);
      half_free(bw);
      redux(ap, bp);
    } else {
      half_link_wire_port(ap, aw, bp);
      half_link_wire_port(bp, bw, ap);
    }
  }
  HVM_DEV void link_wire_port(ull aw, ull bp) {
    ull ap = lock_target(aw);
    if (principal(ap) && principal(bp)) {
      half_free(aw);
      redux(ap, bp);
    } else {
      half_link_wire_port(ap, aw, bp);
      half_link_port_port(bp, ap);
    }
  }
  HVM_DEV void half_link_wire_port(ull ap, ull aw, ull bp) {
    if (ptag(ap) == T_VAR) {
      if (cas(paddr(ap), pvar(aw), bp) == pvar(aw)) {
        half_free(aw);
      } else if (ptag(bp) == T_VAR) {
        store(aw, pred(paddr(bp)));
      } else if (principal(bp)) {
        store(aw, bp);
        resolve_redirect_pri(ap, aw, bp);
      } else {
        fail(HVM64_ERR_BAD_PAIR, bp);
      }
    } else {
      half_free(aw);
    }
  }
  HVM_DEV void resolve_redirect_pri(ull ap, ull aw, ull bp) {
    unsigned it = 0;
    for (;;) {
      ull tw = paddr(ap);
      ull tp = load(tw);
      if (tp == P_LOCK) {
        if (!spin(it)) return;
        continue;
      }
      if (ptag(tp) == T_RED) {
        half_free(tw);
        ap = tp;
        continue;
      }
      if (ptag(tp) == T_VAR) {
        if (cas(tw, tp, bp) == tp) {
          tw = paddr(tp);
          tp = load(tw);
          unsigned it2 = 0;
          while (tp != P_LOCK && ptag(tp) == T_RED) {
            half_free(tw);
            tw = paddr(tp);
            tp = load(tw);
            if (!spin(it2)) return;
          }
          return;
        }
        if (!spin(it)) return;
        continue;
      }
      if (principal(tp) || tp == P_GONE) {
        ull xw = aw < tw ? aw : tw;
        ull yw = aw < tw ? tw : aw;
        ull xp = swap(xw, P_GONE);
        if (xp != P_GONE) {
          ull yp = swap(yw, P_GONE);
          redux(xp, yp);
        } else {
          half_free(xw);
          unsigned it3 = 0;
          while (cas(yw, P_GONE, P_LOCK) != P_GONE)
            if (!spin(it3)) return;
          half_free(yw);
        }
        return;
      }
      fail(HVM64_ERR_BAD_PAIR, tp);
      return;
    }
  }
  HVM_DEV void link_trg_port(ull a, ull b) {
    if (trg_is_wire(a)) link_wire_port(a, b);
    else link_port_port(a, b);
  }
  HVM_DEV void link_trg(ull a, ull b) {
    bool aw = trg_is_wire(a), bw = trg_is_wire(b);
    if (aw && bw) link_wire_wire(a, b);
    else if (aw) link_wire_port(a, b);
    else if (bw) link_wire_port(b, a);
    else link_port_port(a, b);
  }
  HVM_DEV ull trg_target(ull t) { return trg_is_wire(t) ? load(t) : t; }
  // The target of a Trg about to be consumed by a VM instruction.  A wire is
  // locked rather than read: every path of the instruction then either frees
  // that wire or links it at once (which would lock it first), so taking the
  // lock up front saves a round trip and changes nothing observable.
  HVM_DEV ull trg_take(ull t) { return trg_is_wire(t) ? lock_target(t) : t; }
  // link_trg_port for a Trg taken with trg_take (its target already known).
  HVM_DEV void link_taken(ull t, ull target, ull b) {
    if (!trg_is_wire(t)) return link_port_port(t, b);
    if (principal(target) && principal(b)) {
      half_free(t);
      redux(target, b);
    } else {
      half_link_wire_port(target, t, b);
      half_link_port_port(b, target);
    }
  }
  HVM_DEV void free_trg(ull t) {
    if (trg_is_wire(t)) half_free(t);
  }

  // ---- rules (runtime/src/interact.rs) ----------------------------------------
  HVM_DEV void anni2(ull a, ull b) {  // interact.rs:72-79
    count(&W->rw[RW_ANNI], 1);
    ull a1 = paddr(a), b1 = paddr(b);
    link_wire_wire(a1, b1);
    link_wire_wire(a1 ^ 8, b1 ^ 8);
  }
  HVM_DEV void comm22(ull a, ull b) {  // interact.rs:118-141
    count(&W->rw[RW_COMM], 1);
    count(&W->rw[EX_COMM22], 1);
    ull a1 = paddr(a), b1 = paddr(b);
    ull A1 = alloc(), A2 = alloc(), B1 = alloc(), B2 = alloc();
    unsigned ta = ptag(a), la = plab(a), tb = ptag(b), lb = plab(b);
    link_port_port(pvar(A1), pvar(B1));
    link_port_port(pvar(A1 ^ 8), pvar(B2));
    link_port_port(pvar(A2), pvar(B1 ^ 8));
    link_port_port(pvar(A2 ^ 8), pvar(B2 ^ 8));
    link_wire_port(a1, mkport(tb, lb, B1));
    link_wire_port(a1 ^ 8, mkport(tb, lb, B2));
    link_wire_port(b1, mkport(ta, la, A1));
    link_wire_port(b1 ^ 8, mkport(ta, la, A2));
  }
  HVM_DEV void comm02(ull a, ull b) {  // interact.rs:162-168
    count(&W->rw[RW_COMM], 1);
    ull b1 = paddr(b);
    link_wire_port(b1, a);
    link_wire_port(b1 ^ 8, a);
  }
  HVM_DEV void switch_num(ull a, ull b) {  // interact.rs:201-223
    count(&W->rw[RW_OPER], 1);
    ull a1 = paddr(a);
    uint32_t num = uint32_t(b);
    uint32_t n = num_tag(num) == NT_U24 ? num_payload(num) : 0;
    if (n == 0) {
      ull x = alloc();
      link_port_port(pvar(x ^ 8), P_ERA);
      link_wire_port(a1 ^ 8, pvar(x));
      link_wire_port(a1, mkport(T_CTR, 0, x));
    } else {
      ull x = alloc(), y = alloc();
      link_port_port(pvar(x), P_ERA);
      link_port_port(pvar(x ^ 8), mkport(T_CTR, 0, y));
      link_port_port(pvar(y), ull(num_u24(n - 1)));
      link_wire_port(a1 ^ 8, pvar(y ^ 8));
      link_wire_port(a1, mkport(T_CTR, 0, x));
    }
  }
  HVM_DEV uint32_t binary(uint32_t a, uint32_t op, uint32_t b) {
    int e = 0;
    uint32_t r = num_binary(a, op, b, &e);
    if (e) fail(HVM64_ERR_DIV0, net);
    return r;
  }
  HVM_DEV void op_num(ull a, ull b) {  // interact.rs:251-270
    uint32_t op = plab(a);
    ull a1 = paddr(a);
    ull t1 = load(a1);
    if (ptag(t1) == T_NUM) {
      count(&W->rw[RW_OPER], 1);
      half_free(a1);
      ull out = binary(uint32_t(b), op, uint32_t(t1));
      link_wire_port(a1 ^ 8, out);
    } else {
      ull x = alloc();
      link_port_port(pvar(x), ull(num_unary(op, uint32_t(b))));
      link_wire_port(a1 ^ 8, pvar(x ^ 8));
      link_wire_port(a1, mkport(T_OP, NT_SYM, x));
    }
  }

  // def.rs:30-37 (LabSet::has); the expansion agent's set is LabSet::ALL.
  HVM_DEV bool def_has(ull ref, unsigned lab) {
    if (ref & X_BIT) return lab < 0xFFFF;
    unsigned id = unsigned((paddr(ref) >> 3) - 1);
    if (id >= P.ndefs) {
      fail(HVM64_ERR_BAD_INPUT, ref);
      return true;
    }
    const DevDef& d = P.defs[id];
    if (lab >= d.min_safe) return false;
    unsigned w = lab >> 6;
    if (w >= d.lab_len) return false;
    return (P.labbits[d.lab_off + w] >> (lab & 63)) & 1;
  }
  // def.rs:177-189
  HVM_DEV void call(ull port, ull trg) {
    if (ptag(trg) == T_CTR && !def_has(port, plab(trg))) return comm02(port, trg);
    count(&W->rw[RW_DREF], 1);
    if (port & X_BIT) return expand_call(port, trg);
    unsigned before = allocs;
    run_def(unsigned((paddr(port) >> 3) - 1), trg);
    count(&W->rw[EX_DNODES], allocs - before);
  }

  // ---- interact.rs:6-44 --------------------------------------------------------
  HVM_DEV void interact(ull a, ull b) {
    unsigned at = ptag(a), bt = ptag(b);
    if (at <= T_VAR || bt <= T_VAR) return fail(HVM64_ERR_BAD_PAIR, a);
    bool an = at == T_REF || at == T_NUM, bn = bt == T_REF || bt == T_NUM;
    if (at == T_REF && bn && !skippable(a)) return call(a, b);
    if (an && bt == T_REF && !skippable(b)) return call(b, a);
    if (an && bn) {
      count(&W->rw[RW_ERAS], 1);
      return;
    }
    if (at == T_CTR && bt == T_SWITCH && plab(a) != 0) return comm22(a, b);
    if (at == T_SWITCH && bt == T_CTR && plab(b) != 0) return comm22(a, b);
    if ((at == T_CTR && bt == T_OP) || (at == T_OP && bt == T_CTR)) return comm22(a, b);
    if (at == T_CTR && bt == T_CTR && plab(a) != plab(b)) return comm22(a, b);
    if (at == bt && at >= T_OP) return anni2(a, b);
    if (at == T_REF && bt == T_CTR && plab(b) >= plab(a)) return comm02(a, b);
    if (at == T_CTR && bt == T_REF && plab(a) >= plab(b)) return comm02(b, a);
    if (at == T_NUM && bt == T_CTR) return comm02(a, b);
    if (at == T_CTR && bt == T_NUM) return comm02(b, a);
    if (at == T_REF && a == P_ERA) return comm02(a, b);
    if (bt == T_REF && b == P_ERA) return comm02(b, a);
    if (at == T_REF) return call(a, b);
    if (bt == T_REF) return call(b, a);
    if (at == T_OP && bt == T_NUM) return op_num(a, b);
    if (at == T_NUM && bt == T_OP) return op_num(b, a);
    if (at == T_SWITCH && bt == T_NUM) return switch_num(a, b);
    if (at == T_NUM && bt == T_SWITCH) return switch_num(b, a);
    fail(HVM64_ERR_BAD_PAIR, a);
  }

  // ---- instruction VM (runtime/src/instruction.rs:400-500, def.rs:217-289) ----
  HVM_DEV void do_ctr(unsigned lab, ull trg, ull& o1, ull& o2) {
    ull port = trg_take(trg);
    if (ptag(port) == T_CTR && plab(port) == lab) {
      free_trg(trg);
      count(&W->rw[RW_ANNI], 1);
      o1 = paddr(port);  // Trg::wire
      o2 = paddr(port) ^ 8;
      return;
    }
    ull n = alloc();
    link_taken(trg, port, mkport(T_CTR, lab, n));
    o1 = pvar(n);
    o2 = pvar(n ^ 8);
  }
  HVM_DEV void do_op(unsigned op, ull trg, ull& o1, ull& o2) {
    ull port = trg_take(trg);
    if (ptag(port) == T_NUM) {
      free_trg(trg);
      ull n = alloc();
      store(n, ull(num_unary(op, uint32_t(port))));
      o1 = mkport(T_OP, NT_SYM, n);
      o2 = pvar(n ^ 8);
      return;
    }
    if (port == P_ERA) {
      free_trg(trg);
      o1 = o2 = P_ERA;
      return;
    }
    ull n = alloc();
    link_taken(trg, port, mkport(T_OP, op, n));
    o1 = pvar(n);
    o2 = pvar(n ^ 8);
  }
  HVM_DEV ull do_op_num(unsigned op, ull trg, uint32_t rhs) {
    ull port = trg_take(trg);
    if (ptag(port) == T_NUM) {
      count(&W->rw[RW_OPER], 1);
      free_trg(trg);
      return ull(binary(uint32_t(port), op, rhs));
    }
    if (port == P_ERA) {
      free_trg(trg);
      return P_ERA;
    }
    ull n = alloc();
    link_taken(trg, port, mkport(T_OP, op, n));
    store(n, ull(rhs));
    return pvar(n ^ 8);
  }
  HVM_DEV ull create_wire_to(ull port) {  // node.rs:176-182
    ull a = alloc();
    half_free(a ^ 8);
    link_port_port(port, pvar(a));
    return a;
  }
  HVM_DEV void do_switch(ull trg, ull& o1, ull& o2) {
    ull port = trg_take(trg);
    if (ptag(port) == T_NUM) {
      count(&W->rw[RW_OPER], 1);
      free_trg(trg);
      uint32_t num = uint32_t(port);
      uint32_t n = num_tag(num) == NT_U24 ? num_payload(num) : 0;
      ull c1 = alloc();
      if (n == 0) {
        link_port_port(pvar(c1 ^ 8), P_ERA);
        o1 = mkport(T_CTR, 0, c1);
        o2 = create_wire_to(pvar(c1));
      } else {
        ull c2 = alloc();
        link_port_port(pvar(c1), P_ERA);
        link_port_port(pvar(c1 ^ 8), mkport(T_CTR, 0, c2));
        link_port_port(pvar(c2), ull(num_u24(n - 1)));
        o1 = mkport(T_CTR, 0, c1);
        o2 = create_wire_to(pvar(c2 ^ 8));
      }
      return;
    }
    if (port == P_ERA) {
      count(&W->rw[RW_ERAS], 1);
      free_trg(trg);
      o1 = o2 = P_ERA;
      return;
    }
    ull m = alloc();
    link_taken(trg, port, mkport(T_SWITCH, 0, m));
    o1 = pvar(m);
    o2 = pvar(m ^ 8);
  }

  HVM_DEV void run_def(unsigned id, ull t0) {
    if (id >= P.ndefs) return fail(HVM64_ERR_BAD_INPUT, id);
    const DevDef d = P.defs[id];
    if (d.nregs <= SMALL_REGS) {
      exec(d, t0, StridedRegs{W->regs + lane, 32});
    } else {
      ull R[MAX_REGS];
      exec(d, t0, StridedRegs{R, 1});
    }
  }
  HVM_DEV void exec(const DevDef& d, ull t0, StridedRegs R) {
    R[0] = t0;
    const DevInstr* ins = P.instrs + d.ins_off;
    for (unsigned k = 0; k < d.ins_len; k++) {
      const DevInstr I = ins[k];
      switch (I.k) {
        case I_CONST: R[I.a] = I.port; break;
        case I_LINK: count(&W->rw[EX_DLINKS], 1); link_trg(R[I.a], R[I.b]); break;
        case I_LINKCONST: count(&W->rw[EX_DLINKS], 1); link_trg_port(R[I.a], I.port); break;
        case I_CTR: {
          ull x, y;
          do_ctr(I.lab, R[I.a], x, y);
          R[I.b] = x;
          R[I.c] = y;
          break;
        }
        case I_OP: {
          ull x, y;
          do_op(I.op, R[I.a], x, y);
          R[I.b] = x;
          R[I.c] = y;
          break;
        }
        case I_OPNUM: R[I.c] = do_op_num(I.op, R[I.a], uint32_t(I.port)); break;
        case I_SWITCH: {
          ull x, y;
          do_switch(R[I.a], x, y);
          R[I.b] = x;
          R[I.c] = y;
          break;
        }
        case I_WIRES: {
          ull a = alloc();
          R[I.a] = pvar(a);
          R[I.b] = a;
          R[I.c] = pvar(a ^ 8);
          R[I.d] = a ^ 8;
          break;
        }
      }
    }
  }

  // ---- expansion agent (runtime/src/net.rs:63-108) ----------------------------
  // An agent is a Ref port with X_BIT whose address names a heap word holding
  // its output port (the reference boxes an `ExpandDef { out }`).
  HVM_DEV ull new_expand(ull out) {
    ull w = alloc();
    half_free(w ^ 8);
    store(w, out);
    return mkport(T_REF, 0xFFFF, X_BIT | w);
  }
  HVM_DEV ull take_expand(ull port) {
    ull w = paddr(port) & ~X_BIT;
    unsigned it = 0;
    ull out;
    while ((out = load(w)) == P_LOCK)
      if (!spin(it)) break;
    half_free(w);
    return out;
  }
  HVM_DEV void expand_call(ull self, ull port) {
    if (ptag(port) == T_REF && port != P_ERA) {
      if (port & X_BIT) {
        ull a = take_expand(self), b = take_expand(port);
        return link_port_port(a, b);
      }
      return call(port, self);
    }
    ull out = take_expand(self);
    unsigned t = ptag(port);
    if (t == T_RED) return fail(HVM64_ERR_BAD_PAIR, port);
    if (t == T_REF || t == T_NUM || t == T_VAR) return link_port_port(out, port);
    ull o1 = paddr(port);
    ull n = alloc();
    link_port_port(out, mkport(t, plab(port), n));
    link_wire_port(o1, new_expand(pvar(n)));
    link_wire_port(o1 ^ 8, new_expand(pvar(n ^ 8)));
  }
  // net.rs:65-69
  HVM_DEV ull expand(ull root) {
    ull a = alloc();
    half_free(a ^ 8);
    link_wire_port(root, new_expand(pvar(a)));
    return a;
  }
};

}  // namespace dev
}  // namespace hvm
