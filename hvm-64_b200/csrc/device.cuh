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
#include <stddef.h>

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

#ifndef HVM_SCAP
#define HVM_SCAP 512
#endif
#ifndef HVM_HEADROOM
#define HVM_HEADROOM 192
#endif
constexpr int WARPS = 2;            // warps per reducer block
constexpr int THREADS = WARPS * 32;
constexpr int SCAP = HVM_SCAP;      // per-warp shared-memory redex stack (power of two)
constexpr int HEADROOM = HVM_HEADROOM;  // stack slots kept free for the redexes of one step
static_assert((SCAP & (SCAP - 1)) == 0 && SCAP >= 64, "SCAP is a power of two, at least 64");
static_assert(HEADROOM >= 0 && SCAP - HEADROOM >= 32, "a step's window needs SCAP - HEADROOM >= 32");
constexpr int CHUNK = 32;           // redexes per global-queue slot
constexpr int POOL = 64;            // per-warp pool of free nodes ready for reuse
constexpr unsigned ICACHE = 32;     // instructions of the step's Def staged in shared memory
constexpr unsigned SMALL_REGS = 10; // Defs with at most this many registers use shared memory

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
  ull max_warps;   // holders (warps + queued slots) per net beyond which no work is donated; 0: no cap
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
  ull stat_lane_sum, stat_lane_max, stat_total;  // per-lane interaction cycles (sum, per-step max), warp lifetime
  ull stat_prof[32];  // profiling build: loads, exchanges, CAS (count, cycles), stores, per-rule cycles
  ull pad5[16];
  ull req_head;       // serving: requests admitted so far
  ull pad6[15];
  ull req_tail;       // serving: requests the host has written (host copies, device reads)
  int stop;           // serving: the host asks the reducer to end once idle
  int pad7;
  ull pad8[14];
  ull free_top;       // shared stack of free-node batches: batch head address | push count << 44
  ull reuse_mark;     // bump position from which free nodes are shared between warps
  ull captured;       // pre-reduce: redexes recorded by inert Defs (see capture)
  ull rw_done;        // interactions folded so far, when the run has an interaction limit
  ull pad9[12];
};

constexpr int NCOUNT = 8;  // rw[5] then comm22, dref_nodes, dref_links
enum : int { EX_COMM22 = 5, EX_DNODES, EX_DLINKS };

struct NetState {  // 112 bytes
  ull root;            // byte offset of the root wire
  long long pending;   // warps holding this net's work + queued chunks
  ull rw[NCOUNT];
  int prog;            // DevDef index of the boot program
  int status;
  ull ticket, t_admit; // serving: the request running in this slot
};

struct Slot {  // 544 bytes: one chunk of up to 32 redexes of one net
  ull seq;
  unsigned net;
  unsigned count;
  ull pad[2];
  ull r[2 * CHUNK];
};

// Serving: one request (host -> device) and one completion record (device ->
// host).  Both live in page-locked host memory mapped into the device.
struct ServeReq {  // 16 bytes
  ull ticket;       // nonzero
  unsigned slot;    // net slot the request runs in
  unsigned prog;    // DevDef index of the Def to boot
};
struct ServeDone {  // 128 bytes; `ticket` is written last
  ull ticket;
  int status;
  unsigned pairs;   // (address, word) pairs gathered into the slot's output
  ull root;
  ull rw[NCOUNT];
  ull t_admit, t_done;  // %globaltimer, ns
  ull pad[2];
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
  // per-warp overflow stacks: warp g of the reducer grid owns
  // spill[2 * spill_cap * g ...] (spill_cap redexes); null: none
  unsigned spill_cap;
  ull* spill;
  unsigned ovf_flush;           // free-list length at which a lane publishes it (see free_list_push)
  // register files of Def calls needing more than LOCAL_REGS registers:
  // warp g owns bigregs[32 * MAX_REGS * g ...], [register][lane]; null: none
  ull* bigregs;
  // pre-reduce (all zero otherwise): boot without the expansion agent
  // (Net::reduce after Net::boot, transform/src/pre_reduce.rs:145-147); the
  // buffer for redexes inert Defs capture; an interaction limit
  unsigned no_expand, capture_cap;
  ull* capture;
  ull rw_limit;
  unsigned gen;  // 1: the compiled Def functions match the loaded Book (HVM_GEN_INCLUDE builds)
  // serving (all zero for a batch run)
  unsigned serve;
  const ServeReq* req;         // device ring of req_cap requests
  ServeDone* done;             // per slot (mapped host memory)
  ull* out;                    // per slot: out_cap (address, word) pairs (mapped host memory)
  unsigned req_cap, out_cap;
};

// The run's parameters: one constant-memory block per device, uploaded on
// the launching stream before the run's kernels (constant-bank operands cost
// no instruction; a per-block shared-memory copy measured 11 % slower).  A
// run owns the block until its kernels finish: the host runner gives runs on
// one device turns (hvm64.cu, DeviceTurn).  The host emulation uses a plain
// global.
#ifdef __CUDACC__
__constant__ Params g_P;
#else
inline Params g_P;
#endif

// ---- platform layer ------------------------------------------------------------
// The runtime below is written against these few operations.  Under nvcc
// they are strong GPU-scope PTX accesses and CUDA atomics; under a host
// compiler (the CPU emulation harness the tests build from this same file)
// they are std::atomic_ref operations, so the protocol logic can be exercised
// with many host threads.
#ifdef __CUDACC__
#define HVM_DEV __device__
#define HVM_INL __device__ __forceinline__
// Rare paths stay out of line so the hot loop stays small (instruction cache)
// and needs fewer registers.
#define HVM_COLD __device__ __noinline__
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
// Fetch-and-add on a word of a warp's shared-memory state (`p` is a generic
// pointer into shared memory).  A plain shared-memory atomic per lane:
// aggregating the converged lanes first (match, leader, shuffle) measured
// 8 % slower overall -- its extra instructions cost more than the few lanes
// that serialise on the word.
__device__ __forceinline__ int smem_add_i32(int* p, int v) {
  int old;
  unsigned a = unsigned(__cvta_generic_to_shared(p));
  asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned smem_add_u32(unsigned* p, unsigned v) {
  return unsigned(smem_add_i32(reinterpret_cast<int*>(p), int(v)));
}
// A release fence: the node fills and links before it are visible to any
// lane that later reaches the node through a port published after it.
__device__ __forceinline__ void mem_fence() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void pause_brief() { __nanosleep(64); }
// LOCK-fill nodes [s, s+n) with 16-byte stores.
__device__ __forceinline__ void lock_fill(ull* H, ull s, ull n) {
  ulonglong2* c = reinterpret_cast<ulonglong2*>(H) + s;
  for (ull k = 0; k < n; k++) c[k] = make_ulonglong2(P_LOCK, P_LOCK);
}
#else
#define HVM_DEV
#define HVM_INL inline
#define HVM_COLD __attribute__((noinline))
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
inline int smem_add_i32(int* p, int v) { return atom_add_i32(p, v); }
inline unsigned smem_add_u32(unsigned* p, unsigned v) { return atom_add_u32(p, v); }
inline void mem_fence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void pause_brief() { std::this_thread::yield(); }
inline void lock_fill(ull* H, ull s, ull n) {
  for (ull k = 0; k < 2 * n; k++) st_gpu(H + 2 * s + k, P_LOCK);
}
#endif
#ifdef HVM_EMU_CHECK_ALLOC
// Host test builds only: per node, whether it is handed out (top bit); a node
// handed out while out, or reclaimed while not out, is counted here.
inline std::atomic<unsigned>* g_node_out = nullptr;
inline std::atomic<unsigned long long> g_alloc_faults{0};
inline void check_handed_out(ull node) {
  if (node && (g_node_out[node >> 4].fetch_or(1u) & 1u)) g_alloc_faults++;
}
inline void check_reclaimed(ull node) {
  if (!(g_node_out[node >> 4].fetch_and(~1u) & 1u)) g_alloc_faults++;
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

// Per-warp shared state of the reducer (one per warp; the CPU emulation
// harness gives each host thread one too).  Warps' states lie back to back in
// shared memory and `icache` is filled with 16-byte stores, so the size is
// kept a multiple of 16.
struct alignas(16) WarpSmem {
  ull stk[2 * SCAP];          // redex stack (ring of SCAP pairs)
  ull regs[SMALL_REGS * 32];  // VM registers, [register][lane]
  ull pool[POOL];             // free nodes ready for reuse
  ull freed[POOL];            // nodes reclaimed during the current step
  ull sel[64];                // the redexes chosen for the current step
  DevInstr icache[ICACHE];    // the instructions of `icache_def`, staged for this step
  DevDef idef;                // that Def's header
  unsigned icache_def;        // Def index staged in icache (~0u: none)
  ull rw[NCOUNT];             // counters of the warp's current net
  unsigned cnt[NCOUNT * 32];  // per lane: counts of this step, [counter][lane] (folded into rw)
  ull ovf[32];                // per lane: free list head | pushes since published << 48 (see free_list_push)
  ull fw[4 * 32];             // per lane: words freed alone by the current interaction
  ull bnext[32], bend[32];    // per lane: pre-LOCKed bump chunk [bnext, bend), node indices
  unsigned allocs[32];        // per lane: nodes allocated (for the DREF statistics)
  unsigned ring_base;         // this step's pushes go to stack slots ring_base + k ...
  unsigned ring_cap;          // ... for k < ring_cap; push k >= ring_cap goes to the overflow stack
  ull* sp;                    // this warp's overflow stack in HBM (null: none; pushes go to the queue)
  ull* bigregs;               // this warp's register files for Defs above LOCAL_REGS (null: none)
  unsigned sp_n, sp_cap;      // redexes in it between steps, and its capacity
  int pool_cap;               // 0: no reuse pool (reclaimed nodes go to `ovf`)
#ifdef HVM_PROFILE_OPS
  ull prof[32];               // profiling build: op counts and wait cycles, cycles per rule
#endif
  ull st_steps, st_lanes, st_busy, st_idle, st_lane_sum, st_lane_max, st_total;
  unsigned ring_cnt;
  int pool_n;
  int freed_n;
  unsigned pad;
};
static_assert(sizeof(WarpSmem) % 16 == 0 && offsetof(WarpSmem, icache) % 16 == 0,
              "icache of every warp's state must be 16-byte aligned");

// Initial per-lane / per-warp runtime state (lane `ln` of warp state `W`).
HVM_INL void lane_init(WarpSmem* W, unsigned ln) {
  for (int k = 0; k < NCOUNT; k++) W->cnt[k * 32 + ln] = 0;
  W->ovf[ln] = 0;
  for (int k = 0; k < 4; k++) W->fw[k * 32 + ln] = 0;
  W->bnext[ln] = W->bend[ln] = 0;
  W->allocs[ln] = 0;
}

// ---- cold paths as free functions over scalars -------------------------------
// (A Lane never has its address taken, so its state stays in registers.)
HVM_COLD void run_fail(unsigned net, int code, ull info) {
  if (atom_cas32(&g_P.ctrl->error, 0, code) == 0) {
    g_P.ctrl->error_info = info;
    g_P.ctrl->error_net = int(net);
  }
}
HVM_INL bool run_failed() { return ld_gpu32(&g_P.ctrl->error) != 0; }
// run_fail for the failure branches of code that is inlined at many sites
// (heap accesses, bounded waits): a call there, even one never taken, makes
// every such site keep its live registers across the call, which costs the
// reducer about a tenth of its throughput.
// (Only the code is recorded: storing the net and detail too measured 4 %
// slower.)
HVM_INL void run_fail_here(int code) { atom_cas32(&g_P.ctrl->error, 0, code); }
// One poll of a bounded wait; false = abandon the wait.
HVM_INL bool run_spin(unsigned net, unsigned& it) {
  ++it;
  if ((it & 63) == 0) {
    if (run_failed()) return false;
    if (it > g_P.ctrl->spin_limit) {
      run_fail_here(HVM64_ERR_TIMEOUT);
      return false;
    }
    pause_brief();
  }
  return true;
}
HVM_INL ull* heap_at(unsigned net, ull a) {
  if (a >= g_P.heap_bytes) {
    run_fail_here(HVM64_ERR_BAD_ADDR);
    a = 0;
  }
  return g_P.heap + (a >> 3);
}
// wire.rs:342-350: wait until the word is not LOCK and take it.
HVM_COLD ull relock(unsigned net, ull w) {
  unsigned it = 0;
  for (;;) {
    ull got = atom_exch(heap_at(net, w), P_LOCK);
    if (got != P_LOCK) return got;
    if (!run_spin(net, it)) return P_ERA;
  }
}
HVM_COLD uint32_t binary_op(unsigned net, uint32_t a, uint32_t op, uint32_t b) {
  int e = 0;
  uint32_t r = num_binary(a, op, b, &e);
  if (e) run_fail(net, HVM64_ERR_DIV0, net);
  return r;
}
// Neither the warp's stack nor its overflow stack had room: the platform
// driver ships the redex to shared work (the CUDA driver: a one-redex queue
// slot, or HVM64_ERR_QUEUE when the queue is full -- it never waits).
HVM_COLD void push_overflow(unsigned net, ull a, ull b);
// A lane's free list of reclaimed nodes is linked through their left words
// (right words LOCK); the lane's head word holds the first node's address in
// bits 0-47 and the number of nodes pushed since the list was last
// published in bits 48-63.
//
// Free nodes move between warps through one shared stack of batches, once
// the heap is past its reuse mark (Ctrl::reuse_mark; a batch run sets it at
// half the heap, a server at 0): a lane's list is published whole once it
// holds Params::ovf_flush nodes (OVF_FLUSH for a batch, 32 for a server, which
// keeps fewer nodes stranded per lane), the batch's head node linking the next batch through
// its right word, and a lane whose list is empty takes a batch before it
// takes fresh nodes from the bump pointer.  Below the mark, allocation stays
// on the bump pointer and the lanes' own lists (no shared traffic).  The top
// word carries a push/pop count above the address bits, so a pop whose
// batch was taken and republished meanwhile fails its CAS (ABA).
#ifndef HVM_OVF_FLUSH
#define HVM_OVF_FLUSH 128
#endif
constexpr unsigned OVF_FLUSH = HVM_OVF_FLUSH;  // batch runs (a server publishes after 32)
constexpr ull FT_ADDR = (1ull << 44) - 1;
constexpr ull FT_TAG = 1ull << 44;
constexpr ull OVF_ADDR = (1ull << 48) - 1;
HVM_INL bool past_reuse_mark() { return ld_gpu(&g_P.ctrl->bump) >= g_P.ctrl->reuse_mark; }
HVM_COLD void free_publish(unsigned net, ull* ovf) {
  ull head = *ovf & OVF_ADDR;
  if (!head) return;
  ull* top = &g_P.ctrl->free_top;
  unsigned it = 0;
  for (;;) {
    ull t = ld_gpu(top);
    st_gpu(heap_at(net, head | 8), t & FT_ADDR);
    mem_fence();  // the batch's links are visible before its head is
    if (atom_cas(top, t, (head & FT_ADDR) | ((t & ~FT_ADDR) + FT_TAG)) == t) break;
    if (!run_spin(net, it)) return;  // lost CASes are other lanes' progress; still bounded
  }
  *ovf = 0;
}
// Take one batch from the shared stack as the lane's list; false when empty.
HVM_COLD bool free_take(unsigned net, ull* ovf) {
  ull* top = &g_P.ctrl->free_top;
  for (int tries = 0; tries < 64; tries++) {
    ull t = ld_gpu(top);
    ull a = t & FT_ADDR;
    if (a == 0) return false;
    // Stale when the batch was taken meanwhile; then the CAS below fails.
    ull next = ld_gpu(heap_at(net, a | 8));
    if (atom_cas(top, t, (next & FT_ADDR) | ((t & ~FT_ADDR) + FT_TAG)) == t) {
      mem_fence();
      st_gpu(heap_at(net, a | 8), P_LOCK);
      *ovf = a;
      return true;
    }
  }
  return false;
}
// Pop the lane's free list (or, past the reuse mark, a shared batch) / take
// a new pre-LOCKed bump chunk.
struct Refill {
  ull node, bnext, bend;
};
HVM_COLD Refill alloc_refill(unsigned net, ull* ovf) {
  if ((*ovf & OVF_ADDR) != 0 || (past_reuse_mark() && free_take(net, ovf))) {
    ull a = *ovf & OVF_ADDR, n = *ovf >> 48;
    *ovf = (ld_gpu(heap_at(net, a)) & OVF_ADDR) | ((n ? n - 1 : 0) << 48);
    st_gpu(heap_at(net, a), P_LOCK);
    mem_fence();
    return {a, 0, 0};
  }
  ull n = g_P.ctrl->chunk_nodes;
  ull s = atom_add(&g_P.ctrl->bump, n);
  if (s + n > g_P.ctrl->heap_nodes) {
    run_fail(net, HVM64_ERR_OOM, s);
    return {0, 0, 0};
  }
  lock_fill(g_P.heap, s, n);
  mem_fence();  // LOCK is visible before any of these nodes escapes
  return {s << 4, s + 1, s + n};
}
// A reclaimed node (both words LOCK) onto a lane's free list.
HVM_INL void free_list_push(unsigned net, ull* ovf, ull node) {
  ull n = (*ovf >> 48) + 1;
  st_gpu(heap_at(net, node), *ovf & OVF_ADDR);
  *ovf = node | (n < 0xFFFF ? n << 48 : 0xFFFFull << 48);
  if (n >= g_P.ovf_flush && past_reuse_mark()) free_publish(net, ovf);
}

// ---- the runtime proper ------------------------------------------------------
// Every rule, link operation and VM instruction is one out-of-line function
// over a three-word context (warp state, lane, net).  A lane's mutable state
// (freed-word slots, bump chunk) lives in its warp's shared memory, so these
// functions keep nothing in local memory and each exists once in the binary:
// the hot code fits the instruction cache.
struct Ctx {
  WarpSmem* W;
  unsigned lane;
  unsigned net;
};

#define LS(field) (c.W->field[c.lane])             // a lane's slot
#define FW(k) (c.W->fw[(k) * 32 + c.lane])          // freed-word slot k

HVM_INL ull hload(const Ctx& c, ull a) {
#if defined(HVM_PROFILE_OPS) && defined(__CUDACC__)
  long long t = clock64();
  ull v = ld_gpu(heap_at(c.net, a));
  asm volatile("" : "+l"(v));
  atomicAdd(&c.W->prof[0], 1ull);
  atomicAdd(&c.W->prof[1], ull(clock64() - t));
  return v;
#else
  return ld_gpu(heap_at(c.net, a));
#endif
}
#if defined(HVM_PROFILE_OPS) && defined(__CUDACC__)
HVM_INL ull prof_done(const Ctx& c, int k, long long t, ull v) {
  asm volatile("" : "+l"(v));
  atomicAdd(&c.W->prof[k], 1ull);
  atomicAdd(&c.W->prof[k + 1], ull(clock64() - t));
  return v;
}
HVM_INL void hstore(const Ctx& c, ull a, ull v) {
  atomicAdd(&c.W->prof[6], 1ull);
  st_gpu(heap_at(c.net, a), v);
}
HVM_INL ull hswap(const Ctx& c, ull a, ull v) {
  long long t = clock64();
  return prof_done(c, 2, t, atom_exch(heap_at(c.net, a), v));
}
HVM_INL ull hcas(const Ctx& c, ull a, ull e, ull v) {
  long long t = clock64();
  return prof_done(c, 4, t, atom_cas(heap_at(c.net, a), e, v));
}
#define PROF_RULE(idx) long long prof_t0 = clock64(); struct ProfEnd { const Ctx& c; long long t; int k; \
  __device__ ~ProfEnd() { atomicAdd(&c.W->prof[8 + 2 * k], 1ull); atomicAdd(&c.W->prof[9 + 2 * k], ull(clock64() - t)); } } prof_end{c, prof_t0, idx};
#else
HVM_INL void hstore(const Ctx& c, ull a, ull v) { st_gpu(heap_at(c.net, a), v); }
HVM_INL ull hswap(const Ctx& c, ull a, ull v) { return atom_exch(heap_at(c.net, a), v); }
HVM_INL ull hcas(const Ctx& c, ull a, ull e, ull v) { return atom_cas(heap_at(c.net, a), e, v); }
#define PROF_RULE(k)
#endif
HVM_INL void count(const Ctx& c, int k, ull v = 1) { c.W->cnt[k * 32 + c.lane] += unsigned(v); }

// wire.rs:342-350
HVM_INL ull lock_target(const Ctx& c, ull w) {
  ull got = hswap(c, w, P_LOCK);
  return got != P_LOCK ? got : relock(c.net, w);
}

// ---- allocator -------------------------------------------------------------
// The reference's allocator (runtime/src/allocator.rs:73-110) writes LOCK
// into both words of every node it hands out and links a node into a free
// list once both halves are FREE.  Here a node is LOCK-filled when it becomes
// free (or when its bump chunk is taken) and that fill is fenced before the
// node is handed out again, so alloc() itself touches no heap memory.  A node
// whose two halves are both freed by the same interaction is reclaimed
// without reading the other half; otherwise the reference's store-FREE /
// read-other-half / CAS sequence decides which lane reclaims.
HVM_COLD void recycle(const Ctx& c, ull node) {
#ifdef HVM_EMU_CHECK_ALLOC
  check_reclaimed(node);
#endif
  int k = c.W->pool_cap ? smem_add_i32(&c.W->freed_n, 1) : POOL;
  if (k < c.W->pool_cap) {
    c.W->freed[k] = node;
  } else {
    free_list_push(c.net, &LS(ovf), node);  // right word already LOCK
  }
}
HVM_COLD ull alloc_slow(const Ctx& c) {
  Refill r = alloc_refill(c.net, &LS(ovf));
  if (r.bend) {
    LS(bnext) = r.bnext;
    LS(bend) = r.bend;
  }
  return r.node;
}
#ifdef HVM_EMU_CHECK_ALLOC
HVM_INL ull alloc_unchecked(const Ctx& c);
HVM_INL ull alloc(const Ctx& c) {
  ull n = alloc_unchecked(c);
  check_handed_out(n);
  return n;
}
HVM_INL ull alloc_unchecked(const Ctx& c) {
#else
HVM_INL ull alloc(const Ctx& c) {
#endif
  LS(allocs)++;
  if (c.W->pool_cap) {
    int k = smem_add_i32(&c.W->pool_n, -1) - 1;
    if (k >= 0) return c.W->pool[k];
  }
  ull b = LS(bnext);
  if (b != LS(bend)) {
    LS(bnext) = b + 1;
    return b << 4;
  }
  return alloc_slow(c);
}
// A word freed alone: a node found fully free is claimed by CAS on its left
// word, then kept only if its right word is still free -- between the load
// and the CAS the node may have been reclaimed by the other half's owner,
// reused, and half-freed again (ABA); then the left word is handed back.
HVM_COLD void claim(const Ctx& c, ull w, ull other) {
  if (!w || other != P_FREE) return;
  ull l = w & ~8ull;
  if (hcas(c, l, P_FREE, P_LOCK) != P_FREE) return;
  if (hload(c, l | 8) == P_FREE) {
    hstore(c, l | 8, P_LOCK);
    recycle(c, l);
  } else {
    hstore(c, l, P_FREE);
  }
}
// End of an interaction: look at the other half of every word freed alone
// (the loads are in flight together).
HVM_COLD void settle(const Ctx& c) {
  PROF_RULE(6)
  ull w0 = FW(0), w1 = FW(1), w2 = FW(2), w3 = FW(3);
  if (!(w0 | w1 | w2 | w3)) return;
  ull o0 = w0 ? hload(c, w0 ^ 8) : 0, o1 = w1 ? hload(c, w1 ^ 8) : 0;
  ull o2 = w2 ? hload(c, w2 ^ 8) : 0, o3 = w3 ? hload(c, w3 ^ 8) : 0;
  FW(0) = FW(1) = FW(2) = FW(3) = 0;
  claim(c, w0, o0);
  claim(c, w1, o1);
  claim(c, w2, o2);
  claim(c, w3, o3);
}
HVM_COLD void half_free(const Ctx& c, ull a) {
  PROF_RULE(8)
  ull x = a ^ 8;
  int k = -1;
  if (a != 0) {
    if (FW(0) == x) k = 0;
    else if (FW(1) == x) k = 1;
    else if (FW(2) == x) k = 2;
    else if (FW(3) == x) k = 3;
  }
  if (k >= 0) {  // both halves freed by this interaction: no one else can claim the node
    FW(k) = 0;
    ull l = a & ~8ull;
    hstore(c, l, P_LOCK);
    hstore(c, l | 8, P_LOCK);
    recycle(c, l);
    return;
  }
  hstore(c, a, P_FREE);
  if (FW(0) == 0) FW(0) = a;
  else if (FW(1) == 0) FW(1) = a;
  else if (FW(2) == 0) FW(2) = a;
  else if (FW(3) == 0) FW(3) = a;
  else {
    settle(c);
    FW(0) = a;
  }
}

// ---- redex pushes (linker.rs:70-85) -----------------------------------------
// The reference's queue is an unbounded vector (linker.rs:308-344); here a
// step's k-th push goes to the warp's shared-memory stack while it has room,
// then to the warp's private overflow stack in HBM (slot sp_n + k - ring_cap),
// then to the global queue.  None of these waits for anyone.
HVM_COLD void push_spill(const Ctx& c, ull a, ull b, unsigned j) {
  unsigned i = c.W->sp_n + j;
  if (c.W->sp && i < c.W->sp_cap) {
    c.W->sp[2 * ull(i)] = a;
    c.W->sp[2 * ull(i) + 1] = b;
    return;
  }
  push_overflow(c.net, a, b);
}
HVM_INL void push(const Ctx& c, ull a, ull b) {
  unsigned cap = c.W->ring_cap;
  unsigned k = smem_add_u32(&c.W->ring_cnt, 1u);
  if (k < cap) {
    unsigned i = (c.W->ring_base + k) & unsigned(SCAP - 1);
    c.W->stk[2 * i] = a;
    c.W->stk[2 * i + 1] = b;
  } else {
    push_spill(c, a, b, k - cap);
  }
}
// After a step that pushed `cnt` redexes (the value of ring_cnt): how many of
// them went to the overflow stack (the rest of those past ring_cap went to
// the queue).
HVM_INL unsigned spilled_of(const WarpSmem* W, unsigned cnt) {
  if (cnt <= W->ring_cap || !W->sp) return 0;
  unsigned over = cnt - W->ring_cap, room = W->sp_cap - W->sp_n;
  return over < room ? over : room;
}
// Upper bound on the redexes one interaction of rule class `cls` pushes
// (redex_class codes): an instruction of a Def pushes at most one (each
// link resolves to at most one active pair); a Def call that commutes
// instead (def.rs:182-184) pushes two, comm22 four, the other rules fewer.
HVM_INL unsigned pushes_bound(unsigned cls) {
  if (cls >= 64 && cls - 64 < g_P.ndefs) {
    unsigned r = g_P.defs[cls - 64].redexes;
    return r > 4 ? r : 4;
  }
  return 4;
}
HVM_INL void redux(const Ctx& c, ull a, ull b) {
  if (skippable(a) && skippable(b)) count(c, RW_ERAS);
  else push(c, a, b);
}

// ---- linker (runtime/src/linker.rs:25-203) ----------------------------------
HVM_INL void half_link_port_port(const Ctx& c, ull a, ull b) {
  if (ptag(a) == T_VAR) hstore(c, paddr(a), b);
}
HVM_INL void link_port_port(const Ctx& c, ull a, ull b) {
  if (principal(a) && principal(b)) {
    redux(c, a, b);
  } else {
    half_link_port_port(c, a, b);
    half_link_port_port(c, b, a);
  }
}
HVM_COLD void resolve_redirect_pri(const Ctx& c, ull ap, ull aw, ull bp);
// The CAS lost against another lane linking the same wire: leave a redirect
// (linker.rs:109-123).
HVM_COLD void half_link_failed(const Ctx& c, ull ap, ull aw, ull bp) {
  if (ptag(bp) == T_VAR) {
    hstore(c, aw, pred(paddr(bp)));
  } else if (principal(bp)) {
    hstore(c, aw, bp);
    resolve_redirect_pri(c, ap, aw, bp);
  } else {
    run_fail(c.net, HVM64_ERR_BAD_PAIR, bp);
  }
}
HVM_COLD void half_link_wire_port(const Ctx& c, ull ap, ull aw, ull bp) {
  if (ptag(ap) == T_VAR) {
    if (hcas(c, paddr(ap), pvar(aw), bp) == pvar(aw)) half_free(c, aw);
    else half_link_failed(c, ap, aw, bp);
  } else {
    half_free(c, aw);
  }
}
HVM_COLD void link_wire_wire(const Ctx& c, ull aw, ull bw) {
  PROF_RULE(9)
  // Both words belong to nodes this interaction consumes, so no other lane
  // takes them: the two exchanges go out together (one round trip instead of
  // two) and give the values the reference's take-one-then-the-other does; a
  // word its creator has not written yet (LOCK) is waited for after both.
  ull ap = hswap(c, aw, P_LOCK);
  ull bp = hswap(c, bw, P_LOCK);
  if (ap == P_LOCK) ap = relock(c.net, aw);
  if (bp == P_LOCK) bp = relock(c.net, bw);
  if (principal(ap) && principal(bp)) {
    half_free(c, aw);
    half_free(c, bw);
    redux(c, ap, bp);
  } else {
    half_link_wire_port(c, ap, aw, bp);
    half_link_wire_port(c, bp, bw, ap);
  }
}
// link_wire_port for a wire whose target `ap` was already taken (locked).
HVM_COLD void link_locked_wire_port(const Ctx& c, ull aw, ull ap, ull bp) {
  PROF_RULE(10)
  if (principal(ap) && principal(bp)) {
    half_free(c, aw);
    redux(c, ap, bp);
  } else {
    half_link_wire_port(c, ap, aw, bp);
    half_link_port_port(c, bp, ap);
  }
}
HVM_INL void link_wire_port(const Ctx& c, ull aw, ull bp) { link_locked_wire_port(c, aw, lock_target(c, aw), bp); }
HVM_COLD void resolve_redirect_pri(const Ctx& c, ull ap, ull aw, ull bp) {
  unsigned it = 0;
  for (;;) {
    ull tw = paddr(ap);
    ull tp = hload(c, tw);
    if (tp == P_LOCK) {
      if (!run_spin(c.net, it)) return;
      continue;
    }
    if (ptag(tp) == T_RED) {
      half_free(c, tw);
      ap = tp;
      continue;
    }
    if (ptag(tp) == T_VAR) {
      if (hcas(c, tw, tp, bp) == tp) {
        tw = paddr(tp);
        tp = hload(c, tw);
        unsigned it2 = 0;
        while (tp != P_LOCK && ptag(tp) == T_RED) {
          half_free(c, tw);
          tw = paddr(tp);
          tp = hload(c, tw);
          if (!run_spin(c.net, it2)) return;
        }
        return;
      }
      if (!run_spin(c.net, it)) return;
      continue;
    }
    if (principal(tp) || tp == P_GONE) {
      ull xw = aw < tw ? aw : tw;
      ull yw = aw < tw ? tw : aw;
      ull xp = hswap(c, xw, P_GONE);
      if (xp != P_GONE) {
        ull yp = hswap(c, yw, P_GONE);
        redux(c, xp, yp);
      } else {
        half_free(c, xw);
        unsigned it3 = 0;
        while (hcas(c, yw, P_GONE, P_LOCK) != P_GONE)
          if (!run_spin(c.net, it3)) return;
        half_free(c, yw);
      }
      return;
    }
    run_fail(c.net, HVM64_ERR_BAD_PAIR, tp);
    return;
  }
}
// Trg (linker.rs:228-304): a wire is its address with the Red tag.
HVM_INL void link_trg_port(const Ctx& c, ull a, ull b) {
  if (trg_is_wire(a)) link_wire_port(c, a, b);
  else link_port_port(c, a, b);
}
HVM_COLD void link_trg(const Ctx& c, ull a, ull b) {
  bool aw = trg_is_wire(a), bw = trg_is_wire(b);
  if (aw && bw) link_wire_wire(c, a, b);
  else if (aw) link_wire_port(c, a, b);
  else if (bw) link_wire_port(c, b, a);
  else link_port_port(c, a, b);
}
HVM_INL void free_trg(const Ctx& c, ull t) {
  if (trg_is_wire(t)) half_free(c, t);
}
// The target of a Trg about to be consumed by a VM instruction.  A wire is
// locked rather than read: every path of the instruction then either frees
// that wire or links it at once (which would lock it first), so taking the
// lock up front saves a round trip and changes nothing observable.
HVM_INL ull trg_take(const Ctx& c, ull t) { return trg_is_wire(t) ? lock_target(c, t) : t; }
// link_trg_port for a Trg taken with trg_take.
HVM_INL void link_taken(const Ctx& c, ull t, ull target, ull b) {
  if (trg_is_wire(t)) link_locked_wire_port(c, t, target, b);
  else link_port_port(c, t, b);
}

// ---- rules (runtime/src/interact.rs) ------------------------------------------
HVM_COLD void anni2(const Ctx& c, ull a, ull b) {  // interact.rs:72-79
  PROF_RULE(0)
  count(c, RW_ANNI);
  ull a1 = paddr(a), b1 = paddr(b);
  link_wire_wire(c, a1, b1);
  link_wire_wire(c, a1 ^ 8, b1 ^ 8);
}
HVM_COLD void comm22(const Ctx& c, ull a, ull b) {  // interact.rs:118-141
  PROF_RULE(1)
  count(c, RW_COMM);
  count(c, EX_COMM22);
  ull a1 = paddr(a), b1 = paddr(b);
  ull A1 = alloc(c), A2 = alloc(c), B1 = alloc(c), B2 = alloc(c);
  unsigned ta = ptag(a), la = plab(a), tb = ptag(b), lb = plab(b);
  link_port_port(c, pvar(A1), pvar(B1));
  link_port_port(c, pvar(A1 ^ 8), pvar(B2));
  link_port_port(c, pvar(A2), pvar(B1 ^ 8));
  link_port_port(c, pvar(A2 ^ 8), pvar(B2 ^ 8));
  link_wire_port(c, a1, mkport(tb, lb, B1));
  link_wire_port(c, a1 ^ 8, mkport(tb, lb, B2));
  link_wire_port(c, b1, mkport(ta, la, A1));
  link_wire_port(c, b1 ^ 8, mkport(ta, la, A2));
}
HVM_COLD void comm02(const Ctx& c, ull a, ull b) {  // interact.rs:162-168
  PROF_RULE(2)
  count(c, RW_COMM);
  ull b1 = paddr(b);
  link_wire_port(c, b1, a);
  link_wire_port(c, b1 ^ 8, a);
}
HVM_COLD void switch_num(const Ctx& c, ull a, ull b) {  // interact.rs:201-223
  PROF_RULE(3)
  count(c, RW_OPER);
  ull a1 = paddr(a);
  uint32_t num = uint32_t(b);
  uint32_t n = num_tag(num) == NT_U24 ? num_payload(num) : 0;
  if (n == 0) {
    ull x = alloc(c);
    link_port_port(c, pvar(x ^ 8), P_ERA);
    link_wire_port(c, a1 ^ 8, pvar(x));
    link_wire_port(c, a1, mkport(T_CTR, 0, x));
  } else {
    ull x = alloc(c), y = alloc(c);
    link_port_port(c, pvar(x), P_ERA);
    link_port_port(c, pvar(x ^ 8), mkport(T_CTR, 0, y));
    link_port_port(c, pvar(y), ull(num_u24(n - 1)));
    link_wire_port(c, a1 ^ 8, pvar(y ^ 8));
    link_wire_port(c, a1, mkport(T_CTR, 0, x));
  }
}
HVM_COLD void op_num(const Ctx& c, ull a, ull b) {  // interact.rs:251-270
  PROF_RULE(4)
  uint32_t op = plab(a);
  ull a1 = paddr(a);
  ull t1 = hload(c, a1);
  if (ptag(t1) == T_NUM) {
    count(c, RW_OPER);
    half_free(c, a1);
    ull out = binary_op(c.net, uint32_t(b), op, uint32_t(t1));
    link_wire_port(c, a1 ^ 8, out);
  } else {
    ull x = alloc(c);
    link_port_port(c, pvar(x), ull(num_unary(op, uint32_t(b))));
    link_wire_port(c, a1 ^ 8, pvar(x ^ 8));
    link_wire_port(c, a1, mkport(T_OP, NT_SYM, x));
  }
}

// ---- instruction VM (runtime/src/instruction.rs:400-500, def.rs:217-289) -----
HVM_COLD void do_ctr(const Ctx& c, unsigned lab, ull trg, ull& o1, ull& o2) {
  PROF_RULE(11)
  ull port = trg_take(c, trg);
  if (ptag(port) == T_CTR && plab(port) == lab) {
    free_trg(c, trg);
    count(c, RW_ANNI);
    o1 = paddr(port);  // Trg::wire
    o2 = paddr(port) ^ 8;
    return;
  }
  ull n = alloc(c);
  link_taken(c, trg, port, mkport(T_CTR, lab, n));
  o1 = pvar(n);
  o2 = pvar(n ^ 8);
}
HVM_COLD void do_op(const Ctx& c, unsigned op, ull trg, ull& o1, ull& o2) {
  ull port = trg_take(c, trg);
  if (ptag(port) == T_NUM) {
    free_trg(c, trg);
    ull n = alloc(c);
    hstore(c, n, ull(num_unary(op, uint32_t(port))));
    o1 = mkport(T_OP, NT_SYM, n);
    o2 = pvar(n ^ 8);
    return;
  }
  if (port == P_ERA) {
    free_trg(c, trg);
    o1 = o2 = P_ERA;
    return;
  }
  ull n = alloc(c);
  link_taken(c, trg, port, mkport(T_OP, op, n));
  o1 = pvar(n);
  o2 = pvar(n ^ 8);
}
HVM_COLD ull do_op_num(const Ctx& c, unsigned op, ull trg, uint32_t rhs) {
  ull port = trg_take(c, trg);
  if (ptag(port) == T_NUM) {
    count(c, RW_OPER);
    free_trg(c, trg);
    return ull(binary_op(c.net, uint32_t(port), op, rhs));
  }
  if (port == P_ERA) {
    free_trg(c, trg);
    return P_ERA;
  }
  ull n = alloc(c);
  link_taken(c, trg, port, mkport(T_OP, op, n));
  hstore(c, n, ull(rhs));
  return pvar(n ^ 8);
}
HVM_COLD ull create_wire_to(const Ctx& c, ull port) {  // node.rs:176-182
  ull a = alloc(c);
  half_free(c, a ^ 8);
  link_port_port(c, port, pvar(a));
  return a;
}
HVM_COLD void do_switch(const Ctx& c, ull trg, ull& o1, ull& o2) {
  ull port = trg_take(c, trg);
  if (ptag(port) == T_NUM) {
    count(c, RW_OPER);
    free_trg(c, trg);
    uint32_t num = uint32_t(port);
    uint32_t n = num_tag(num) == NT_U24 ? num_payload(num) : 0;
    ull c1 = alloc(c);
    if (n == 0) {
      link_port_port(c, pvar(c1 ^ 8), P_ERA);
      o1 = mkport(T_CTR, 0, c1);
      o2 = create_wire_to(c, pvar(c1));
    } else {
      ull c2 = alloc(c);
      link_port_port(c, pvar(c1), P_ERA);
      link_port_port(c, pvar(c1 ^ 8), mkport(T_CTR, 0, c2));
      link_port_port(c, pvar(c2), ull(num_u24(n - 1)));
      o1 = mkport(T_CTR, 0, c1);
      o2 = create_wire_to(c, pvar(c2 ^ 8));
    }
    return;
  }
  if (port == P_ERA) {
    count(c, RW_ERAS);
    free_trg(c, trg);
    o1 = o2 = P_ERA;
    return;
  }
  ull m = alloc(c);
  link_taken(c, trg, port, mkport(T_SWITCH, 0, m));
  o1 = pvar(m);
  o2 = pvar(m ^ 8);
}
// Runs a Def's instruction list over a register file (base + i * stride).
// An inert Def's call (transform/src/pre_reduce.rs:96-101): the redex is
// recorded for the host, which puts it back into the net's redexes.
HVM_COLD void capture(const Ctx& c, ull port, ull trg) {
  ull k = atom_add(&g_P.ctrl->captured, 1ull);
  if (k >= g_P.capture_cap) return run_fail(c.net, HVM64_ERR_OUTPUT, k);
  g_P.capture[2 * k] = port;
  g_P.capture[2 * k + 1] = trg;
}
HVM_COLD void exec(const Ctx& c, const DevDef& d, ull t0, ull* R, unsigned stride, const DevInstr* ins) {
  R[0] = t0;
  for (unsigned k = 0; k < d.ins_len; k++) {
    const DevInstr I = ins[k];
    ull* ra = R + I.a * stride;
    switch (I.k) {
      case I_CONST: *ra = I.port; break;
      case I_LINK: count(c, EX_DLINKS); link_trg(c, *ra, R[I.b * stride]); break;
      case I_LINKCONST: count(c, EX_DLINKS); link_trg_port(c, *ra, I.port); break;
      case I_CTR: do_ctr(c, I.lab, *ra, R[I.b * stride], R[I.c * stride]); break;
      case I_OP: do_op(c, I.op, *ra, R[I.b * stride], R[I.c * stride]); break;
      case I_OPNUM: R[I.c * stride] = do_op_num(c, I.op, *ra, uint32_t(I.port)); break;
      case I_SWITCH: do_switch(c, *ra, R[I.b * stride], R[I.c * stride]); break;
      case I_WIRES: {
        ull a = alloc(c);
        R[I.a * stride] = pvar(a);
        R[I.b * stride] = a;
        R[I.c * stride] = pvar(a ^ 8);
        R[I.d * stride] = a ^ 8;
        break;
      }
      case I_CAPTURE: capture(c, I.port, *ra); break;
    }
  }
}
HVM_COLD void exec_large(const Ctx& c, const DevDef& d, ull t0) {
  if (d.nregs <= LOCAL_REGS) {
    ull R[LOCAL_REGS];
    return exec(c, d, t0, R, 1, g_P.instrs + d.ins_off);
  }
  // (the reference grows its register scratch to any Def, runtime/src/def.rs:221-223)
  if (!c.W->bigregs || d.nregs > MAX_REGS) return run_fail(c.net, HVM64_ERR_BAD_INPUT, d.nregs);
  exec(c, d, t0, c.W->bigregs + c.lane, 32, g_P.instrs + d.ins_off);
}
// A compiled build (hvm64 compile) includes the Book's Defs as functions;
// they run when the loaded Book is the one they were generated from.
#ifdef HVM_GEN_INCLUDE
#include HVM_GEN_INCLUDE
#endif
HVM_COLD void run_def(const Ctx& c, unsigned id, ull t0) {
  PROF_RULE(5)
  if (id >= g_P.ndefs) return run_fail(c.net, HVM64_ERR_BAD_INPUT, id);
#ifdef HVM_GEN_INCLUDE
  if (g_P.gen && gen_call(c, id, t0)) return;
#endif
  ull* R = c.W->regs + c.lane;
  if (id == c.W->icache_def) {  // staged by the warp for this step
    const DevDef& d = c.W->idef;
    if (d.nregs <= SMALL_REGS) return exec(c, d, t0, R, 32, c.W->icache);
    return exec_large(c, d, t0);
  }
  const DevDef d = g_P.defs[id];
  if (d.nregs <= SMALL_REGS) exec(c, d, t0, R, 32, g_P.instrs + d.ins_off);
  else exec_large(c, d, t0);
}

// def.rs:30-37 (LabSet::has); the expansion agent's set is LabSet::ALL.
HVM_INL bool def_has(const Ctx& c, ull ref, unsigned lab) {
  if (ref & X_BIT) return lab < 0xFFFF;
  unsigned id = unsigned((paddr(ref) >> 3) - 1);
  if (id >= g_P.ndefs) {
    run_fail(c.net, HVM64_ERR_BAD_INPUT, ref);
    return true;
  }
  const DevDef& d = g_P.defs[id];
  if (lab >= d.min_safe) return false;
  unsigned w = lab >> 6;
  if (w >= d.lab_len) return false;
  return (g_P.labbits[d.lab_off + w] >> (lab & 63)) & 1;
}

// ---- expansion agent (runtime/src/net.rs:63-108) ----------------------------
// An agent is a Ref port with X_BIT whose address names a heap word holding
// its output port (the reference boxes an `ExpandDef { out }`).
HVM_COLD ull new_expand(const Ctx& c, ull out) {
  ull w = alloc(c);
  half_free(c, w ^ 8);
  hstore(c, w, out);
  return mkport(T_REF, 0xFFFF, X_BIT | w);
}
HVM_COLD ull take_expand(const Ctx& c, ull port) {
  ull w = paddr(port) & ~X_BIT;
  unsigned it = 0;
  ull out;
  while ((out = hload(c, w)) == P_LOCK)
    if (!run_spin(c.net, it)) break;
  half_free(c, w);
  return out;
}
HVM_COLD void call(const Ctx& c, ull port, ull trg);
HVM_COLD void expand_call(const Ctx& c, ull self, ull port) {
  if (ptag(port) == T_REF && port != P_ERA) {
    if (port & X_BIT) {
      ull a = take_expand(c, self), b = take_expand(c, port);
      return link_port_port(c, a, b);
    }
    return call(c, port, self);
  }
  ull out = take_expand(c, self);
  unsigned t = ptag(port);
  if (t == T_RED) return run_fail(c.net, HVM64_ERR_BAD_PAIR, port);
  if (t == T_REF || t == T_NUM || t == T_VAR) return link_port_port(c, out, port);
  ull o1 = paddr(port);
  ull n = alloc(c);
  link_port_port(c, out, mkport(t, plab(port), n));
  link_wire_port(c, o1, new_expand(c, pvar(n)));
  link_wire_port(c, o1 ^ 8, new_expand(c, pvar(n ^ 8)));
}
// net.rs:65-69
HVM_COLD ull expand(const Ctx& c, ull root) {
  ull a = alloc(c);
  half_free(c, a ^ 8);
  link_wire_port(c, root, new_expand(c, pvar(a)));
  return a;
}
// def.rs:177-189
HVM_COLD void call(const Ctx& c, ull port, ull trg) {
  if (ptag(trg) == T_CTR && !def_has(c, port, plab(trg))) return comm02(c, port, trg);
  count(c, RW_DREF);
  if (port & X_BIT) return expand_call(c, port, trg);
  unsigned before = LS(allocs);
  run_def(c, unsigned((paddr(port) >> 3) - 1), trg);
  count(c, EX_DNODES, LS(allocs) - before);
}

// ---- interact.rs:6-44 ----------------------------------------------------------
HVM_COLD void interact(const Ctx& c, ull a, ull b) {
  PROF_RULE(7)
  unsigned at = ptag(a), bt = ptag(b);
  if (at <= T_VAR || bt <= T_VAR) return run_fail(c.net, HVM64_ERR_BAD_PAIR, a);
  bool an = at == T_REF || at == T_NUM, bn = bt == T_REF || bt == T_NUM;
  if (at == T_REF && bn && !skippable(a)) return call(c, a, b);
  if (an && bt == T_REF && !skippable(b)) return call(c, b, a);
  if (an && bn) return count(c, RW_ERAS);
  if (at == T_CTR && bt == T_SWITCH && plab(a) != 0) return comm22(c, a, b);
  if (at == T_SWITCH && bt == T_CTR && plab(b) != 0) return comm22(c, a, b);
  if ((at == T_CTR && bt == T_OP) || (at == T_OP && bt == T_CTR)) return comm22(c, a, b);
  if (at == T_CTR && bt == T_CTR && plab(a) != plab(b)) return comm22(c, a, b);
  if (at == bt && at >= T_OP) return anni2(c, a, b);
  if (at == T_REF && bt == T_CTR && plab(b) >= plab(a)) return comm02(c, a, b);
  if (at == T_CTR && bt == T_REF && plab(a) >= plab(b)) return comm02(c, b, a);
  if (at == T_NUM && bt == T_CTR) return comm02(c, a, b);
  if (at == T_CTR && bt == T_NUM) return comm02(c, b, a);
  if (at == T_REF && a == P_ERA) return comm02(c, a, b);
  if (bt == T_REF && b == P_ERA) return comm02(c, b, a);
  if (at == T_REF) return call(c, a, b);
  if (bt == T_REF) return call(c, b, a);
  if (at == T_OP && bt == T_NUM) return op_num(c, a, b);
  if (at == T_NUM && bt == T_OP) return op_num(c, b, a);
  if (at == T_SWITCH && bt == T_NUM) return switch_num(c, a, b);
  if (at == T_NUM && bt == T_SWITCH) return switch_num(c, b, a);
  run_fail(c.net, HVM64_ERR_BAD_PAIR, a);
}

// ---- normal-form gather (device-side readback) -------------------------------
// Walks net `net`'s normal form from word `root` the way host readback does
// (host/src/readback.rs:23-87): the root word, both words of every node it
// reaches, each redirect chain a Var goes through.  Writes the first `cap`
// (address, word) pairs to `out` and returns how many there are; `stk` (scap
// entries) is the depth-first stack.  *deep is set when the stack overflowed
// (the count is then incomplete).
HVM_COLD unsigned gather_walk(unsigned net, ull root, ull* out, unsigned cap, ull* stk,
                                             unsigned scap, bool* deep) {
  const ull hb = g_P.heap_bytes;
  unsigned sp = 0, n = 0;
  auto emit = [&](ull w, ull v) {
    if (n < cap) {
      out[2 * n] = w;
      out[2 * n + 1] = v;
    }
    n++;
  };
  auto live = [&](ull p) {
    ull a = p & A_MASK;
    return (p >> 48) == 0 && a != 0 && a < hb;
  };
  stk[sp++] = root;
  while (sp) {
    ull w = stk[--sp];
    ull v = ld_gpu(heap_at(net, w));
    emit(w, v);
    unsigned t = unsigned(v & 7);
    if (t == T_VAR || t == T_RED) {
      if (live(v)) {
        ull e = paddr(v);
        for (unsigned g = 0; g < (1u << 20); g++) {
          ull x = ld_gpu(heap_at(net, e));
          emit(e, x);
          if ((x & 7) != T_RED || !live(x)) break;
          e = paddr(x);
        }
      }
    } else if (t == T_OP || t == T_CTR || t == T_SWITCH) {
      if (sp + 2 > scap) {
        *deep = true;
        break;
      }
      ull a = paddr(v);
      stk[sp++] = a ^ 8;
      stk[sp++] = a;
    }
  }
  return n;
}

// A normal form split for a parallel gather.  A single walk is a chain of
// dependent loads, so one thread first expands the top of the tree breadth
// first (at most GTOP words, until a level holds 32 items or more); the items
// left at the edge, and every word that starts a redirect chain, become
// subtrees that other threads walk with gather_walk.  Every subtree's pairs
// form one contiguous run of gather_walk's depth-first order, so sizes summed
// bottom-up over the expanded top give every run's offset.
constexpr unsigned GTOP = 512, GTASKS = 256;
enum : unsigned char { GATHER_LEAF = 0, GATHER_NODE = 1, GATHER_SUB = 2 };
struct GatherTop {
  ull* w;              // the item's word address
  ull* v;              // its word (leaf and node items)
  ull* sz;             // size in pairs, then (gather_place) offset
  unsigned* ref;       // node: index of its first child (the second follows); subtree: its number
  unsigned char* kind;
  unsigned nt, nk;     // items, subtrees
};
HVM_DEV void gather_top(unsigned net, ull root, GatherTop& T) {
  const ull hb = g_P.heap_bytes;
  auto live = [&](ull p) {
    ull a = p & A_MASK;
    return (p >> 48) == 0 && a != 0 && a < hb;
  };
  unsigned nt = 1, nk = 0, lo = 0, hi = 1, depth = 0;
  T.w[0] = root;
  while (lo < hi) {
    const unsigned width = hi - lo;
    // (expanding a level adds at most `width` chain subtrees and 2 * width
    // items to the next level, which may all become subtrees: checked here so
    // that the numbers of items and subtrees stay within the arrays)
    if (width >= 32u || nt + 2 * width > GTOP || nk + 3 * width > GTASKS || depth >= 48) {
      for (unsigned k = lo; k < hi; k++) {  // the edge: subtrees
        T.kind[k] = GATHER_SUB;
        T.ref[k] = nk++;
      }
      break;
    }
    for (unsigned k = lo; k < hi; k++) {
      ull v = ld_gpu(heap_at(net, T.w[k]));
      T.v[k] = v;
      unsigned t = unsigned(v & 7);
      if (t == T_OP || t == T_CTR || t == T_SWITCH) {
        T.kind[k] = GATHER_NODE;
        T.ref[k] = nt;
        T.w[nt++] = paddr(v);
        T.w[nt++] = paddr(v) ^ 8;
      } else if ((t == T_VAR || t == T_RED) && live(v)) {
        T.kind[k] = GATHER_SUB;  // a redirect chain: walked as a subtree
        T.ref[k] = nk++;
      } else {
        T.kind[k] = GATHER_LEAF;
      }
    }
    lo = hi;
    hi = nt;
    depth++;
  }
  T.nt = nt;
  T.nk = nk;
}
// Sizes bottom-up from the subtrees' counts (tc, by subtree number); returns
// the whole walk's pair count.  (Children follow their parent in T.)
HVM_DEV ull gather_sizes(GatherTop& T, const unsigned* tc) {
  for (unsigned k = T.nt; k-- > 0;)
    T.sz[k] = T.kind[k] == GATHER_LEAF ? 1
              : T.kind[k] == GATHER_SUB ? ull(tc[T.ref[k]])
                                        : 1 + T.sz[T.ref[k]] + T.sz[T.ref[k] + 1];
  return T.sz[0];
}
// After gather_sizes: turns sizes into offsets (a node reads its first child's
// size before overwriting it with the child's offset) and writes the top's
// own words at theirs; the subtrees then go at T.sz[k].
HVM_DEV void gather_place(GatherTop& T, const unsigned* tc, ull* dst) {
  (void)tc;
  T.sz[0] = 0;
  for (unsigned k = 0; k < T.nt; k++) {
    const ull at = T.sz[k];
    if (T.kind[k] == GATHER_SUB) continue;
    dst[2 * at] = T.w[k];
    dst[2 * at + 1] = T.v[k];
    if (T.kind[k] == GATHER_NODE) {
      unsigned c = T.ref[k];
      ull s0 = T.sz[c];
      T.sz[c] = at + 1;
      T.sz[c + 1] = at + 1 + s0;
    }
  }
}

#undef LS
#undef FW

}  // namespace dev
}  // namespace hvm
