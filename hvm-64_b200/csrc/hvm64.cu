// Kernels, device queue, runner and C ABI of the B200 interaction-net reducer.
//
// Work distribution.  Each warp owns a LIFO redex stack in shared memory and
// processes up to 32 redexes per step, one per lane.  Redexes an interaction
// creates collect in a per-lane buffer and are appended to the warp's stack
// after the step (warp prefix sum).  Work moves between warps through one
// global lock-free queue of 32-redex slots (bounded MPMC ring with per-slot
// sequence numbers): a warp whose stack is deep donates its oldest redexes
// when other warps are hungry, spills when its stack would overflow, and an
// idle warp takes a slot.  A warp holds one net's work at a time, so batched
// reduction attributes every interaction to its net without tagging redexes.
//
// Termination, per net: `pending` counts the warps holding the net's work plus
// the net's queued slots.  A warp that takes a slot inherits the slot's unit;
// a donation adds one; a warp whose stack drains removes one.  Zero means
// normal form; the run ends when every net got there (`nets_left == 0`).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "device.cuh"

namespace hvm {
namespace dev {

// ---- global redex queue --------------------------------------------------------
// Single-thread reservation; data movement may be done by the whole warp.
// Never waits for a consumer: a full queue returns false at once and the
// caller keeps the work.  A lost CAS means another producer got its slot, so
// retrying under contention always makes progress; the retry count is still
// bounded (then the reservation fails like a full queue).
__device__ bool q_reserve_push(ull& pos) {
  Ctrl* C = g_P.ctrl;
  ull mask = C->q_mask;
  pos = ld_gpu(&C->q_tail);
  for (unsigned tries = 0; tries < (1u << 20); tries++) {
    Slot* s = &g_P.q[pos & mask];
    long long dif = (long long)ld_gpu(&s->seq) - (long long)pos;
    if (dif == 0) {
      ull old = atomicCAS(&C->q_tail, pos, pos + 1);
      if (old == pos) return true;
      pos = old;
    } else if (dif < 0) {
      return false;  // full: the slot still holds the previous lap's redexes
    } else {
      pos = ld_gpu(&C->q_tail);
    }
    if ((tries & 63) == 63 && run_failed()) return false;
  }
  return false;
}
__device__ void q_publish(ull pos) {
  __threadfence();
  st_gpu(&g_P.q[pos & g_P.ctrl->q_mask].seq, pos + 1);
}
__device__ bool q_reserve_pop(ull& pos) {
  Ctrl* C = g_P.ctrl;
  ull mask = C->q_mask;
  pos = ld_gpu(&C->q_head);
  for (int tries = 0; tries < 64; tries++) {
    Slot* s = &g_P.q[pos & mask];
    long long dif = (long long)ld_gpu(&s->seq) - (long long)(pos + 1);
    if (dif == 0) {
      ull old = atomicCAS(&C->q_head, pos, pos + 1);
      if (old == pos) return true;
      pos = old;
    } else if (dif < 0) {
      return false;  // empty
    } else {
      pos = ld_gpu(&C->q_head);
    }
  }
  return false;
}
__device__ void q_release(ull pos) {
  __threadfence();
  st_gpu(&g_P.q[pos & g_P.ctrl->q_mask].seq, pos + g_P.ctrl->q_mask + 1);
}

// Neither stack of the pushing warp had room (or the pusher has no overflow
// stack: the boot kernel): ship one redex as its own slot.  A full queue
// ends the run with HVM64_ERR_QUEUE instead of waiting for consumers, which
// could all be waiting the same way.
__device__ __noinline__ void push_overflow(unsigned net, ull a, ull b) {
  ull pos;
  if (!q_reserve_push(pos)) {
    run_fail(net, HVM64_ERR_QUEUE, 1);
    return;
  }
  atomicAdd(reinterpret_cast<ull*>(&g_P.nets[net].pending), 1ull);
  Slot* s = &g_P.q[pos & g_P.ctrl->q_mask];
  st_gpu(reinterpret_cast<ull*>(&s->net), (1ull << 32) | net);
  st_gpu(&s->r[0], a);
  st_gpu(&s->r[1], b);
  q_publish(pos);
  atomicAdd(&g_P.ctrl->stat_overflow, 1ull);
}

__device__ __forceinline__ ull shfl(ull v, int src) { return __shfl_sync(0xffffffffu, v, src); }

// Warp-cooperative: publish one queue slot of net `cur` holding the redexes
// (ra, rb) of lanes < cnt.  Returns false, changing nothing, when the queue
// has no room.
__device__ bool donate_vals(ull ra, ull rb, unsigned cnt, int cur) {
  const unsigned lane = threadIdx.x & 31;
  ull pos = 0;
  int ok = 0;
  if (lane == 0) {
    ok = q_reserve_push(pos) ? 1 : 0;
    if (ok) atomicAdd(reinterpret_cast<ull*>(&g_P.nets[cur].pending), 1ull);
  }
  ok = __shfl_sync(0xffffffffu, ok, 0);
  if (!ok) return false;
  pos = shfl(pos, 0);
  Slot* s = &g_P.q[pos & g_P.ctrl->q_mask];
  if (lane < cnt) {
    st_gpu(&s->r[2 * lane], ra);
    st_gpu(&s->r[2 * lane + 1], rb);
  }
  if (lane == 0) st_gpu(reinterpret_cast<ull*>(&s->net), (ull(cnt) << 32) | unsigned(cur));
  __threadfence();
  __syncwarp();
  if (lane == 0) q_publish(pos);
  return true;
}
// The `cnt` oldest redexes of the warp's shared-memory stack into a slot.
__device__ bool donate(const ull* S, unsigned& bot, unsigned cnt, int cur) {
  const unsigned lane = threadIdx.x & 31;
  unsigned k = (bot + lane) & (SCAP - 1);
  ull ra = lane < cnt ? S[2 * k] : 0, rb = lane < cnt ? S[2 * k + 1] : 0;
  if (!donate_vals(ra, rb, cnt, cur)) return false;
  bot += cnt;
  return true;
}
// The 32 newest redexes of the warp's overflow stack into a slot.
__device__ bool donate_spill(WarpSmem& W, int cur) {
  const unsigned lane = threadIdx.x & 31;
  unsigned n = W.sp_n;
  if (n < 32u) return false;
  ull i = n - 32u + lane;
  ull ra = W.sp[2 * i], rb = W.sp[2 * i + 1];
  if (!donate_vals(ra, rb, 32u, cur)) return false;
  __syncwarp();
  if (lane == 0) W.sp_n = n - 32u;
  __syncwarp();
  return true;
}

// Fold the lanes' per-step counts into the warp's counters.
__device__ __forceinline__ void fold_counts(WarpSmem& W) {
  const unsigned lane = threadIdx.x & 31;
  __syncwarp();
#pragma unroll
  for (int k = 0; k < NCOUNT; k++) {
    unsigned v = __reduce_add_sync(0xffffffffu, W.cnt[k * 32 + lane]);
    W.cnt[k * 32 + lane] = 0;
    if (lane == 0 && v) W.rw[k] += v;
  }
  __syncwarp();
}

// The same, out of line; a run with an interaction limit also adds what was
// folded to the run's total and stops the run once the total passes the
// limit (Net::reduce(limit), runtime/src/net.rs:41-52; checked every fold, so
// a run may overshoot by what its warps do between folds).
__device__ __noinline__ void fold_counts_cold(WarpSmem& W, int cur) {
  const unsigned lane = threadIdx.x & 31;
  __syncwarp();
  ull done = 0;
#pragma unroll
  for (int k = 0; k < NCOUNT; k++) {
    unsigned v = __reduce_add_sync(0xffffffffu, W.cnt[k * 32 + lane]);
    W.cnt[k * 32 + lane] = 0;
    if (lane == 0 && v) W.rw[k] += v;
    if (k <= RW_OPER) done += v;
  }
  if (lane == 0 && g_P.rw_limit && done && atomicAdd(&g_P.ctrl->rw_done, done) + done > g_P.rw_limit)
    run_fail(unsigned(cur), HVM64_ERR_LIMIT, g_P.rw_limit);
  __syncwarp();
}

// Flush the warp's counters into its net (one atomic per counter).
__device__ void flush_counters(WarpSmem& W, int cur) {
  const unsigned lane = threadIdx.x & 31;
  fold_counts(W);
  if (lane < unsigned(NCOUNT)) {
    ull v = W.rw[lane];
    if (v) atomicAdd(&g_P.nets[cur].rw[lane], v);
    W.rw[lane] = 0;
  }
  __syncwarp();
}

// ---- serving -------------------------------------------------------------------
// A served net's normal form leaves the device as the (address, word) pairs
// that host readback (host/src/readback.rs:23-87) would load: the root word,
// both words of every node it reaches, and each redirect chain a Var goes
// through.  Lane 0 walks it depth-first, using the warp's redex ring (empty
// when a net completes) as its stack, and writes the pairs into the slot's
// output in mapped host memory.
// A served net's normal form leaves the device as gathered pairs in the
// slot's output (mapped host memory).  Lane 0 walks it, using the warp's redex
// ring (empty when a net completes) as its stack.
__device__ __noinline__ unsigned serve_gather(WarpSmem& W, unsigned slot, ull root, int& status) {
  ull* out = g_P.out + ull(slot) * g_P.out_cap * 2;
  bool deep = false;
  unsigned n = gather_walk(slot, root, out, g_P.out_cap, W.stk, 2 * SCAP, &deep);
  if (deep || n > g_P.out_cap) status = HVM64_ERR_OUTPUT;
  return n < g_P.out_cap ? n : g_P.out_cap;
}

// Batch readback on the device: one warp per net counts its normal form's
// (address, word) pairs (out == nullptr) or writes them at offs[i], in
// gather_walk's order, with the net split into subtrees walked by the lanes
// (gather_top, gather_sizes, gather_place).  The count pass keeps each
// subtree's count in tcounts (GTASKS per net) for the write pass.  A net
// whose walk overflows a lane's stack gets count ~0u and is read back from a
// heap image instead.
constexpr unsigned GATHER_STACK = 256;
__global__ void __launch_bounds__(32) gather_kernel(unsigned first, unsigned n, unsigned* counts, const ull* offs,
                                                    ull* out, unsigned* tcounts) {
  __shared__ ull tw[GTOP], tv[GTOP], tsz[GTOP];
  __shared__ unsigned tref[GTOP];
  __shared__ unsigned char tkind[GTOP];
  __shared__ unsigned ntop, bad;
  const unsigned lane = threadIdx.x;
  if (blockIdx.x >= n) return;
  const unsigned i = first + blockIdx.x;
  if (out && counts[i] == ~0u) return;
  unsigned* tc = tcounts + size_t(blockIdx.x) * GTASKS;
  GatherTop T{tw, tv, tsz, tref, tkind, 0, 0};
  if (lane == 0) {
    gather_top(i, g_P.nets[i].root, T);
    ntop = T.nt;
    bad = 0;
  }
  __syncwarp();
  T.nt = ntop;
  ull stk[GATHER_STACK];
  if (!out) {
    for (unsigned k = lane; k < T.nt; k += 32) {
      if (tkind[k] != GATHER_SUB) continue;
      bool deep = false;
      unsigned c = gather_walk(i, tw[k], nullptr, 0, stk, GATHER_STACK, &deep);
      tc[tref[k]] = deep ? ~0u : c;
      if (deep) bad = 1;
    }
    __syncwarp();
    if (lane == 0) {
      ull total = gather_sizes(T, tc);
      counts[i] = (bad || total >= 0xFFFFFFFFull) ? ~0u : unsigned(total);
    }
    return;
  }
  ull* dst = out + 2 * offs[i];
  if (lane == 0) {
    gather_sizes(T, tc);
    gather_place(T, tc, dst);
  }
  __syncwarp();
  for (unsigned k = lane; k < T.nt; k += 32) {
    if (tkind[k] != GATHER_SUB) continue;
    bool deep = false;
    gather_walk(i, tw[k], dst + 2 * tsz[k], tc[tref[k]], stk, GATHER_STACK, &deep);
  }
}

// After a served net's normal form is gathered, nothing refers to its nodes
// any more: every node the normal form reaches (through principal ports, as
// the gather walks it) and the root node go back on lane 0's free list, so a
// long-running server reuses them for later requests.  The walk uses the
// warp's ring as its stack; a normal form deeper than that keeps the rest.
__device__ __noinline__ void serve_release(WarpSmem& W, unsigned slot, ull root) {
  ull* stk = W.stk;
  const unsigned cap = 2 * SCAP;
  unsigned sp = 0;
  ull w0 = ld_gpu(heap_at(slot, root));
  auto visit = [&](ull v) {
    unsigned t = unsigned(v & 7);
    if ((t == T_OP || t == T_CTR || t == T_SWITCH) && sp < cap) stk[sp++] = paddr(v);
  };
  visit(w0);
  for (unsigned guard = 0; sp && guard < (1u << 24); guard++) {
    ull a = stk[--sp];
    ull l = ld_gpu(heap_at(slot, a)), r = ld_gpu(heap_at(slot, a | 8));
    visit(l);
    visit(r);
    st_gpu(heap_at(slot, a | 8), P_LOCK);
    free_list_push(slot, &W.ovf[0], a);
  }
  // the root node: its left word held the root wire, its right half was
  // freed when the root was allocated (runtime/src/net.rs:65-69)
  ull rn = root & ~8ull;
  st_gpu(heap_at(slot, rn | 8), P_LOCK);
  free_list_push(slot, &W.ovf[0], rn);
  mem_fence();
}

// The net in `slot` reached normal form: gather it and post its completion
// record (the ticket last, after a system-scope fence).  Lane 0 only.
__device__ __noinline__ void serve_complete(WarpSmem& W, unsigned slot) {
  __threadfence();
  NetState& ns = g_P.nets[slot];
  int status = ld_gpu32(&ns.status);
  if (ld_gpu32(&g_P.ctrl->error)) status = ld_gpu32(&g_P.ctrl->error);
  ull root = ld_gpu(&ns.root);
  unsigned n = serve_gather(W, slot, root, status);
  volatile ServeDone* d = g_P.done + slot;
  d->status = status;
  d->pairs = n;
  d->root = root;
  for (int k = 0; k < NCOUNT; k++) d->rw[k] = ld_gpu(&ns.rw[k]);
  d->t_admit = ld_gpu(&ns.t_admit);
  d->t_done = globaltimer();
  __threadfence_system();
  d->ticket = ld_gpu(&ns.ticket);
  __threadfence_system();
  if (status == 0) serve_release(W, slot, root);
}

// Take the next request, if the host has written one, and boot it in this
// warp: its first redexes land in the (empty) ring.  Lane 0 only; returns the
// slot + 1, or 0.
__device__ __noinline__ unsigned serve_admit(WarpSmem& W, Ctx& c) {
  Ctrl* C = g_P.ctrl;
  ull t = ld_gpu(&C->req_tail);
  ull h = ld_gpu(&C->req_head);
  bool got = false;
  while (h < t) {
    ull old = atomicCAS(&C->req_head, h, h + 1);
    if (old == h) {
      got = true;
      break;
    }
    h = old;
  }
  if (!got) return 0;
  mem_fence();
  const ServeReq* r = g_P.req + (h % g_P.req_cap);
  ull ticket = ld_gpu(&r->ticket);
  ull sp = ld_gpu(reinterpret_cast<const ull*>(&r->slot));
  unsigned slot = unsigned(sp), prog = unsigned(sp >> 32);
  if (slot >= g_P.nnets) {
    run_fail(0, HVM64_ERR_BAD_INPUT, slot);
    return 0;
  }
  NetState& ns = g_P.nets[slot];
  for (int k = 0; k < NCOUNT; k++) st_gpu(&ns.rw[k], 0);
  st_gpu(reinterpret_cast<ull*>(&ns.pending), 1);  // this warp holds the new net
  ns.prog = int(prog);
  ns.status = 0;
  st_gpu(&ns.ticket, ticket);
  st_gpu(&ns.t_admit, globaltimer());
  mem_fence();
  atomicAdd(reinterpret_cast<ull*>(&C->nets_left), 1ull);
  c.net = slot;
  W.ring_base = 0;
  W.ring_cap = unsigned(SCAP - HEADROOM);
  W.ring_cnt = 0;
  ull root = alloc(c);
  half_free(c, root ^ 8);  // only the left word is the root wire; the node is reclaimed once it is freed
  if (prog < g_P.ndefs && !(g_P.defs[prog].flags & 1)) W.rw[RW_DREF]++;
  run_def(c, prog, pvar(root));
  settle(c);
  root = expand(c, root);
  settle(c);
  st_gpu(&ns.root, root);
  return slot + 1;
}

#ifndef HVM_QW
#define HVM_QW 2
#endif
constexpr int QW = HVM_QW;  // selection window: 32 * QW newest redexes

#ifndef HVM_MINB
#define HVM_MINB 7
#endif
constexpr size_t SMEM_BYTES = sizeof(WarpSmem) * WARPS;
static_assert(SMEM_BYTES <= 32 * 1024, "seven reducer blocks per SM must fit in shared memory");

__global__ void __launch_bounds__(THREADS, HVM_MINB) reduce_kernel() {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem& W = reinterpret_cast<WarpSmem*>(smem_raw)[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u, gt = ~lt & ~(1u << lane);
  ull* S = W.stk;
  Ctrl* C = g_P.ctrl;
  Ctx c{&W, lane, 0};
  lane_init(&W, lane);
  if (lane < unsigned(NCOUNT)) W.rw[lane] = 0;
#ifdef HVM_PROFILE_OPS
  W.prof[lane] = 0;
#endif
  if (lane == 0) {
    W.pool_n = 0;
    W.freed_n = 0;
    W.ring_cnt = 0;
    W.icache_def = ~0u;
    W.pool_cap = POOL;
    W.ring_base = 0;
    W.ring_cap = 0;
    const ull gw = ull(blockIdx.x) * WARPS + (threadIdx.x >> 5);
    W.sp = g_P.spill ? g_P.spill + 2ull * g_P.spill_cap * gw : nullptr;
    W.bigregs = g_P.bigregs ? g_P.bigregs + ull(32 * MAX_REGS) * gw : nullptr;
    W.sp_cap = g_P.spill ? g_P.spill_cap : 0u;
    W.sp_n = 0;
    W.st_steps = W.st_lanes = W.st_busy = W.st_idle = W.st_lane_sum = W.st_lane_max = 0;
  }
  __syncwarp();
  unsigned top = 0, bot = 0;  // warp-uniform ring indices
  int cur = -1;               // the net whose work this warp holds
  bool hungry = false;
  unsigned idle = 0, step = 0;
  // Deadline from this launch's start (a replayed launch gets a fresh one).
  const ull deadline = globaltimer() + C->timeout_ns;
  const long long born = clock64();
  unsigned nap = 0;  // idle backoff, ns

  for (;;) {
    // The error word is polled only now and then: every warp reading it each
    // step would make its L2 line a hot spot.
    if ((step & 31) == 0) {
      int err = 0;
      if (lane == 0) err = ld_gpu32(&C->error);
      if (__shfl_sync(0xffffffffu, err, 0)) break;
    }

    // Refill a low stack from the overflow stack (its newest redexes), so
    // steps stay full and the warp keeps the net while either holds work.
    {
      const unsigned spn = W.sp_n;
      constexpr unsigned LOW = unsigned(SCAP - HEADROOM) < 64u ? unsigned(SCAP - HEADROOM) : 64u;
      if (spn && top - bot < LOW) {
        unsigned m = min(spn, unsigned(SCAP - HEADROOM) - (top - bot));
        const ull* src = W.sp + 2ull * (spn - m);
        for (unsigned i = lane; i < m; i += 32) {
          unsigned k = (top + i) & (SCAP - 1);
          S[2 * k] = src[2 * i];
          S[2 * k + 1] = src[2 * i + 1];
        }
        top += m;
        __syncwarp();
        if (lane == 0) W.sp_n = spn - m;
        __syncwarp();
      }
    }

    if (top == bot) {
      if (cur >= 0) {
        flush_counters(W, cur);
        int fin = 0;
        if (lane == 0) {
          if (g_P.serve) __threadfence();  // this warp's heap writes, before its share is released
          long long old = (long long)atomicAdd(reinterpret_cast<ull*>(&g_P.nets[cur].pending), ~0ull);
          fin = old == 1;
          if (fin && g_P.serve) serve_complete(W, unsigned(cur));
          if (fin) atomicAdd(reinterpret_cast<ull*>(&C->nets_left), ~0ull);
        }
        __syncwarp();
        cur = -1;
      }
      ull pos = 0;
      int got = 0;
      if (lane == 0) got = q_reserve_pop(pos) ? 1 : 0;
      got = __shfl_sync(0xffffffffu, got, 0);
      if (!got) {
        // Idle: back off exponentially (1 us .. 64 us) so that waiting warps
        // do not crowd the queue's and the counters' L2 lines.
        int stop = 0;
        unsigned admitted = 0;
        if (lane == 0) {
          if (!hungry) atomicAdd(reinterpret_cast<ull*>(&C->hungry), 1ull);
          if (g_P.serve) {
            // Serving: boot the next request here, or end once the host has
            // asked to stop and nothing is admitted, queued or running.
            admitted = serve_admit(W, c);
            if (!admitted && ld_gpu32(&C->stop) && ld_gpu64s(&C->nets_left) <= 0 &&
                ld_gpu(&C->req_head) >= ld_gpu(&C->req_tail))
              stop = 1;
            else if (!admitted && (++idle & 15) == 0 && globaltimer() > deadline) {
              run_fail(0, HVM64_ERR_TIMEOUT, 3);  // a server lives at most timeout_ms
              stop = 1;
            }
          } else if (ld_gpu64s(&C->nets_left) <= 0) {
            stop = 1;
          } else if ((++idle & 15) == 0 && globaltimer() > deadline) {
            run_fail(0, HVM64_ERR_TIMEOUT, 1);
            stop = 1;
          }
          if (ld_gpu32(&C->error)) stop = 1;
        }
        hungry = true;
        if (__shfl_sync(0xffffffffu, stop, 0)) break;
        admitted = __shfl_sync(0xffffffffu, admitted, 0);
        if (admitted) {
          if (lane == 0) atomicAdd(reinterpret_cast<ull*>(&C->hungry), ~0ull);
          hungry = false;
          nap = 0;
          idle = 0;
          cur = int(admitted - 1);
          c.net = unsigned(cur);
          bot = 0;
          __syncwarp();  // lane 0's boot pushes are in shared memory before the others read the count
          {
            const unsigned cnt = W.ring_cnt;
            top = min(cnt, W.ring_cap);
            const unsigned spilled = spilled_of(&W, cnt);
            __syncwarp();
            if (lane == 0) W.sp_n += spilled;
            __syncwarp();
          }
          continue;
        }
        // (a serving reducer naps at most 8 us: new requests wait on it)
        nap = nap ? min(nap * 2, g_P.serve ? 8192u : 65536u) : 1024u;
        long long t0 = clock64();
        __nanosleep(nap);
        if (lane == 0) W.st_idle += ull(clock64() - t0);
        continue;
      }
      nap = 0;
      if (hungry && lane == 0) atomicAdd(reinterpret_cast<ull*>(&C->hungry), ~0ull);
      hungry = false;
      idle = 0;
      pos = shfl(pos, 0);
      __threadfence();
      Slot* s = &g_P.q[pos & C->q_mask];
      unsigned cnt = 0, net = 0;
      if (lane == 0) {
        ull meta = ld_gpu(reinterpret_cast<const ull*>(&s->net));
        net = unsigned(meta);
        cnt = unsigned(meta >> 32);
      }
      cnt = __shfl_sync(0xffffffffu, cnt, 0);
      net = __shfl_sync(0xffffffffu, net, 0);
      if (net >= g_P.nnets || cnt > unsigned(CHUNK)) {  // never expected; refuse to index with it
        if (lane == 0) run_fail(net, HVM64_ERR_BAD_ADDR, (ull(cnt) << 32) | net);
        break;
      }
      if (lane < cnt) {
        S[2 * lane] = ld_gpu(&s->r[2 * lane]);
        S[2 * lane + 1] = ld_gpu(&s->r[2 * lane + 1]);
      }
      __syncwarp();
      if (lane == 0) q_release(pos);
      bot = 0;
      top = cnt;
      cur = int(net);
      c.net = net;
      if (cnt == 0) continue;
    }

    // A run that never reaches normal form ends at the deadline.
    if ((++step & 1023) == 0) {
      int late = 0;
      if (lane == 0 && globaltimer() > deadline) {
        run_fail(unsigned(cur), HVM64_ERR_TIMEOUT, 2);
        late = 1;
      }
      if (__shfl_sync(0xffffffffu, late, 0)) break;
    }

    // Keep HEADROOM slots free for this step's new redexes: the oldest
    // redexes move to the overflow stack, or to the queue; if neither has
    // room the step's pushes overflow instead (nothing waits).
    while ((top - bot) > unsigned(SCAP - HEADROOM)) {
      const unsigned spn = W.sp_n;
      if (W.sp && spn + 32u <= W.sp_cap) {
        unsigned k = (bot + lane) & (SCAP - 1);
        W.sp[2ull * (spn + lane)] = S[2 * k];
        W.sp[2ull * (spn + lane) + 1] = S[2 * k + 1];
        bot += 32u;
        __syncwarp();
        if (lane == 0) W.sp_n = spn + 32u;
        __syncwarp();
      } else if (!donate(S, bot, 32u, cur)) {
        break;
      }
      if (lane == 0) atomicAdd(&C->stat_spilled, 1ull);
    }

    // Choose this step's redexes: among the newest 32 * QW, the rule class
    // most common among the newest 32 (ties: the newest); up to 32 of that
    // class run this step, one per lane, and the others go back on the stack
    // in their order.
    const unsigned w = min(top - bot, unsigned(32 * QW));
    ull qa[QW], qb[QW];
    bool qh[QW];
    unsigned qk[QW];
#pragma unroll
    for (int q = 0; q < QW; q++) {
      qh[q] = lane + 32u * q < w;
      qa[q] = qb[q] = 0;
      if (qh[q]) {
        unsigned k = (top - 1 - 32u * q - lane) & (SCAP - 1);
        qa[q] = S[2 * k];
        qb[q] = S[2 * k + 1];
      }
      qk[q] = qh[q] ? redex_class(qa[q], qb[q]) : 0xFFFFFFF0u + unsigned(q);
    }
    unsigned peers = __match_any_sync(0xffffffffu, qk[0]);
    unsigned score = qh[0] ? ((unsigned(__popc(peers)) << 8) | (255u - lane)) : 0u;
    unsigned best = __reduce_max_sync(0xffffffffu, score);
    unsigned key = __shfl_sync(0xffffffffu, qk[0], int(255u - (best & 255u)));
    unsigned nsel = 0, sr[QW], um[QW];
    bool st[QW], su[QW];
#pragma unroll
    for (int q = 0; q < QW; q++) {
      bool sq = qh[q] && qk[q] == key;
      unsigned m = __ballot_sync(0xffffffffu, sq);
      sr[q] = nsel + unsigned(__popc(m & lt));
      st[q] = sq && sr[q] < 32u;
      nsel += unsigned(__popc(m));
      su[q] = qh[q] && !st[q];
      um[q] = __ballot_sync(0xffffffffu, su[q]);
    }
    unsigned n = min(nsel, 32u);
    // Run only as many lanes as the stacks can take the pushes of (a lane of
    // a Def call pushes at most the Def's bound); the rest stay selected-out
    // and go back on the stack below.
    const unsigned nsel32 = n;
    {
      unsigned free_slots = unsigned(SCAP) - (top - bot) + n + (W.sp ? W.sp_cap - W.sp_n : 0u);
      unsigned lim = free_slots / pushes_bound(key);
      n = max(1u, min(n, lim));
    }
    unsigned base = top - w;
    __syncwarp();
    // Entries that stay keep their relative depth (older quarters lower; in a
    // quarter, higher lanes are older).
    unsigned below = 0;
#pragma unroll
    for (int q = QW - 1; q >= 0; q--) {
      if (st[q]) {
        W.sel[2 * sr[q]] = qa[q];
        W.sel[2 * sr[q] + 1] = qb[q];
      }
      if (su[q]) {
        unsigned k = (base + below + unsigned(__popc(um[q] & gt))) & (SCAP - 1);
        S[2 * k] = qa[q];
        S[2 * k + 1] = qb[q];
      }
      below += unsigned(__popc(um[q]));
    }
    top = base + below;
    if (n < nsel32) {  // selected beyond the lane cap: back on the stack
      __syncwarp();
      if (lane >= n && lane < nsel32) {
        unsigned k = (top + lane - n) & (SCAP - 1);
        S[2 * k] = W.sel[2 * lane];
        S[2 * k + 1] = W.sel[2 * lane + 1];
      }
      top += nsel32 - n;
    }
    if (lane == 0) {
      W.ring_cnt = 0;
      W.ring_base = top;
      W.ring_cap = unsigned(SCAP) - (top - bot);
    }
    // A step of Def calls: stage that Def's instructions in shared memory
    // (one cooperative load instead of a dependent fetch per instruction).
    // Every lane reads the staged Def's index before lane 0 may replace it:
    // lanes are not guaranteed to run this in lock-step, and a lane that saw
    // the new index would skip its share of the copy.
    __syncwarp();
    const unsigned staged = W.icache_def;
    __syncwarp();
#ifdef HVM_GEN_INCLUDE
    const bool vm_def = !(g_P.gen && key - 64u < HVM_GEN_NDEFS);  // compiled Defs need no staging
#else
    const bool vm_def = true;
#endif
    if (key >= 64u && key - 64u < g_P.ndefs && key - 64u != staged && vm_def) {
      unsigned id = key - 64u;
      const DevDef d = g_P.defs[id];
      if (d.ins_len <= ICACHE) {
        const uint4* src = reinterpret_cast<const uint4*>(g_P.instrs + d.ins_off);
        uint4* dst = reinterpret_cast<uint4*>(W.icache);
        for (unsigned i = lane; i < d.ins_len; i += 32) dst[i] = __ldg(src + i);
        if (lane == 0) {
          W.idef = d;
          W.icache_def = id;
        }
      } else if (lane == 0) {
        W.icache_def = ~0u;
      }
    }
    long long s0c = clock64();
    __syncwarp();
    unsigned mine = 0;
    if (lane < n) {
      long long l0 = clock64();
      interact(c, W.sel[2 * lane], W.sel[2 * lane + 1]);
      // (a call to settle only when the lane freed a word alone: measured
      // 5 % faster than calling it to find out)
      if (W.fw[lane] | W.fw[32 + lane] | W.fw[64 + lane] | W.fw[96 + lane]) settle(c);
      mine = unsigned(min(clock64() - l0, 0x7fffffffll));
    }
    __syncwarp();
    {
      unsigned mx = __reduce_max_sync(0xffffffffu, mine);
      unsigned sm = __reduce_add_sync(0xffffffffu, mine);
      if (lane == 0) {
        W.st_busy += ull(clock64() - s0c);
        W.st_lanes += n;
        W.st_steps++;
        W.st_lane_sum += sm;
        W.st_lane_max += mx;
      }
    }
    {
      const unsigned cnt = W.ring_cnt;
      top += min(cnt, W.ring_cap);
      const unsigned spilled = spilled_of(&W, cnt);
      __syncwarp();
      if (lane == 0) W.sp_n += spilled;
    }
    // The lanes' counters fold into the warp's when it lets its net go, and
    // out of line every 4096 steps (which bounds a lane's 32-bit counts);
    // folding every step measured 4 % slower.
    if ((step & 4095) == 0) fold_counts_cold(W, cur);
    else __syncwarp();
    // Nodes reclaimed in this step become allocatable after a fence.
    mem_fence();
    __syncwarp();
    {
      int pn = max(W.pool_n, 0);
      int fn = min(W.freed_n, POOL);
      int mv = min(fn, POOL - pn);
      for (int i = int(lane); i < mv; i += 32) W.pool[pn + i] = W.freed[i];
      for (int i = mv + int(lane); i < fn; i += 32) {
        // pool full: the rest goes to this lane's overflow list
        free_list_push(unsigned(cur), &W.ovf[lane], W.freed[i]);
      }
      __syncwarp();
      if (lane == 0) {
        W.pool_n = pn + mv;
        W.freed_n = 0;
      }
      __syncwarp();
    }

    // Share work when other warps are starving, and move work to the global
    // queue when the overflow stack is three quarters full: the overflow
    // stack first, then the oldest half of the shared-memory stack (at most
    // four slots per check).
    const bool sp_high = W.sp_n > W.sp_cap - W.sp_cap / 4u;
    if (top - bot + W.sp_n >= unsigned(C->donate_min) && ((step & 7) == 0 || sp_high)) {
      int give = 0;
      if (lane == 0) {
        long long h = ld_gpu64s(&C->hungry);
        long long queued = (long long)(ld_gpu(&C->q_tail) - ld_gpu(&C->q_head));
        // a net already spread over max_warps holders (warps and queued
        // slots) gets no more, except to relieve a full overflow stack
        ull cap = C->max_warps;
        bool spread = cap && (ull)ld_gpu64s(&g_P.nets[cur].pending) >= cap;
        give = (h > 0 && queued < h && !spread) ? 2 : sp_high ? 1 : 0;
      }
      give = __shfl_sync(0xffffffffu, give, 0);
      if (give) {
        unsigned k = 0;
        for (; k < 4u && W.sp_n >= 32u; k++) {
          if (!donate_spill(W, cur)) break;
          if (lane == 0) atomicAdd(&C->stat_donated, 1ull);
        }
        for (unsigned chunks = give == 2 ? min((top - bot) / 64u, 4u - k) : 0u; chunks; chunks--) {
          if (!donate(S, bot, 32u, cur)) break;
          if (lane == 0) atomicAdd(&C->stat_donated, 1ull);
        }
      }
    }
  }
  if (cur >= 0) flush_counters(W, cur);
  if (lane == 0) {
    atomicAdd(&C->stat_steps, W.st_steps);
    atomicAdd(&C->stat_lanes, W.st_lanes);
    atomicAdd(&C->stat_busy_cycles, W.st_busy);
    atomicAdd(&C->stat_idle_cycles, W.st_idle);
    atomicAdd(&C->stat_lane_sum, W.st_lane_sum);
    atomicAdd(&C->stat_lane_max, W.st_lane_max);
    atomicAdd(&C->stat_total, ull(clock64() - born));
#ifdef HVM_PROFILE_OPS
    for (int k = 0; k < 32; k++) atomicAdd(&C->stat_prof[k], W.prof[k]);
#endif
  }
}

// One warp per net (lane 0 does the work, its state in shared memory like
// the reducer's): allocate the root, run the boot program against it
// (Net::boot / Host::encode_net), then wrap the root in an expansion agent
// (Net::expand, runtime/src/net.rs:65-69).  Redexes collect in the warp's
// stack (SCAP of them; more go out one per queue slot) and the warp
// publishes them to the global queue in slots of up to 32.
__global__ void __launch_bounds__(THREADS) boot_kernel(unsigned first, unsigned count) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem& W = reinterpret_cast<WarpSmem*>(smem_raw)[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31;
  if (lane == 0) {
    W.icache_def = ~0u;
    W.pool_n = W.freed_n = 0;
    W.pool_cap = 0;
    W.sp = nullptr;
    W.sp_n = W.sp_cap = 0;
    const ull gw = ull(blockIdx.x) * WARPS + (threadIdx.x >> 5);
    W.bigregs = g_P.bigregs ? g_P.bigregs + ull(32 * MAX_REGS) * gw : nullptr;
    lane_init(&W, 0);
  }
  const unsigned stride = gridDim.x * WARPS;
  for (unsigned i = first + blockIdx.x * WARPS + (threadIdx.x >> 5); i < first + count; i += stride) {
    NetState& ns = g_P.nets[i];
    if (lane == 0) {
      W.ring_cnt = 0;
      W.ring_base = 0;
      W.ring_cap = SCAP;
      for (int k = 0; k < NCOUNT; k++) W.rw[k] = 0;
      Ctx c{&W, 0, i};
      ull root = alloc(c);
      unsigned prog = unsigned(ns.prog);
      if (prog < g_P.ndefs && !(g_P.defs[prog].flags & 1)) W.rw[RW_DREF]++;
      // Small Defs use register slots 0, 32, 64, ... of W.regs (lane 0's column).
      run_def(c, prog, pvar(root));
      settle(c);
      if (!g_P.no_expand) {
        root = expand(c, root);
        settle(c);
      }
      ns.root = root;
    }
    __syncwarp();
    const unsigned total = min(W.ring_cnt, unsigned(SCAP));
    for (unsigned done = 0; done < total; done += unsigned(CHUNK)) {
      unsigned k = min(total - done, unsigned(CHUNK));
      ull ra = lane < k ? W.stk[2 * (done + lane)] : 0, rb = lane < k ? W.stk[2 * (done + lane) + 1] : 0;
      if (!donate_vals(ra, rb, k, int(i))) {
        if (lane == 0) run_fail(i, HVM64_ERR_QUEUE, 2);
        break;
      }
    }
    if (lane == 0) {
      for (int k = 0; k < NCOUNT; k++) {
        ull v = W.rw[k] + W.cnt[k * 32];
        W.cnt[k * 32] = 0;
        if (v) atomicAdd(&ns.rw[k], v);
      }
      __threadfence();
      if (ld_gpu64s(&ns.pending) > 0) atomicAdd(reinterpret_cast<ull*>(&g_P.ctrl->nets_left), 1ull);
    }
    __syncwarp();
  }
}

__global__ void set_deadline_kernel(Ctrl* c, ull timeout_ns);

__global__ void queue_init_kernel(Slot* q, ull n) {
  ull i = ull(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) q[i].seq = i;
}

}  // namespace dev

// ===========================================================================
// Host runner
// ===========================================================================
namespace {

thread_local std::string g_error;

int set_error(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

#define CU(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) throw Error(HVM64_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

template <class T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (count <= n && p) return;
    release();
    if (count == 0) count = 1;
    CU(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
};

const char* status_name(int s) {
  switch (s) {
    case HVM64_OK: return "ok";
    case HVM64_ERR_OOM: return "out of memory (heap exhausted)";
    case HVM64_ERR_BAD_PAIR: return "no interaction rule for this pair";
    case HVM64_ERR_DIV0: return "attempt to divide by zero";
    case HVM64_ERR_TIMEOUT: return "timed out";
    case HVM64_ERR_BAD_INPUT: return "bad input";
    case HVM64_ERR_CUDA: return "CUDA error";
    case HVM64_ERR_QUEUE: return "device redex queue overflow";
    case HVM64_ERR_BAD_ADDR: return "heap address outside the arena";
    case HVM64_ERR_OUTPUT: return "normal form larger than the request's output buffer";
    case HVM64_ERR_LIMIT: return "interaction limit reached";
  }
  return "unknown error";
}

// Whether this build's compiled Def functions (hvm64 compile) are those of
// `book`: 1 runs them, 0 the instruction VM.
unsigned gen_matches(const Book& book) {
#ifdef HVM_GEN_INCLUDE
  return book.defs.size() >= HVM_GEN_NDEFS && defs_hash(book, HVM_GEN_NDEFS) == HVM_GEN_HASH ? 1u : 0u;
#else
  (void)book;
  return 0u;
#endif
}

// Resident reducer blocks per SM for a tuning (the occupancy limit when the
// tuning leaves it at 0).
int reducer_blocks_per_sm(const hvm64_tuning& t) {
  CU(cudaFuncSetAttribute(dev::reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dev::SMEM_BYTES)));
  int bps = int(t.blocks_per_sm);
  if (bps <= 0) {
    int occ = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, dev::reduce_kernel, dev::THREADS, dev::SMEM_BYTES));
    bps = std::max(1, occ);
  }
  return bps;
}

// Overflow-stack capacity per reducer warp: a power of two in [256, 8192]
// redexes, about half the heap's nodes spread over the warps (live redexes
// hold nodes, so a small heap cannot fill a large overflow stack).
unsigned spill_cap_for(uint64_t heap_bytes, uint64_t warps) {
  uint64_t per = heap_bytes / 16 / std::max<uint64_t>(warps, 1) / 2;
  unsigned c = 256;
  while (c < 8192 && c < per) c *= 2;
  return c;
}

// Boot kernel grid: one warp per net, at most 8 blocks per SM (grid-stride).
unsigned boot_blocks(unsigned count, int sms) {
  unsigned b = (count + dev::WARPS - 1) / dev::WARPS;
  return std::max(1u, std::min(b, unsigned(sms) * 8u));
}

// Runs on one device take turns: a run owns the device's constant-memory
// launch parameters (dev::g_P) from their upload until its kernels finish.
// A persistent reducer launch fills every SM, so runs of different handles
// would not overlap much anyway.  A server holds its device's turn for its
// whole life; another thread then waits (up to the given time) and the
// server's own thread is refused rather than deadlocked.
constexpr int MAX_DEVICES = 64;
struct DeviceSlot {
  std::mutex m;
  std::condition_variable cv;
  bool busy = false, server = false;
  std::thread::id owner;
};
DeviceSlot g_turns[MAX_DEVICES];

class DeviceTurn {
 public:
  DeviceTurn() = default;
  DeviceTurn(int device, uint64_t wait_ms, bool server = false) { take(device, wait_ms, server); }
  DeviceTurn(const DeviceTurn&) = delete;
  DeviceTurn& operator=(const DeviceTurn&) = delete;
  ~DeviceTurn() { release(); }
  void take(int device, uint64_t wait_ms, bool server) {
    if (device < 0 || device >= MAX_DEVICES) throw Error(HVM64_ERR_CUDA, "device index out of range");
    DeviceSlot& d = g_turns[device];
    std::unique_lock<std::mutex> lk(d.m);
    if (d.busy && d.owner == std::this_thread::get_id())
      throw Error(HVM64_ERR_BAD_INPUT, d.server ? "a server started by this thread holds the device: free it first"
                                                : "the device is already in use by this thread");
    if (!d.cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !d.busy; }))
      throw Error(HVM64_ERR_TIMEOUT, "the device stayed in use by another run (a server holds its device until freed)");
    d.busy = true;
    d.server = server;
    d.owner = std::this_thread::get_id();
    dev_ = device;
  }
  void release() {
    if (dev_ < 0) return;
    DeviceSlot& d = g_turns[dev_];
    {
      std::lock_guard<std::mutex> lk(d.m);
      d.busy = d.server = false;
      d.owner = std::thread::id();
    }
    d.cv.notify_all();
    dev_ = -1;
  }

 private:
  int dev_ = -1;
};

// Uploads a run's launch parameters on its stream (inside its turn).
void upload_params(const dev::Params& p, cudaStream_t st) {
  CU(cudaMemcpyToSymbolAsync(dev::g_P, &p, sizeof p, 0, cudaMemcpyHostToDevice, st));
}

}  // namespace

// Default redex-queue capacity: 2^20 slots (570 MB).  A warp whose stack is
// full ships redexes to the queue one per slot in the middle of a step, and a
// warp that finds the queue full waits for consumers; when every warp waits
// like that at once the run stops with TIMEOUT, so the queue is sized for
// bursts from Defs that create many redexes at once.
constexpr unsigned DEFAULT_QLOG2 = 20;

// Host staging for gathered normal forms, shared by the process's runs (one
// gather at a time holds it).  Page-locked up to 4 GiB, so the copy from the
// device runs at full link speed, and never zero-filled; it is kept for the
// life of the process.
struct HostStage {
  std::mutex mu;
  uint64_t* p = nullptr;
  size_t bytes = 0;
  bool pinned = false;
  uint64_t* reserve(size_t need) {  // the caller holds mu
    if (need <= bytes && p) return p;
    if (p) {
      if (pinned) cudaFreeHost(p);
      else delete[] p;
    }
    p = nullptr;
    bytes = 0;
    size_t want = std::max<size_t>(need, size_t(64) << 20);
    pinned = want <= (size_t(4) << 30) && cudaMallocHost(&p, want) == cudaSuccess;
    if (!pinned) {
      cudaGetLastError();  // a failed page-locked allocation is not an error of the run
      p = new uint64_t[(want + 7) / 8];
    }
    bytes = want;
    return p;
  }
};
HostStage g_stage;

// A set of nets reduced together on the current device.
struct Runner {
  Book book;
  std::vector<uint32_t> progs;  // per net: boot program (DevDef index)
  uint64_t heap_bytes = 0;
  int device = 0;
  int sms = 148;

  DevBuf<dev::ull> heap;
  DevBuf<dev::Ctrl> ctrl;
  DevBuf<dev::NetState> nets;
  DevBuf<dev::Slot> q;
  DevBuf<DevDef> d_defs;
  DevBuf<DevInstr> d_instrs;
  DevBuf<dev::ull> d_labbits;
  size_t uploaded_defs = 0;

  std::vector<dev::NetState> host_nets;
  dev::Ctrl host_ctrl{};
  std::vector<uint64_t> image;  // heap image for readback
  bool image_valid = false;
  bool reduced = false;
  uint64_t h2d = 0, d2h = 0;    // bytes copied by the last run + readbacks

  void setup(uint64_t bytes) {
    CU(cudaGetDevice(&device));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (bytes == 0) {
      size_t fr = 0, tot = 0;
      CU(cudaMemGetInfo(&fr, &tot));
      bytes = std::min<uint64_t>(uint64_t(fr) / 2, uint64_t(16) << 30);
    }
    heap_bytes = bytes & ~uint64_t(15);
    if (heap_bytes < 64) throw Error(HVM64_ERR_BAD_INPUT, "heap too small");
  }

  unsigned gen = 0;  // gen_matches(book), as of the last upload
  void upload_book() {
    if (uploaded_defs == book.defs.size() && d_defs.p) return;
    gen = gen_matches(book);
    d_defs.alloc(book.defs.size());
    d_instrs.alloc(book.instrs.size());
    d_labbits.alloc(book.labbits.size());
    CU(cudaMemcpy(d_defs.p, book.defs.data(), book.defs.size() * sizeof(DevDef), cudaMemcpyHostToDevice));
    h2d += book.defs.size() * sizeof(DevDef) + book.instrs.size() * sizeof(DevInstr) + book.labbits.size() * 8;
    if (!book.instrs.empty())
      CU(cudaMemcpy(d_instrs.p, book.instrs.data(), book.instrs.size() * sizeof(DevInstr), cudaMemcpyHostToDevice));
    if (!book.labbits.empty())
      CU(cudaMemcpy(d_labbits.p, book.labbits.data(), book.labbits.size() * 8, cudaMemcpyHostToDevice));
    uploaded_defs = book.defs.size();
  }

  dev::Params params() {
    dev::Params p{};
    p.heap = heap.p;
    p.heap_bytes = heap_bytes;
    p.ctrl = ctrl.p;
    p.nets = nets.p;
    p.nnets = unsigned(progs.size());
    p.q = q.p;
    p.defs = d_defs.p;
    p.instrs = d_instrs.p;
    p.labbits = d_labbits.p;
    p.ndefs = unsigned(book.defs.size());
    p.spill = spill.p;
    p.spill_cap = spill_cap;
    p.ovf_flush = dev::OVF_FLUSH;
    p.bigregs = bigregs.p;
    p.gen = gen;
    p.no_expand = no_expand ? 1u : 0u;
    p.rw_limit = rw_limit;
    p.capture = capture.p;
    p.capture_cap = capture.p ? unsigned(capture.n / 2) : 0u;
    return p;
  }

  // Pre-reduce runs (see PreReducer): boot without the expansion agent,
  // stop past an interaction limit (0: none), and a buffer for the redexes
  // inert Defs capture.
  bool no_expand = false;
  uint64_t rw_limit = 0;
  DevBuf<dev::ull> capture;

  // The reducer grid for a tuning, and the warps' overflow stacks sized to it.
  DevBuf<dev::ull> spill;
  unsigned spill_cap = 0, grid = 0;
  DevBuf<dev::ull> bigregs;
  void prepare_grid(const hvm64_tuning& t) {
    grid = unsigned(sms * reducer_blocks_per_sm(t));
    uint64_t warps = uint64_t(grid) * dev::WARPS;
    spill_cap = spill_cap_for(heap_bytes, warps);
    spill.alloc(2 * size_t(spill_cap) * warps);
    if (book.max_nregs() > LOCAL_REGS) {  // for the reducer's warps and the boot kernel's
      uint64_t w = std::max<uint64_t>(grid, uint64_t(sms) * 8) * dev::WARPS;
      bigregs.alloc(size_t(w) * 32 * MAX_REGS);
    }
  }

  // Reduce nets [first, first+count) (the rest stay untouched); the grid is
  // prepared (prepare_grid) for this tuning.
  void launch(unsigned first, unsigned count, cudaStream_t st) {
    upload_params(params(), st);
    dev::boot_kernel<<<boot_blocks(count, sms), dev::THREADS, dev::SMEM_BYTES, st>>>(first, count);
    CU(cudaGetLastError());
    dev::reduce_kernel<<<grid, dev::THREADS, dev::SMEM_BYTES, st>>>();
    CU(cudaGetLastError());
  }

  void reset_ctrl(const hvm64_tuning& t, cudaStream_t st, unsigned qlog2, uint64_t bump) {
    dev::Ctrl c{};
    c.bump = bump;  // node 0 is reserved
    c.heap_nodes = heap_bytes / 16;
    c.reuse_mark = c.heap_nodes / 2;  // free nodes are shared between warps once half the heap is used
    c.heap_bytes = heap_bytes;
    c.chunk_nodes = t.chunk_nodes ? t.chunk_nodes : 256;
    c.spin_limit = 1ull << 24;
    c.donate_min = t.donate_min ? t.donate_min : 64;
    c.max_warps = t.max_warps_per_net;
    c.q_mask = (1ull << qlog2) - 1;
    c.deadline = ~0ull;  // the boot kernel's deadline; warps of the reducer keep their own
    host_ctrl = c;
    CU(cudaMemcpyAsync(ctrl.p, &c, sizeof c, cudaMemcpyHostToDevice, st));
  }

  // Nets of the last run: [run_first, run_first + run_count).
  unsigned run_first = 0, run_count = 0;

  // Reduce nets [first, first + count) (count clamped to the batch); the
  // other nets' results of earlier runs become unavailable.
  void run(int mode, const hvm64_tuning* tp, double* device_ms, unsigned first = 0, unsigned count = ~0u) {
    hvm64_tuning t{};
    if (tp) t = *tp;
    if (first > progs.size()) throw Error(HVM64_ERR_BAD_INPUT, "net range starts past the batch");
    count = unsigned(std::min<uint64_t>(count, progs.size() - first));
    run_first = first;
    run_count = count;
    DeviceTurn turn(device, t.timeout_ms ? t.timeout_ms : 120000);
    unsigned qlog2 = t.queue_slots_log2 ? t.queue_slots_log2 : DEFAULT_QLOG2;
    if (qlog2 < 4 || qlog2 > 24) throw Error(HVM64_ERR_BAD_INPUT, "queue_slots_log2 out of range");
    h2d = d2h = 0;
    error_detail.clear();
    heap.alloc(heap_bytes / 8);
    ctrl.alloc(1);
    nets.alloc(progs.size());
    q.alloc(size_t(1) << qlog2);
    upload_book();
    prepare_grid(t);
    size_t qn = size_t(1) << qlog2;

    host_nets.assign(progs.size(), dev::NetState{});
    for (size_t i = 0; i < progs.size(); i++) host_nets[i].prog = int(progs[i]);
    if (!(mode == HVM64_BATCH_PERSISTENT && (t.flags & HVM64_TUNE_GRAPH))) {
      CU(cudaMemcpy(nets.p, host_nets.data(), host_nets.size() * sizeof(dev::NetState), cudaMemcpyHostToDevice));
      h2d += host_nets.size() * sizeof(dev::NetState);
    }

    stat_donated = stat_spilled = stat_overflow = 0;
    stat_steps = stat_lanes = stat_busy = stat_idle = 0;
    for (int k = 0; k < 8; k++) stat_g_steps[k] = stat_g_cycles[k] = 0;
    for (int k = 0; k < 32; k++) stat_prof[k] = 0;
    cudaStream_t st = 0;
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    uint64_t timeout_ms = t.timeout_ms ? t.timeout_ms : 120000;
    float total_ms = 0;
    uint64_t bump = 1;
    // One-net-per-launch runs keep every earlier net's nodes, so they take
    // small allocator chunks unless told otherwise.
    if (mode == HVM64_BATCH_PLAIN && t.chunk_nodes == 0) t.chunk_nodes = 32;
    auto one = [&](unsigned first, unsigned count) {
      // One-net-per-launch runs keep earlier nets' nodes: the bump carries on.
      reset_ctrl(t, st, qlog2, bump);
      dev::queue_init_kernel<<<unsigned((qn + 255) / 256), 256, 0, st>>>(q.p, qn);
      CU(cudaGetLastError());
      set_deadline(st, timeout_ms);
      host_ctrl.timeout_ns = timeout_ms * 1000000ull;
      CU(cudaMemcpyAsync(&ctrl.p->timeout_ns, &host_ctrl.timeout_ns, 8, cudaMemcpyHostToDevice, st));
      CU(cudaEventRecord(e0, st));
      launch(first, count, st);
      CU(cudaEventRecord(e1, st));
      CU(cudaEventSynchronize(e1));
      float ms = 0;
      CU(cudaEventElapsedTime(&ms, e0, e1));
      total_ms += ms;
      CU(cudaMemcpy(&host_ctrl, ctrl.p, sizeof host_ctrl, cudaMemcpyDeviceToHost));
      h2d += sizeof(dev::Ctrl);
      d2h += sizeof(dev::Ctrl);
      stat_donated += host_ctrl.stat_donated;
      stat_spilled += host_ctrl.stat_spilled;
      stat_overflow += host_ctrl.stat_overflow;
      stat_steps += host_ctrl.stat_steps;
      stat_lanes += host_ctrl.stat_lanes;
      stat_busy += host_ctrl.stat_busy_cycles;
      stat_idle += host_ctrl.stat_idle_cycles;
      for (int k = 0; k < 32; k++) stat_prof[k] += host_ctrl.stat_prof[k];
      stat_g_steps[0] += host_ctrl.stat_lane_sum;
      stat_g_steps[1] += host_ctrl.stat_lane_max;
      stat_g_steps[2] += host_ctrl.stat_total;
      bump = std::min<uint64_t>(host_ctrl.bump, heap_bytes / 16);
      if (host_ctrl.error) {
        for (unsigned k = first; k < first + count; k++) host_nets[k].status = host_ctrl.error;
        note_error(host_ctrl);
      }
    };
    if (mode == HVM64_BATCH_PLAIN) {
      for (unsigned i = first; i < first + count; i++) one(i, 1);
    } else if (t.flags & HVM64_TUNE_GRAPH) {
      total_ms = run_graph(t, qlog2, timeout_ms, first, count);
      CU(cudaMemcpy(&host_ctrl, ctrl.p, sizeof host_ctrl, cudaMemcpyDeviceToHost));
      d2h += sizeof(dev::Ctrl);
      stat_donated += host_ctrl.stat_donated;
      stat_spilled += host_ctrl.stat_spilled;
      stat_overflow += host_ctrl.stat_overflow;
      stat_steps += host_ctrl.stat_steps;
      stat_lanes += host_ctrl.stat_lanes;
      stat_busy += host_ctrl.stat_busy_cycles;
      stat_idle += host_ctrl.stat_idle_cycles;
      bump = std::min<uint64_t>(host_ctrl.bump, heap_bytes / 16);
      if (host_ctrl.error) {
        for (unsigned k = first; k < first + count; k++) host_nets[k].status = host_ctrl.error;
        note_error(host_ctrl);
      }
    } else {
      one(first, count);
    }
    CU(cudaEventDestroy(e0));
    CU(cudaEventDestroy(e1));
    std::vector<dev::NetState> got(progs.size());
    CU(cudaMemcpy(got.data(), nets.p, got.size() * sizeof(dev::NetState), cudaMemcpyDeviceToHost));
    d2h += got.size() * sizeof(dev::NetState);
    heap_used = bump;
    for (size_t i = 0; i < got.size(); i++) {
      int status = host_nets[i].status;
      host_nets[i] = got[i];
      host_nets[i].status = status;
    }
    if (device_ms) *device_ms = total_ms;
    image_valid = false;
    pairs_valid = false;
    reduced = true;
  }

  void set_deadline(cudaStream_t st, uint64_t timeout_ms);

  // What the device said about its first error (for the error message).
  std::string error_detail;
  void note_error(const dev::Ctrl& h) {
    if (!error_detail.empty()) return;
    if (h.error == HVM64_ERR_TIMEOUT)
      error_detail = h.error_info == 0
                         ? " (a bounded wait on a locked heap word gave up)"
                         : " (the run deadline, tuning timeout_ms, passed)";
    else if (h.error == HVM64_ERR_QUEUE)
      error_detail = " (net " + std::to_string(h.error_net) +
                     (h.error_info == 2 ? ": the boot redexes" : ": a warp's overflow stack was full and") +
                     " found the global redex queue full; a larger tuning queue_slots_log2 gives it more room)";
    else
      error_detail = " (net " + std::to_string(h.error_net) + ")";
  }
  std::string error_message(int code) const { return std::string(status_name(code)) + error_detail; }

  // A persistent run as one CUDA graph: net records, control block, queue
  // init, deadline, launch parameters, boot and reduce, captured once per
  // configuration and replayed by later runs.  Its host sources are
  // page-locked copies that stay valid while the graph does.
  cudaStream_t gs = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::vector<uint64_t> gkey;
  dev::Ctrl* pin_ctrl = nullptr;
  dev::NetState* pin_nets = nullptr;
  dev::Params* pin_params = nullptr;

  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    if (pin_ctrl) cudaFreeHost(pin_ctrl);
    if (pin_nets) cudaFreeHost(pin_nets);
    if (pin_params) cudaFreeHost(pin_params);
    pin_params = nullptr;
    pin_ctrl = nullptr;
    pin_nets = nullptr;
  }
  ~Runner() {
    drop_graph();
    if (gs) cudaStreamDestroy(gs);
  }

  float run_graph(const hvm64_tuning& t, unsigned qlog2, uint64_t timeout_ms, unsigned first, unsigned count) {
    size_t qn = size_t(1) << qlog2;
    const unsigned n = unsigned(progs.size());
    std::vector<uint64_t> key = {t.blocks_per_sm, t.chunk_nodes, t.donate_min, qlog2, t.max_warps_per_net, timeout_ms,
                                 first, count, uint64_t(heap.p), uint64_t(q.p), uint64_t(d_defs.p), uint64_t(spill.p),
                                 spill_cap, grid};
    for (auto p : progs) key.push_back(p);
    if (!gs) CU(cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking));
    if (!gexec || key != gkey) {
      drop_graph();
      CU(cudaHostAlloc(reinterpret_cast<void**>(&pin_ctrl), sizeof(dev::Ctrl), cudaHostAllocDefault));
      CU(cudaHostAlloc(reinterpret_cast<void**>(&pin_nets), sizeof(dev::NetState) * std::max<size_t>(n, 1),
                       cudaHostAllocDefault));
      memcpy(pin_nets, host_nets.data(), sizeof(dev::NetState) * n);
      dev::Ctrl c{};
      c.bump = 1;
      c.heap_nodes = heap_bytes / 16;
      c.reuse_mark = c.heap_nodes / 2;  // free nodes are shared between warps once half the heap is used
      c.heap_bytes = heap_bytes;
      c.chunk_nodes = t.chunk_nodes ? t.chunk_nodes : 256;
      c.spin_limit = 1ull << 24;
      c.donate_min = t.donate_min ? t.donate_min : 64;
      c.max_warps = t.max_warps_per_net;
      c.q_mask = qn - 1;
      c.deadline = ~0ull;
      c.timeout_ns = timeout_ms * 1000000ull;
      *pin_ctrl = c;
      CU(cudaHostAlloc(reinterpret_cast<void**>(&pin_params), sizeof(dev::Params), cudaHostAllocDefault));
      *pin_params = params();
      CU(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaSuccess;
      auto step = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
      };
      step(cudaMemcpyAsync(nets.p, pin_nets, sizeof(dev::NetState) * n, cudaMemcpyHostToDevice, gs));
      step(cudaMemcpyAsync(ctrl.p, pin_ctrl, sizeof(dev::Ctrl), cudaMemcpyHostToDevice, gs));
      dev::queue_init_kernel<<<unsigned((qn + 255) / 256), 256, 0, gs>>>(q.p, qn);
      step(cudaGetLastError());
      dev::set_deadline_kernel<<<1, 1, 0, gs>>>(ctrl.p, c.timeout_ns);
      step(cudaGetLastError());
      step(cudaMemcpyToSymbolAsync(dev::g_P, pin_params, sizeof(dev::Params), 0, cudaMemcpyHostToDevice, gs));
      dev::boot_kernel<<<boot_blocks(count, sms), dev::THREADS, dev::SMEM_BYTES, gs>>>(first, count);
      step(cudaGetLastError());
      dev::reduce_kernel<<<grid, dev::THREADS, dev::SMEM_BYTES, gs>>>();
      step(cudaGetLastError());
      cudaError_t ec = cudaStreamEndCapture(gs, &g);
      if (e == cudaSuccess) e = ec;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&gexec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        gexec = nullptr;
        throw Error(HVM64_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      }
      gkey = key;
    }
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    CU(cudaEventRecord(e0, gs));
    CU(cudaGraphLaunch(gexec, gs));
    CU(cudaEventRecord(e1, gs));
    CU(cudaEventSynchronize(e1));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h2d += sizeof(dev::NetState) * n + sizeof(dev::Ctrl);
    return ms;
  }

  uint64_t stat_donated = 0, stat_spilled = 0, stat_overflow = 0, heap_used = 0;
  uint64_t stat_steps = 0, stat_lanes = 0, stat_busy = 0, stat_idle = 0;
  uint64_t stat_g_steps[8] = {0}, stat_g_cycles[8] = {0}, stat_prof[32] = {0};

  void stats(hvm64_stats* o) const {
    *o = hvm64_stats{};
    for (const auto& n : host_nets) {
      o->comm22 += n.rw[dev::EX_COMM22];
      o->dref_nodes += n.rw[dev::EX_DNODES];
      o->dref_links += n.rw[dev::EX_DLINKS];
    }
    o->heap_nodes_used = heap_used;
    o->donated = stat_donated;
    o->spilled = stat_spilled;
    o->overflowed = stat_overflow;
    o->h2d_bytes = h2d;
    o->d2h_bytes = d2h;
    o->steps = stat_steps;
    o->step_lanes = stat_lanes;
    o->busy_cycles = stat_busy;
    o->idle_cycles = stat_idle;
  }

  // Normal forms gathered on the device (gather_kernel): per net, its
  // (address, word) pairs; a count of ~0u sends that net to the heap image.
  bool pairs_valid = false;
  std::vector<unsigned> gcount;
  std::vector<uint64_t> goff;
  DevBuf<unsigned> d_gcount;
  DevBuf<dev::ull> d_goff, d_gpairs;
  DevBuf<unsigned> d_tcounts;  // gather_kernel's per-subtree counts

  // Gathers the normal forms of the last run's nets (device-side walk).
  void gather_all() {
    const unsigned n = unsigned(progs.size()), first = run_first, cnt = run_count;
    DeviceTurn turn(device, 600000);
    upload_params(params(), 0);
    d_gcount.alloc(n);
    // one warp per net (see gather_kernel)
    gcount.assign(n, ~0u);
    d_tcounts.alloc(size_t(std::max(cnt, 1u)) * dev::GTASKS);
    if (cnt) CU(cudaMemcpy(d_gcount.p, gcount.data(), size_t(n) * 4, cudaMemcpyHostToDevice));
    if (cnt) dev::gather_kernel<<<cnt, 32>>>(first, cnt, d_gcount.p, nullptr, nullptr, d_tcounts.p);
    CU(cudaGetLastError());
    CU(cudaMemcpy(gcount.data(), d_gcount.p, size_t(n) * 4, cudaMemcpyDeviceToHost));
    for (unsigned i = 0; i < n; i++)
      if (i < first || i >= first + cnt) gcount[i] = 0;  // not in this run: read back as an error
    goff.resize(n);
    uint64_t tot = 0;
    for (unsigned i = 0; i < n; i++) {
      goff[i] = tot;
      if (gcount[i] != ~0u) tot += gcount[i];
    }
    d_goff.alloc(n);
    CU(cudaMemcpy(d_goff.p, goff.data(), size_t(n) * 8, cudaMemcpyHostToDevice));
    d_gpairs.alloc(2 * tot);
    if (cnt) dev::gather_kernel<<<cnt, 32>>>(first, cnt, d_gcount.p, d_goff.p, d_gpairs.p, d_tcounts.p);
    CU(cudaGetLastError());
    std::lock_guard<std::mutex> staged(g_stage.mu);
    uint64_t* pairs = g_stage.reserve(16 * tot);
    if (tot) CU(cudaMemcpy(pairs, d_gpairs.p, 16 * tot, cudaMemcpyDeviceToHost));
    d2h += size_t(n) * 4 + 16 * tot;
    h2d += size_t(n) * 8;
    // Every gathered net's text at once, on the host's cores.
    std::vector<uint64_t> roots(cnt);
    for (unsigned i = 0; i < cnt; i++) roots[i] = host_nets[first + i].root;
    unsigned hw = std::thread::hardware_concurrency();
    gtext = readback_pairs_many(book, pairs, goff.data() + first, gcount.data() + first, roots.data(), cnt,
                                heap_bytes / 8, std::max(1u, std::min(hw ? hw : 1u, 16u)));
    pairs_valid = true;
  }
  std::vector<ReadbackOut> gtext;

  std::string readback(unsigned i) {
    if (!reduced) throw Error(HVM64_ERR_BAD_INPUT, "net not reduced yet");
    if (i < run_first || i >= run_first + run_count)
      throw Error(HVM64_ERR_BAD_INPUT, "net " + std::to_string(i) + " was not in the last run's range");
    if (host_nets[i].status) throw Error(host_nets[i].status, status_name(host_nets[i].status));
    if (!pairs_valid) gather_all();
    if (gcount[i] != ~0u) {
      const ReadbackOut& r = gtext[i - run_first];
      if (!r.ok) throw Error(HVM64_ERR_BAD_INPUT, r.error);
      return r.text;
    }
    if (!image_valid) {
      // Copy the used part of the heap (everything below the bump pointer).
      uint64_t used = 0;
      CU(cudaMemcpy(&used, &ctrl.p->bump, 8, cudaMemcpyDeviceToHost));
      used = std::min<uint64_t>(used, heap_bytes / 16);
      image.resize(used * 2);
      CU(cudaMemcpy(image.data(), heap.p, used * 16, cudaMemcpyDeviceToHost));
      d2h += used * 16 + 8;
      image_valid = true;
    }
    std::string out;
    with_big_stack([&] { out = hvm::readback(book, image.data(), image.size(), host_nets[i].root); });
    return out;
  }

  // Net i of the last run (a pre-reduce run) with the redexes inert Defs
  // captured: those with an eraser first, each group in capture order.
  std::string readback_captured(unsigned i) {
    uint64_t n = std::min<uint64_t>(host_ctrl.captured, capture.n / 2);
    std::vector<uint64_t> got(2 * n), pairs;
    if (n) CU(cudaMemcpy(got.data(), capture.p, 16 * n, cudaMemcpyDeviceToHost));
    d2h += 16 * n;
    pairs.reserve(got.size());
    for (int pass = 0; pass < 2; pass++)
      for (uint64_t k = 0; k < n; k++)
        if ((got[2 * k + 1] == PORT_ERA) == (pass == 0)) {
          pairs.push_back(got[2 * k]);
          pairs.push_back(got[2 * k + 1]);
        }
    if (!n) return readback(i);
    uint64_t used = 0;
    CU(cudaMemcpy(&used, &ctrl.p->bump, 8, cudaMemcpyDeviceToHost));
    used = std::min<uint64_t>(used, heap_bytes / 16);
    image.resize(used * 2);
    CU(cudaMemcpy(image.data(), heap.p, used * 16, cudaMemcpyDeviceToHost));
    d2h += used * 16 + 8;
    image_valid = true;
    std::string out;
    with_big_stack([&] {
      out = hvm::readback_net(book, image.data(), image.size(), host_nets[i].root, pairs.data(), pairs.size() / 2);
    });
    return out;
  }
};

namespace dev {
__global__ void set_deadline_kernel(Ctrl* c, ull timeout_ns) { c->deadline = globaltimer() + timeout_ns; }
}  // namespace dev

// ===========================================================================
// Pre-reduce (transform/src/pre_reduce.rs:38-74,136-164) on the device
// ===========================================================================
// One launch per Def, all on one reused heap (the reference's shared `area`):
// the Def is booted without the expansion agent and reduced by the
// persistent reducer.  The redexes inert Defs captured go back into the net
// after those the reduction left, ones with an eraser first (linker.rs:70-85
// puts them in the fast queue, which Host::readback lists first).  The host
// driver (hvm::pre_reduce) orders the Defs and replaces them.
PreReduceRun pre_reduce_one(Runner& r, uint32_t id, const hvm64_tuning& tuning, double& device_ms) {
  PreReduceRun out;
  r.progs.assign(1, id);
  r.uploaded_defs = 0;  // the instruction table changed since the last launch
  double ms = 0;
  r.run(HVM64_BATCH_PERSISTENT, &tuning, &ms);
  device_ms += ms;
  const dev::NetState& ns = r.host_nets[0];
  out.status = ns.status;
  out.pops = r.stat_lanes;
  out.rw[0] = ns.rw[dev::RW_ANNI];
  out.rw[1] = ns.rw[dev::RW_COMM];
  out.rw[2] = ns.rw[dev::RW_ERAS];
  out.rw[3] = ns.rw[dev::RW_DREF];
  out.rw[4] = ns.rw[dev::RW_OPER];
  if (ns.status) out.error = r.error_message(ns.status);
  else out.text = r.readback_captured(0);
  return out;
}

void Runner::set_deadline(cudaStream_t st, uint64_t timeout_ms) {
  dev::set_deadline_kernel<<<1, 1, 0, st>>>(ctrl.p, uint64_t(timeout_ms) * 1000000ull);
  CU(cudaGetLastError());
}


// ===========================================================================
// Serving: one persistent reducer that admits requests while it runs
// ===========================================================================
// The reducer kernel runs until the host stops it.  The host writes requests
// (Def to boot, slot) into a device ring and bumps the ring's tail with async
// copies on a second stream; an idle warp takes a request, boots it in its
// own stack and reduces it alongside everything else in flight.  When a net's
// last holder lets it go, that warp gathers its normal form into the slot's
// output and posts a completion record, both in mapped host memory, which the
// host polls.  Slots bound the nets in flight; the heap is shared and only
// grows (normal forms stay until the server is freed).
// A server's lanes publish their free lists after this many nodes: fewer
// nodes stay stranded per lane over a server's long life.
constexpr unsigned SERVE_OVF_FLUSH = 32;

struct Server {
  Book book;
  int device = 0, sms = 148;
  uint64_t heap_bytes = 0;
  unsigned nslots = 0, out_cap = 0, req_cap = 0;
  DevBuf<dev::ull> heap;
  DevBuf<dev::Ctrl> ctrl;
  DevBuf<dev::NetState> nets;
  DevBuf<dev::Slot> q;
  DevBuf<DevDef> d_defs;
  DevBuf<DevInstr> d_instrs;
  DevBuf<dev::ull> d_labbits;
  DevBuf<dev::ServeReq> req;
  DevBuf<dev::ull> spill, bigregs;
  dev::ServeDone* done = nullptr;  // mapped host memory
  dev::ull* out = nullptr;         // mapped host memory
  dev::ServeReq* req_stage = nullptr;  // pinned staging for the async copies
  uint64_t* tail_stage = nullptr;
  int* stop_stage = nullptr;
  cudaStream_t ks = nullptr, cs = nullptr;
  bool running = false;
  uint64_t tail = 0, next_ticket = 1;
  std::vector<uint64_t> slot_ticket;  // 0: free
  std::vector<uint64_t> slot_nodes;   // the node budget each slot's request holds
  std::vector<unsigned> free_slots;
  uint64_t budget_nodes = 0, reserved_nodes = 0;
  DeviceTurn turn;  // the device's launch parameters are this server's while it runs

  ~Server() { shutdown(); }

  void start(uint64_t bytes, unsigned slots, unsigned out_pairs, const hvm64_tuning& t) {
    CU(cudaGetDevice(&device));
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (slots == 0 || slots > (1u << 20)) throw Error(HVM64_ERR_BAD_INPUT, "slots must be in 1..2^20");
    if (out_pairs == 0) throw Error(HVM64_ERR_BAD_INPUT, "out_pairs must be > 0");
    if (bytes == 0) {
      size_t fr = 0, tot = 0;
      CU(cudaMemGetInfo(&fr, &tot));
      bytes = std::min<uint64_t>(uint64_t(fr) / 2, uint64_t(16) << 30);
    }
    heap_bytes = bytes & ~uint64_t(15);
    nslots = slots;
    out_cap = out_pairs;
    req_cap = 2 * slots + 16;
    unsigned qlog2 = t.queue_slots_log2 ? t.queue_slots_log2 : DEFAULT_QLOG2;
    if (qlog2 < 4 || qlog2 > 24) throw Error(HVM64_ERR_BAD_INPUT, "queue_slots_log2 out of range");
    size_t qn = size_t(1) << qlog2;
    heap.alloc(heap_bytes / 8);
    ctrl.alloc(1);
    nets.alloc(nslots);
    q.alloc(qn);
    req.alloc(req_cap);
    d_defs.alloc(book.defs.size());
    d_instrs.alloc(book.instrs.size());
    d_labbits.alloc(book.labbits.size());
    CU(cudaHostAlloc(reinterpret_cast<void**>(&done), sizeof(dev::ServeDone) * nslots, cudaHostAllocMapped));
    CU(cudaHostAlloc(reinterpret_cast<void**>(&out), sizeof(dev::ull) * 2 * size_t(out_cap) * nslots,
                     cudaHostAllocMapped));
    CU(cudaHostAlloc(reinterpret_cast<void**>(&req_stage), sizeof(dev::ServeReq) * req_cap, cudaHostAllocDefault));
    CU(cudaHostAlloc(reinterpret_cast<void**>(&tail_stage), sizeof(uint64_t) * (req_cap + 1), cudaHostAllocDefault));
    CU(cudaHostAlloc(reinterpret_cast<void**>(&stop_stage), 2 * sizeof(int), cudaHostAllocDefault));
    memset(done, 0, sizeof(dev::ServeDone) * nslots);
    *stop_stage = 0;
    dev::ServeDone* d_done = nullptr;
    dev::ull* d_out = nullptr;
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_done), done, 0));
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_out), out, 0));
    CU(cudaStreamCreateWithFlags(&ks, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    if (!book.defs.empty())
      CU(cudaMemcpyAsync(d_defs.p, book.defs.data(), book.defs.size() * sizeof(DevDef), cudaMemcpyHostToDevice, ks));
    if (!book.instrs.empty())
      CU(cudaMemcpyAsync(d_instrs.p, book.instrs.data(), book.instrs.size() * sizeof(DevInstr),
                         cudaMemcpyHostToDevice, ks));
    if (!book.labbits.empty())
      CU(cudaMemcpyAsync(d_labbits.p, book.labbits.data(), book.labbits.size() * 8, cudaMemcpyHostToDevice, ks));
    CU(cudaMemsetAsync(nets.p, 0, sizeof(dev::NetState) * nslots, ks));
    dev::Ctrl c{};
    c.bump = 1;
    c.heap_nodes = heap_bytes / 16;
    c.heap_bytes = heap_bytes;
    // small allocator chunks: a server's heap is shared by requests for its
    // whole life, so nodes stranded in part-used chunks count against it.
    // Free nodes are shared between warps once half the heap is used, as in a
    // batch run: sharing them from the start measured 3-5x longer tail
    // latencies (allocation from shared lists is a chain of dependent loads)
    // and, in some runs, a stalled reducer.
    c.chunk_nodes = t.chunk_nodes ? t.chunk_nodes : 32;
    c.reuse_mark = c.heap_nodes / 2;
    c.spin_limit = 1ull << 24;
    c.donate_min = t.donate_min ? t.donate_min : 64;
    c.max_warps = t.max_warps_per_net;
    c.q_mask = qn - 1;
    c.deadline = ~0ull;
    // a server runs until stopped, or until its lifetime (timeout_ms) ends
    c.timeout_ns = (t.timeout_ms ? t.timeout_ms : 600000ull) * 1000000ull;
    CU(cudaMemcpyAsync(ctrl.p, &c, sizeof c, cudaMemcpyHostToDevice, ks));
    dev::queue_init_kernel<<<unsigned((qn + 255) / 256), 256, 0, ks>>>(q.p, qn);
    CU(cudaGetLastError());
    dev::Params p{};
    p.heap = heap.p;
    p.heap_bytes = heap_bytes;
    p.ctrl = ctrl.p;
    p.nets = nets.p;
    p.nnets = nslots;
    p.q = q.p;
    p.defs = d_defs.p;
    p.instrs = d_instrs.p;
    p.labbits = d_labbits.p;
    p.ndefs = unsigned(book.defs.size());
    p.serve = 1;
    p.req = req.p;
    p.done = d_done;
    p.out = d_out;
    p.req_cap = req_cap;
    p.out_cap = out_cap;
    const unsigned grid = unsigned(sms * reducer_blocks_per_sm(t));
    const uint64_t warps = uint64_t(grid) * dev::WARPS;
    // Node budget for admission: the heap minus what the allocator can hold
    // back while nothing is live (each lane's part-used chunk and unpublished
    // free list, each warp's reuse pool).
    p.ovf_flush = SERVE_OVF_FLUSH;
    p.gen = gen_matches(book);
    const uint64_t reserve = warps * 32 * (c.chunk_nodes + SERVE_OVF_FLUSH) + warps * dev::POOL;
    if (heap_bytes / 16 <= 2 * reserve)
      throw Error(HVM64_ERR_BAD_INPUT, "heap_bytes too small for a server: its allocator may hold back " +
                                           std::to_string(reserve) + " nodes; give it at least " +
                                           std::to_string(2 * reserve * 16) + " bytes");
    budget_nodes = heap_bytes / 16 - reserve;
    reserved_nodes = 0;
    p.spill_cap = spill_cap_for(heap_bytes, warps);
    spill.alloc(2 * size_t(p.spill_cap) * warps);
    p.spill = spill.p;
    if (book.max_nregs() > LOCAL_REGS) {
      bigregs.alloc(size_t(warps) * 32 * MAX_REGS);
      p.bigregs = bigregs.p;
    }
    turn.take(device, t.timeout_ms ? t.timeout_ms : 120000, true);  // held until shutdown
    upload_params(p, ks);
    CU(cudaStreamSynchronize(ks));  // tables and parameters in place before the reducer starts
    dev::reduce_kernel<<<grid, dev::THREADS, dev::SMEM_BYTES, ks>>>();
    CU(cudaGetLastError());
    running = true;
    slot_ticket.assign(nslots, 0);
    slot_nodes.assign(nslots, 0);
    free_slots.clear();
    for (unsigned i = nslots; i-- > 0;) free_slots.push_back(i);
  }

  // Nonzero when the reducer stopped on an error (read without waiting).
  int device_error() {
    int e = 0;
    if (cudaStreamQuery(ks) == cudaSuccess) {
      dev::Ctrl h{};
      CU(cudaMemcpy(&h, ctrl.p, sizeof h, cudaMemcpyDeviceToHost));
      e = h.error;
    }
    return e;
  }

  // Admits a request that may hold up to `nodes` live heap nodes (0: an
  // even share of the budget, budget / slots) when a slot and that much of
  // the node budget are free.
  uint64_t submit(const std::string& name, uint64_t nodes) {
    if (!running) throw Error(HVM64_ERR_BAD_INPUT, "server is not running");
    auto it = book.ids.find(name);
    if (it == book.ids.end()) throw Error(HVM64_ERR_BAD_INPUT, "no definition named @" + name);
    if (free_slots.empty()) throw Error(HVM64_ERR_QUEUE, "no free slot: poll and collect results first");
    if (nodes == 0) nodes = std::max<uint64_t>(1, budget_nodes / nslots);
    if (nodes > budget_nodes)
      throw Error(HVM64_ERR_BAD_INPUT, "request needs " + std::to_string(nodes) + " nodes; the server's budget is " +
                                           std::to_string(budget_nodes));
    if (reserved_nodes + nodes > budget_nodes)
      throw Error(HVM64_ERR_QUEUE, "not enough free node budget: poll and collect results first");
    unsigned slot = free_slots.back();
    free_slots.pop_back();
    uint64_t ticket = next_ticket++;
    slot_ticket[slot] = ticket;
    slot_nodes[slot] = nodes;
    reserved_nodes += nodes;
    unsigned k = unsigned(tail % req_cap);
    req_stage[k] = dev::ServeReq{ticket, slot, it->second};
    CU(cudaMemcpyAsync(req.p + k, req_stage + k, sizeof(dev::ServeReq), cudaMemcpyHostToDevice, cs));
    tail_stage[k] = ++tail;
    CU(cudaMemcpyAsync(&ctrl.p->req_tail, tail_stage + k, 8, cudaMemcpyHostToDevice, cs));
    CU(cudaStreamSynchronize(cs));
    return ticket;
  }

  // Nodes ever taken from the bump pointer (the heap's high-water mark),
  // read while the reducer runs.
  uint64_t heap_high() {
    if (!running) return 0;
    CU(cudaMemcpyAsync(tail_stage + req_cap, &ctrl.p->bump, 8, cudaMemcpyDeviceToHost, cs));
    CU(cudaStreamSynchronize(cs));
    return tail_stage[req_cap];
  }

  size_t poll(uint64_t* tickets, size_t cap) {
    size_t n = 0;
    for (unsigned s = 0; s < nslots && n < cap; s++) {
      uint64_t t = slot_ticket[s];
      if (t && reinterpret_cast<volatile dev::ServeDone*>(done + s)->ticket == t) tickets[n++] = t;
    }
    return n;
  }

  int result(uint64_t ticket, hvm64_rewrites* rw, double* latency_us, std::string& text) {
    unsigned s = 0;
    while (s < nslots && slot_ticket[s] != ticket) s++;
    if (s == nslots) throw Error(HVM64_ERR_BAD_INPUT, "unknown or collected ticket");
    volatile dev::ServeDone* d = done + s;
    if (d->ticket != ticket) throw Error(HVM64_ERR_BAD_INPUT, "request not finished yet");
    std::atomic_thread_fence(std::memory_order_acquire);
    int status = d->status;
    if (rw) *rw = hvm64_rewrites{d->rw[0], d->rw[1], d->rw[2], d->rw[3], d->rw[4]};
    if (latency_us) *latency_us = double(d->t_done - d->t_admit) / 1000.0;
    if (status == 0) {
      std::vector<uint64_t> pairs(2 * size_t(d->pairs));
      memcpy(pairs.data(), out + 2 * size_t(out_cap) * s, pairs.size() * 8);
      uint64_t root = d->root;
      with_big_stack([&] { text = readback_pairs(book, pairs.data(), d->pairs, heap_bytes / 8, root); });
    }
    slot_ticket[s] = 0;
    reserved_nodes -= slot_nodes[s];
    slot_nodes[s] = 0;
    free_slots.push_back(s);
    return status;
  }

  // Stops the reducer at once: `stop` ends idle warps, and the run's error
  // word (which every warp polls between steps) ends warps still reducing
  // requests, whose results are abandoned.
  void shutdown() {
    if (running) {
      stop_stage[0] = 1;
      stop_stage[1] = HVM64_ERR_TIMEOUT;
      cudaMemcpyAsync(&ctrl.p->stop, stop_stage, sizeof(int), cudaMemcpyHostToDevice, cs);
      cudaMemcpyAsync(&ctrl.p->error, stop_stage + 1, sizeof(int), cudaMemcpyHostToDevice, cs);
      cudaStreamSynchronize(cs);
      cudaStreamSynchronize(ks);
      running = false;
    }
    turn.release();
    if (ks) cudaStreamDestroy(ks);
    if (cs) cudaStreamDestroy(cs);
    ks = cs = nullptr;
    if (done) cudaFreeHost(done);
    if (out) cudaFreeHost(out);
    if (req_stage) cudaFreeHost(req_stage);
    if (tail_stage) cudaFreeHost(tail_stage);
    if (stop_stage) cudaFreeHost(stop_stage);
    done = nullptr;
    out = nullptr;
    req_stage = nullptr;
    tail_stage = nullptr;
    stop_stage = nullptr;
  }
};
}  // namespace hvm

// ===========================================================================
// C ABI (include/hvm64.h)
// ===========================================================================
using hvm::Error;

struct hvm64_book {
  hvm::Book book;
};
struct hvm64_net {
  hvm::Runner r;
  bool bound = false;
};
struct hvm64_batch {
  hvm::Runner r;
};

template <class F> static int guarded(F f) {
  try {
    f();
    return HVM64_OK;
  } catch (Error& e) {
    return hvm::set_error(e.code, e.msg);
  } catch (std::bad_alloc&) {
    return hvm::set_error(HVM64_ERR_OOM, "host out of memory");
  } catch (std::exception& e) {
    return hvm::set_error(HVM64_ERR_BAD_INPUT, e.what());
  }
}

static int copy_out(const std::string& s, char* buf, size_t cap, size_t* len) {
  if (len) *len = s.size();
  if (buf && cap) {
    size_t n = std::min(cap - 1, s.size());
    memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return HVM64_OK;
}

extern "C" {

const char* hvm64_last_error(void) { return hvm::g_error.c_str(); }
const char* hvm64_version(void) { return "hvm64-b200 0.1 (sm_100a)"; }

int hvm64_book_load(const char* text, size_t len, hvm64_book** out) {
  if (!text || !out) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    auto b = std::make_unique<hvm64_book>();
    std::string src(text, len);
    hvm::with_big_stack([&] { b->book.load(hvm::parse_book(src)); });
    *out = b.release();
  });
}
uint32_t hvm64_book_def_count(const hvm64_book* b) { return b ? b->book.def_count() : 0; }
const char* hvm64_book_def_name(const hvm64_book* b, uint32_t i) {
  return (b && i < b->book.names.size()) ? b->book.names[i].c_str() : nullptr;
}
void hvm64_book_free(hvm64_book* b) { delete b; }

int hvm64_net_create(const hvm64_book* book, uint64_t heap_bytes, hvm64_net** out) {
  if (!book || !out) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    auto n = std::make_unique<hvm64_net>();
    n->r.book = book->book;
    n->r.setup(heap_bytes);
    *out = n.release();
  });
}
int hvm64_net_boot(hvm64_net* net, const char* name) {
  if (!net || !name) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    auto it = net->r.book.ids.find(name);
    if (it == net->r.book.ids.end()) throw Error(HVM64_ERR_BAD_INPUT, std::string("no definition named @") + name);
    net->r.progs.assign(1, it->second);
    net->bound = true;
    net->r.reduced = false;
  });
}
int hvm64_net_encode(hvm64_net* net, const char* text, size_t len) {
  if (!net || !text) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    std::string src(text, len);
    uint32_t prog = 0;
    hvm::with_big_stack([&] {
      auto arena = std::make_shared<hvm::Arena>();
      hvm::AstNet n = hvm::parse_net(src, *arena);
      prog = net->r.book.add_expr(n);
      net->r.book.keep.push_back(arena);
    });
    net->r.progs.assign(1, prog);
    net->bound = true;
    net->r.reduced = false;
  });
}
int hvm64_net_normal(hvm64_net* net, const hvm64_tuning* t, hvm64_rewrites* out, double* device_ms) {
  if (!net) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  if (!net->bound) return hvm::set_error(HVM64_ERR_BAD_INPUT, "net has no root (boot or encode it first)");
  int rc = guarded([&] { net->r.run(HVM64_BATCH_PERSISTENT, t, device_ms); });
  if (rc) return rc;
  const auto& s = net->r.host_nets[0];
  if (out) *out = hvm64_rewrites{s.rw[0], s.rw[1], s.rw[2], s.rw[3], s.rw[4]};
  if (s.status) return hvm::set_error(s.status, net->r.error_message(s.status));
  return HVM64_OK;
}
int hvm64_net_readback(hvm64_net* net, char* buf, size_t cap, size_t* len) {
  if (!net) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  std::string s;
  int rc = guarded([&] { s = net->r.readback(0); });
  if (rc) return rc;
  return copy_out(s, buf, cap, len);
}
void hvm64_net_free(hvm64_net* net) { delete net; }

int hvm64_batch_create(const hvm64_book* book, uint32_t n, const char* const* entries, uint64_t heap_bytes,
                       hvm64_batch** out) {
  if (!book || !out || (n && !entries)) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    auto b = std::make_unique<hvm64_batch>();
    b->r.book = book->book;
    b->r.setup(heap_bytes);
    b->r.progs.resize(n);
    hvm::with_big_stack([&] {
      for (uint32_t i = 0; i < n; i++) {
        const char* e = entries[i];
        if (!e) throw Error(HVM64_ERR_BAD_INPUT, "null entry");
        if (e[0] == '=') {
          auto arena = std::make_shared<hvm::Arena>();
          b->r.progs[i] = b->r.book.add_expr(hvm::parse_net(e + 1, *arena));
          b->r.book.keep.push_back(arena);
        } else {
          auto it = b->r.book.ids.find(e);
          if (it == b->r.book.ids.end()) throw Error(HVM64_ERR_BAD_INPUT, std::string("no definition named @") + e);
          b->r.progs[i] = it->second;
        }
      }
    });
    *out = b.release();
  });
}
int hvm64_batch_normal_range(hvm64_batch* b, int mode, const hvm64_tuning* t, uint32_t first, uint32_t count,
                             hvm64_rewrites* per_net, int* status, double* device_ms) {
  if (!b) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  if (mode != HVM64_BATCH_PERSISTENT && mode != HVM64_BATCH_PLAIN)
    return hvm::set_error(HVM64_ERR_BAD_INPUT, "unknown batch mode");
  if (first > b->r.progs.size() || count > b->r.progs.size() - first)
    return hvm::set_error(HVM64_ERR_BAD_INPUT, "net range outside the batch");
  int rc = guarded([&] { b->r.run(mode, t, device_ms, first, count); });
  if (rc) return rc;
  int worst = 0;
  for (uint32_t k = 0; k < count; k++) {
    const auto& s = b->r.host_nets[first + k];
    if (per_net) per_net[k] = hvm64_rewrites{s.rw[0], s.rw[1], s.rw[2], s.rw[3], s.rw[4]};
    if (status) status[k] = s.status;
    if (s.status && !worst) worst = s.status;
  }
  if (worst) return hvm::set_error(worst, b->r.error_message(worst));
  return HVM64_OK;
}
int hvm64_batch_normal(hvm64_batch* b, int mode, const hvm64_tuning* t, hvm64_rewrites* per_net, int* status,
                       double* device_ms) {
  if (!b) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return hvm64_batch_normal_range(b, mode, t, 0, uint32_t(b->r.progs.size()), per_net, status, device_ms);
}
int hvm64_batch_readback(hvm64_batch* b, uint32_t i, char* buf, size_t cap, size_t* len) {
  if (!b || i >= b->r.progs.size()) return hvm::set_error(HVM64_ERR_BAD_INPUT, "bad batch index");
  std::string s;
  int rc = guarded([&] { s = b->r.readback(i); });
  if (rc) return rc;
  return copy_out(s, buf, cap, len);
}
void hvm64_batch_free(hvm64_batch* b) { delete b; }

int hvm64_batch_stats(const hvm64_batch* b, hvm64_stats* out) {
  if (!b || !out) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  b->r.stats(out);
  return HVM64_OK;
}
// Diagnostic (not in the public header): steps and cycles of the last run
// by the number of distinct rule classes among the lanes of a step.
int hvm64_internal_class_steps(const hvm64_batch* b, uint64_t* steps8, uint64_t* prof32) {
  if (!b) return HVM64_ERR_BAD_INPUT;
  for (int k = 0; k < 8; k++) steps8[k] = b->r.stat_g_steps[k];
  for (int k = 0; k < 32; k++) prof32[k] = b->r.stat_prof[k];
  return HVM64_OK;
}

int hvm64_net_stats(const hvm64_net* n, hvm64_stats* out) {
  if (!n || !out) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  n->r.stats(out);
  return HVM64_OK;
}

int hvm64_book_compile_source(const hvm64_book* book, char* buf, size_t cap, size_t* out_len) {
  if (!book) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] { copy_out(hvm::compile_defs_cuda(book->book), buf, cap, out_len); });
}
int hvm64_book_is_compiled(const hvm64_book* book) { return book ? int(hvm::gen_matches(book->book)) : 0; }

int hvm64_book_format(const char* text, size_t len, char* buf, size_t cap, size_t* out_len) {
  if (!text) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    std::string src(text, len), out;
    hvm::with_big_stack([&] { out = hvm::print_book(hvm::parse_book(src)); });
    copy_out(out, buf, cap, out_len);
  });
}

int hvm64_pre_reduce(const char* text, size_t len, const char* skip, uint64_t max_rwts, uint64_t heap_bytes,
                     const hvm64_tuning* tuning, hvm64_rewrites* out, char* buf, size_t cap, size_t* out_len,
                     char* not_normal, size_t nn_cap, size_t* nn_len) {
  if (!text) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    hvm::AstBook ast;
    hvm::Runner r;
    std::string src(text, len);
    hvm::with_big_stack([&] {
      ast = hvm::parse_book(src);
      r.book.load(ast, true);
    });
    // names separated by spaces or newlines (src/args.rs:51: value_delimiter ' ')
    std::set<std::string> sk;
    std::string names = skip ? skip : "";
    size_t s0 = 0;
    while (s0 <= names.size()) {
      size_t e = names.find_first_of(" \n", s0);
      if (e == std::string::npos) e = names.size();
      if (e > s0) sk.insert(names.substr(s0, e - s0));
      s0 = e + 1;
    }
    hvm64_tuning t{};
    if (tuning) t = *tuning;
    r.setup(heap_bytes);
    r.no_expand = true;
    if (max_rwts != ~uint64_t(0)) {
      // A bound on device work only (what counts is the pops, checked after
      // the run): a popped redex makes at most one plus a Def's instruction
      // count of interactions.
      uint64_t per = 1;
      for (const hvm::DevDef& d : r.book.defs) per = std::max<uint64_t>(per, uint64_t(d.ins_len) + 1);
      r.rw_limit = max_rwts > ~uint64_t(0) / per ? 0 : std::max<uint64_t>(max_rwts * per, 1);
    }
    r.capture.alloc(2 * (size_t(1) << 16));
    double ms = 0;
    hvm::PreReduceOut res;
    hvm::with_big_stack([&] {
      res = hvm::pre_reduce(ast, r.book, sk, max_rwts,
                            [&](uint32_t id) { return hvm::pre_reduce_one(r, id, t, ms); });
    });
    if (out) *out = hvm64_rewrites{res.rw[0], res.rw[1], res.rw[2], res.rw[3], res.rw[4]};
    copy_out(res.text, buf, cap, out_len);
    std::string nn;
    for (const std::string& n : res.not_normal) nn += n + "\n";
    copy_out(nn, not_normal, nn_cap, nn_len);
  });
}

}  // extern "C"

// ===========================================================================
// Normalisation without device allocation (hvm64_net_normal_noalloc)
// ===========================================================================
// Every device buffer of this entry point -- control block, net record, redex
// queue, Book tables and node heap -- is carved out of one file-scope array
// that the library holds on every GPU that loads it, until the process exits.
// In host code `g_noalloc_scratch` only names a host-side stand-in: its device
// address comes from cudaGetSymbolAddress, taken once per device with that
// device current, and every kernel is handed that address.
namespace hvm {
namespace noalloc {
constexpr uint64_t SCRATCH_BYTES = uint64_t(64) << 20;  // 64 MiB in all
constexpr unsigned QLOG2 = 13;                           // 8192 queue slots of 32 redexes
// The reducer grid is capped at MAX_WARPS warps (4 blocks of 2 warps on
// each of 148 SMs), each with an overflow stack of SPILL redexes, and lanes
// take allocator chunks of CHUNK_NODES nodes: every lane holding a part-used
// chunk ties up at most MAX_WARPS * 32 * CHUNK_NODES (303,104) nodes.
constexpr unsigned MAX_WARPS = 148 * 4 * 2;
constexpr unsigned SPILL = 256;
constexpr unsigned CHUNK_NODES = 8;
constexpr uint64_t round_up(uint64_t x) { return (x + 255) & ~uint64_t(255); }
constexpr uint64_t OFF_CTRL = 0;
constexpr uint64_t OFF_NET = round_up(OFF_CTRL + sizeof(dev::Ctrl));
constexpr uint64_t OFF_QUEUE = round_up(OFF_NET + sizeof(dev::NetState));
constexpr uint64_t OFF_BOOK = round_up(OFF_QUEUE + (uint64_t(1) << QLOG2) * sizeof(dev::Slot));
constexpr uint64_t BOOK_BYTES = uint64_t(4) << 20;      // Def headers + instructions + label sets
constexpr uint64_t OFF_SPILL = round_up(OFF_BOOK + BOOK_BYTES);
constexpr uint64_t OFF_HEAP = round_up(OFF_SPILL + uint64_t(MAX_WARPS) * SPILL * 16);
constexpr uint64_t HEAP_BYTES = (SCRATCH_BYTES - OFF_HEAP) & ~uint64_t(15);
static_assert(OFF_HEAP < SCRATCH_BYTES, "scratch layout");
}  // namespace noalloc
}  // namespace hvm

static __device__ __align__(256) unsigned char g_noalloc_scratch[hvm::noalloc::SCRATCH_BYTES];

namespace hvm {
namespace noalloc {
constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
unsigned char* g_dev_scratch[MAX_DEVICES] = {};

// The device address of the scratch array on the current device (set-up on
// the first call per device).
unsigned char* scratch_here(int device) {
  if (device < 0 || device >= MAX_DEVICES) throw Error(HVM64_ERR_CUDA, "device index out of range");
  std::lock_guard<std::mutex> g(g_setup_mu);
  if (!g_dev_scratch[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(HVM64_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_dev_scratch[device] = static_cast<unsigned char*>(p);
  }
  return g_dev_scratch[device];
}

uint64_t timeout_ms_of(const hvm64_tuning& t) { return t.timeout_ms ? t.timeout_ms : 120000; }

std::string run(const Book& book, const char* name, const hvm64_tuning* tp, hvm64_rewrites* out) {
  hvm64_tuning t{};
  if (tp) t = *tp;
  if (t.queue_slots_log2 && t.queue_slots_log2 != QLOG2)
    throw Error(HVM64_ERR_BAD_INPUT, "the no-allocation entry point has a fixed queue of 2^13 slots "
                                     "(queue_slots_log2 must be 0 or 13)");
  auto it = book.ids.find(name);
  if (it == book.ids.end()) throw Error(HVM64_ERR_BAD_INPUT, std::string("no definition named @") + name);
  uint64_t defs_b = book.defs.size() * sizeof(DevDef), ins_b = book.instrs.size() * sizeof(DevInstr);
  uint64_t lab_b = book.labbits.size() * 8;
  uint64_t off_ins = round_up(defs_b), off_lab = off_ins + round_up(ins_b);
  if (book.max_nregs() > LOCAL_REGS)
    throw Error(HVM64_ERR_BAD_INPUT, "a definition of this Book needs " + std::to_string(book.max_nregs()) +
                                         " registers; the no-allocation entry point runs Defs of up to " +
                                         std::to_string(LOCAL_REGS));
  if (off_lab + lab_b > BOOK_BYTES)
    throw Error(HVM64_ERR_BAD_INPUT, "Book too large for the no-allocation entry point: its device tables need " +
                                         std::to_string(off_lab + lab_b) + " bytes, the limit is " +
                                         std::to_string(BOOK_BYTES));
  int device = 0, sms = 0;
  CU(cudaGetDevice(&device));
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  unsigned char* base = scratch_here(device);
  DeviceTurn turn(device, timeout_ms_of(t));
  dev::Ctrl* ctrl = reinterpret_cast<dev::Ctrl*>(base + OFF_CTRL);
  dev::NetState* ns = reinterpret_cast<dev::NetState*>(base + OFF_NET);
  dev::Slot* q = reinterpret_cast<dev::Slot*>(base + OFF_QUEUE);
  unsigned char* bk = base + OFF_BOOK;
  dev::ull* heap = reinterpret_cast<dev::ull*>(base + OFF_HEAP);
  cudaStream_t st = 0;

  // The array keeps the previous call's contents: everything a run reads
  // before writing is set here (control block, net record, queue sequence
  // numbers, Book tables).  Heap nodes are LOCK-filled as they are handed out.
  if (defs_b) CU(cudaMemcpyAsync(bk, book.defs.data(), defs_b, cudaMemcpyHostToDevice, st));
  if (ins_b) CU(cudaMemcpyAsync(bk + off_ins, book.instrs.data(), ins_b, cudaMemcpyHostToDevice, st));
  if (lab_b) CU(cudaMemcpyAsync(bk + off_lab, book.labbits.data(), lab_b, cudaMemcpyHostToDevice, st));
  dev::NetState hn{};
  hn.prog = int(it->second);
  CU(cudaMemcpyAsync(ns, &hn, sizeof hn, cudaMemcpyHostToDevice, st));
  uint64_t timeout_ms = t.timeout_ms ? t.timeout_ms : 120000;
  dev::Ctrl c{};
  c.bump = 1;
  c.heap_nodes = HEAP_BYTES / 16;
  c.reuse_mark = c.heap_nodes / 2;
  c.heap_bytes = HEAP_BYTES;
  c.chunk_nodes = t.chunk_nodes ? std::min<uint32_t>(t.chunk_nodes, 64) : CHUNK_NODES;
  c.spin_limit = 1ull << 24;
  c.donate_min = t.donate_min ? t.donate_min : 64;
  c.max_warps = t.max_warps_per_net;
  c.q_mask = (1ull << QLOG2) - 1;
  c.deadline = ~0ull;
  c.timeout_ns = timeout_ms * 1000000ull;
  CU(cudaMemcpyAsync(ctrl, &c, sizeof c, cudaMemcpyHostToDevice, st));
  unsigned qn = 1u << QLOG2;
  dev::queue_init_kernel<<<(qn + 255) / 256, 256, 0, st>>>(q, qn);
  CU(cudaGetLastError());
  dev::set_deadline_kernel<<<1, 1, 0, st>>>(ctrl, c.timeout_ns);
  CU(cudaGetLastError());

  dev::Params p{};
  p.heap = heap;
  p.heap_bytes = HEAP_BYTES;
  p.ctrl = ctrl;
  p.nets = ns;
  p.nnets = 1;
  p.q = q;
  p.defs = reinterpret_cast<const DevDef*>(bk);
  p.instrs = reinterpret_cast<const DevInstr*>(bk + off_ins);
  p.labbits = reinterpret_cast<const dev::ull*>(bk + off_lab);
  p.ndefs = unsigned(book.defs.size());
  p.spill = reinterpret_cast<dev::ull*>(base + OFF_SPILL);
  p.spill_cap = SPILL;
  p.gen = gen_matches(book);
  p.ovf_flush = dev::OVF_FLUSH;
  hvm64_tuning tg = t;
  if (tg.blocks_per_sm == 0 || tg.blocks_per_sm > 4) tg.blocks_per_sm = 4;
  unsigned grid = std::min(unsigned(sms * reducer_blocks_per_sm(tg)), MAX_WARPS / unsigned(dev::WARPS));
  upload_params(p, st);
  dev::boot_kernel<<<1, dev::THREADS, dev::SMEM_BYTES, st>>>(0, 1);
  CU(cudaGetLastError());
  dev::reduce_kernel<<<grid, dev::THREADS, dev::SMEM_BYTES, st>>>();
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(st));

  dev::Ctrl hc{};
  CU(cudaMemcpy(&hc, ctrl, sizeof hc, cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(&hn, ns, sizeof hn, cudaMemcpyDeviceToHost));
  if (hc.error) {
    std::string msg = status_name(hc.error);
    if (hc.error == HVM64_ERR_OOM)
      msg += " (the no-allocation heap holds " + std::to_string(HEAP_BYTES / 16) + " nodes)";
    throw Error(hc.error, msg);
  }
  if (out) *out = hvm64_rewrites{hn.rw[0], hn.rw[1], hn.rw[2], hn.rw[3], hn.rw[4]};
  // Normal form: copy the used part of the heap to the host and read it back.
  uint64_t used = std::min<uint64_t>(hc.bump, HEAP_BYTES / 16);
  std::vector<uint64_t> image(used * 2);
  CU(cudaMemcpy(image.data(), heap, used * 16, cudaMemcpyDeviceToHost));
  std::string text;
  with_big_stack([&] { text = readback(book, image.data(), image.size(), hn.root); });
  return text;
}
}  // namespace noalloc
}  // namespace hvm

extern "C" int hvm64_net_normal_noalloc(const hvm64_book* book, const char* def_name, const hvm64_tuning* tuning,
                                        hvm64_rewrites* out, char* buf, size_t cap, size_t* len) {
  if (!book || !def_name) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  std::string s;
  int rc = guarded([&] { s = hvm::noalloc::run(book->book, def_name, tuning, out); });
  if (rc) return rc;
  return copy_out(s, buf, cap, len);
}

struct hvm64_server {
  hvm::Server s;
};

extern "C" {

int hvm64_server_create(const hvm64_book* book, uint64_t heap_bytes, uint32_t slots, uint32_t out_pairs,
                        const hvm64_tuning* tuning, hvm64_server** out) {
  if (!book || !out) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    auto sv = std::make_unique<hvm64_server>();
    sv->s.book = book->book;
    hvm64_tuning t{};
    if (tuning) t = *tuning;
    sv->s.start(heap_bytes, slots, out_pairs, t);
    *out = sv.release();
  });
}
int hvm64_server_submit(hvm64_server* sv, const char* def_name, uint64_t* ticket) {
  return hvm64_server_submit_nodes(sv, def_name, 0, ticket);
}
int hvm64_server_submit_nodes(hvm64_server* sv, const char* def_name, uint64_t nodes, uint64_t* ticket) {
  if (!sv || !def_name || !ticket) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] { *ticket = sv->s.submit(def_name, nodes); });
}
int hvm64_server_budget(hvm64_server* sv, uint64_t* budget, uint64_t* reserved, uint64_t* heap_high) {
  if (!sv) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  return guarded([&] {
    if (budget) *budget = sv->s.budget_nodes;
    if (reserved) *reserved = sv->s.reserved_nodes;
    if (heap_high) *heap_high = sv->s.heap_high();
  });
}
int hvm64_server_poll(hvm64_server* sv, uint64_t* tickets, size_t cap, size_t* n) {
  if (!sv || !n || (cap && !tickets)) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  *n = sv->s.poll(tickets, cap);
  if (*n == 0) {
    int e = 0;
    int rc = guarded([&] { e = sv->s.device_error(); });
    if (rc) return rc;
    if (e) return hvm::set_error(e, std::string("the serving reducer stopped: ") + hvm::status_name(e));
  }
  return HVM64_OK;
}
int hvm64_server_result(hvm64_server* sv, uint64_t ticket, hvm64_rewrites* rw, int* status, double* device_us,
                        char* buf, size_t cap, size_t* len) {
  if (!sv) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  std::string text;
  int st = 0;
  int rc = guarded([&] { st = sv->s.result(ticket, rw, device_us, text); });
  if (rc) return rc;
  if (status) *status = st;
  if (st) return hvm::set_error(st, hvm::status_name(st));
  return copy_out(text, buf, cap, len);
}
void hvm64_server_free(hvm64_server* sv) { delete sv; }

}  // extern "C"
