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
#include <chrono>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "device.cuh"

namespace hvm {
namespace dev {

// ---- global redex queue --------------------------------------------------------
// Single-thread reservation; data movement may be done by the whole warp.
__device__ bool q_reserve_push(const Params& P, Lane& L, ull& pos, bool must) {
  Ctrl* C = P.ctrl;
  ull mask = C->q_mask;
  pos = ld_gpu(&C->q_tail);
  unsigned it = 0;
  for (;;) {
    Slot* s = &P.q[pos & mask];
    long long dif = (long long)ld_gpu(&s->seq) - (long long)pos;
    if (dif == 0) {
      ull old = atomicCAS(&C->q_tail, pos, pos + 1);
      if (old == pos) return true;
      pos = old;
    } else if (dif < 0) {
      if (!must) return false;  // full
      pos = ld_gpu(&C->q_tail);
    } else {
      pos = ld_gpu(&C->q_tail);
    }
    if (!L.spin(it)) {
      if (must && !L.failed()) L.fail(HVM64_ERR_QUEUE, pos);
      return false;
    }
  }
}
__device__ void q_publish(const Params& P, ull pos) {
  __threadfence();
  st_gpu(&P.q[pos & P.ctrl->q_mask].seq, pos + 1);
}
__device__ bool q_reserve_pop(const Params& P, ull& pos) {
  Ctrl* C = P.ctrl;
  ull mask = C->q_mask;
  pos = ld_gpu(&C->q_head);
  for (int tries = 0; tries < 64; tries++) {
    Slot* s = &P.q[pos & mask];
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
__device__ void q_release(const Params& P, ull pos) {
  __threadfence();
  st_gpu(&P.q[pos & P.ctrl->q_mask].seq, pos + P.ctrl->q_mask + 1);
}

// A lane's buffer is full in the middle of an interaction: ship it as one slot.
__device__ void Lane::overflow() {
  atomicAdd(reinterpret_cast<ull*>(&P.nets[net].pending), 1ull);
  ull pos;
  if (!q_reserve_push(P, *this, pos, true)) {
    pn = 0;
    return;
  }
  Slot* s = &P.q[pos & P.ctrl->q_mask];
  st_gpu(reinterpret_cast<ull*>(&s->net), (ull(unsigned(pn)) << 32) | net);
  for (int k = 0; k < 2 * pn; k++) st_gpu(&s->r[k], pb[k]);
  q_publish(P, pos);
  atomicAdd(&P.ctrl->stat_overflow, 1ull);
  pn = 0;
}

__device__ __forceinline__ ull shfl(ull v, int src) { return __shfl_sync(0xffffffffu, v, src); }

// Warp-cooperative: move the `cnt` oldest redexes of the warp's stack into a
// queue slot.  Returns false if the queue had no room (only when !must).
__device__ bool donate(const Params& P, Lane& L, ull* S, unsigned& bot, unsigned cnt, int cur, bool must) {
  const unsigned lane = threadIdx.x & 31;
  ull pos = 0;
  int ok = 0;
  if (lane == 0) {
    atomicAdd(reinterpret_cast<ull*>(&P.nets[cur].pending), 1ull);
    ok = q_reserve_push(P, L, pos, must) ? 1 : 0;
    if (!ok) atomicAdd(reinterpret_cast<ull*>(&P.nets[cur].pending), ~0ull);
  }
  ok = __shfl_sync(0xffffffffu, ok, 0);
  if (!ok) return false;
  pos = shfl(pos, 0);
  Slot* s = &P.q[pos & P.ctrl->q_mask];
  if (lane < cnt) {
    unsigned k = (bot + lane) & (SCAP - 1);
    st_gpu(&s->r[2 * lane], S[2 * k]);
    st_gpu(&s->r[2 * lane + 1], S[2 * k + 1]);
  }
  if (lane == 0) st_gpu(reinterpret_cast<ull*>(&s->net), (ull(cnt) << 32) | unsigned(cur));
  __threadfence();
  __syncwarp();
  if (lane == 0) q_publish(P, pos);
  bot += cnt;
  return true;
}

// Flush a warp's per-lane counters into its net (warp reduction, one atomic
// per counter).
__device__ void flush_counters(const Params& P, Lane& L, int cur) {
  const unsigned lane = threadIdx.x & 31;
  for (int k = 0; k < NCOUNT; k++) {
    ull v = L.rw[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0 && v) atomicAdd(&P.nets[cur].rw[k], v);
    L.rw[k] = 0;
  }
}

__global__ void __launch_bounds__(THREADS) reduce_kernel(Params P) {
  __shared__ ull stk[WARPS][2 * SCAP];
  __shared__ unsigned stops[WARPS];
  const unsigned lane = threadIdx.x & 31;
  const unsigned budget0 = unsigned(P.ctrl->lane_budget);
  ull* S = stk[threadIdx.x >> 5];
  Ctrl* C = P.ctrl;
  Lane L(P);
  unsigned top = 0, bot = 0;  // warp-uniform ring indices
  int cur = -1;               // the net whose work this warp holds
  bool hungry = false;
  unsigned idle = 0, step = 0;

  for (;;) {
    int err = 0;
    if (lane == 0) err = ld_gpu32(&C->error);
    if (__shfl_sync(0xffffffffu, err, 0)) break;

    if (top == bot) {
      if (cur >= 0) {
        flush_counters(P, L, cur);
        if (lane == 0) {
          long long old = (long long)atomicAdd(reinterpret_cast<ull*>(&P.nets[cur].pending), ~0ull);
          if (old == 1) atomicAdd(reinterpret_cast<ull*>(&C->nets_left), ~0ull);
        }
        cur = -1;
      }
      ull pos = 0;
      int got = 0;
      if (lane == 0) got = q_reserve_pop(P, pos) ? 1 : 0;
      got = __shfl_sync(0xffffffffu, got, 0);
      if (!got) {
        int stop = 0;
        if (lane == 0) {
          if (!hungry) atomicAdd(reinterpret_cast<ull*>(&C->hungry), 1ull);
          if (ld_gpu64s(&C->nets_left) <= 0) stop = 1;
          else if ((++idle & 255) == 0 && globaltimer() > C->deadline) {
            L.fail(HVM64_ERR_TIMEOUT, 1);
            stop = 1;
          }
        }
        hungry = true;
        if (__shfl_sync(0xffffffffu, stop, 0)) break;
        __nanosleep(256);
        continue;
      }
      if (hungry && lane == 0) atomicAdd(reinterpret_cast<ull*>(&C->hungry), ~0ull);
      hungry = false;
      idle = 0;
      pos = shfl(pos, 0);
      __threadfence();
      Slot* s = &P.q[pos & C->q_mask];
      unsigned cnt = 0, net = 0;
      if (lane == 0) {
        ull meta = ld_gpu(reinterpret_cast<const ull*>(&s->net));
        net = unsigned(meta);
        cnt = unsigned(meta >> 32);
      }
      cnt = __shfl_sync(0xffffffffu, cnt, 0);
      net = __shfl_sync(0xffffffffu, net, 0);
      if (net >= P.nnets || cnt > unsigned(CHUNK)) {  // never expected; refuse to index with it
        if (lane == 0) L.fail(HVM64_ERR_BAD_ADDR, (ull(cnt) << 32) | net);
        break;
      }
      if (lane < cnt) {
        S[2 * lane] = ld_gpu(&s->r[2 * lane]);
        S[2 * lane + 1] = ld_gpu(&s->r[2 * lane + 1]);
      }
      __syncwarp();
      if (lane == 0) q_release(P, pos);
      bot = 0;
      top = cnt;
      cur = int(net);
      L.net = net;
      if (cnt == 0) continue;
    }

    // A run that never reaches normal form ends at the deadline.
    if ((++step & 1023) == 0) {
      int late = 0;
      if (lane == 0 && globaltimer() > C->deadline) {
        L.fail(HVM64_ERR_TIMEOUT, 2);
        late = 1;
      }
      if (__shfl_sync(0xffffffffu, late, 0)) break;
    }

    // Take up to 32 redexes off the top, one per lane.  A lane then keeps
    // reducing: first the newest redex its own interactions made, else one
    // more from the warp's stack, until its budget for this step is spent.
    // Nothing is pushed to the stack during the step, so lanes only pop.
    unsigned n = min(top - bot, 32u);
    ull a = 0, b = 0;
    if (lane < n) {
      unsigned k = (top - n + lane) & (SCAP - 1);
      a = S[2 * k];
      b = S[2 * k + 1];
    }
    if (lane == 0) stops[threadIdx.x >> 5] = top - n;
    __syncwarp();
    if (lane < n) {
      unsigned budget = budget0;
      for (;;) {
        L.interact(a, b);
        L.settle();
        if (--budget == 0) break;
        if (L.pn > 0) {
          L.pn--;
          a = L.pb[2 * L.pn];
          b = L.pb[2 * L.pn + 1];
          continue;
        }
        unsigned old = atomicSub(&stops[threadIdx.x >> 5], 1u);
        if (int(old - bot) <= 0) break;
        unsigned k = (old - 1) & (SCAP - 1);
        a = S[2 * k];
        b = S[2 * k + 1];
      }
    }
    __syncwarp();
    {
      unsigned st = stops[threadIdx.x >> 5];
      top = int(st - bot) > 0 ? st : bot;
    }
    __syncwarp();

    // Append every lane's new redexes.
    unsigned c = unsigned(L.pn), incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= unsigned(o)) incl += v;
    }
    unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned pre = incl - c;
    while ((top - bot) + total > unsigned(SCAP)) {
      unsigned cnt = min(top - bot, 32u);
      if (!donate(P, L, S, bot, cnt, cur, true)) break;
      if (lane == 0) atomicAdd(&C->stat_spilled, 1ull);
    }
    for (unsigned k = 0; k < c; k++) {
      unsigned slot = (top + pre + k) & (SCAP - 1);
      S[2 * slot] = L.pb[2 * k];
      S[2 * slot + 1] = L.pb[2 * k + 1];
    }
    L.pn = 0;
    top += total;
    __syncwarp();

    // Share the oldest work when other warps are starving.
    if (top - bot >= unsigned(C->donate_min) && ((step & 3) == 0)) {
      int give = 0;
      if (lane == 0) {
        long long h = ld_gpu64s(&C->hungry);
        long long queued = (long long)(ld_gpu(&C->q_tail) - ld_gpu(&C->q_head));
        give = h > 0 && queued < h;
      }
      if (__shfl_sync(0xffffffffu, give, 0)) {
        if (donate(P, L, S, bot, 32u, cur, false) && lane == 0) atomicAdd(&C->stat_donated, 1ull);
      }
    }
  }
  if (cur >= 0) flush_counters(P, L, cur);
}

// One thread per net: allocate the root, run the boot program against it
// (Net::boot / Host::encode_net), then wrap the root in an expansion agent
// (Net::expand, runtime/src/net.rs:65-69).  Redexes go to the global queue.
__global__ void boot_kernel(Params P, unsigned first, unsigned count) {
  unsigned i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= first + count) return;
  Lane L(P);
  L.net = i;
  NetState& ns = P.nets[i];
  ull root = L.alloc();
  unsigned prog = unsigned(ns.prog);
  if (prog < P.ndefs && !(P.defs[prog].flags & 1)) L.rw[RW_DREF]++;
  L.run_def(prog, pvar(root));
  L.settle();
  root = L.expand(root);
  L.settle();
  ns.root = root;
  if (L.pn) L.overflow();
  for (int k = 0; k < NCOUNT; k++)
    if (L.rw[k]) atomicAdd(&ns.rw[k], L.rw[k]);
  __threadfence();
  if (ld_gpu64s(&ns.pending) > 0) atomicAdd(reinterpret_cast<ull*>(&P.ctrl->nets_left), 1ull);
}

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
  }
  return "unknown error";
}

}  // namespace

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

  void upload_book() {
    if (uploaded_defs == book.defs.size() && d_defs.p) return;
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
    p.ctrl = ctrl.p;
    p.nets = nets.p;
    p.nnets = unsigned(progs.size());
    p.q = q.p;
    p.defs = d_defs.p;
    p.instrs = d_instrs.p;
    p.labbits = d_labbits.p;
    p.ndefs = unsigned(book.defs.size());
    return p;
  }

  // Reduce nets [first, first+count) (the rest stay untouched).
  void launch(unsigned first, unsigned count, const hvm64_tuning& t, cudaStream_t st) {
    dev::Params p = params();
    unsigned bt = 128;
    dev::boot_kernel<<<(count + bt - 1) / bt, bt, 0, st>>>(p, first, count);
    CU(cudaGetLastError());
    int bps = int(t.blocks_per_sm);
    if (bps <= 0) {
      int occ = 0;
      CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, dev::reduce_kernel, dev::THREADS, 0));
      bps = std::max(1, occ);
    }
    dev::reduce_kernel<<<unsigned(sms * bps), dev::THREADS, 0, st>>>(p);
    CU(cudaGetLastError());
  }

  void reset_ctrl(const hvm64_tuning& t, cudaStream_t st, unsigned qlog2, uint64_t bump) {
    dev::Ctrl c{};
    c.bump = bump;  // node 0 is reserved
    c.heap_nodes = heap_bytes / 16;
    c.heap_bytes = heap_bytes;
    c.chunk_nodes = t.chunk_nodes ? t.chunk_nodes : 256;
    c.spin_limit = 1ull << 24;
    c.donate_min = t.donate_min ? t.donate_min : 64;
    c.lane_budget = t.lane_budget ? t.lane_budget : 8;
    c.q_mask = (1ull << qlog2) - 1;
    // The deadline is set on the device clock right before launch.
    c.deadline = ~0ull;
    host_ctrl = c;
    CU(cudaMemcpyAsync(ctrl.p, &c, sizeof c, cudaMemcpyHostToDevice, st));
  }

  void run(int mode, const hvm64_tuning* tp, double* device_ms) {
    hvm64_tuning t{};
    if (tp) t = *tp;
    unsigned qlog2 = t.queue_slots_log2 ? t.queue_slots_log2 : 16;
    if (qlog2 < 4 || qlog2 > 24) throw Error(HVM64_ERR_BAD_INPUT, "queue_slots_log2 out of range");
    h2d = d2h = 0;
    heap.alloc(heap_bytes / 8);
    ctrl.alloc(1);
    nets.alloc(progs.size());
    q.alloc(size_t(1) << qlog2);
    upload_book();
    size_t qn = size_t(1) << qlog2;

    host_nets.assign(progs.size(), dev::NetState{});
    for (size_t i = 0; i < progs.size(); i++) host_nets[i].prog = int(progs[i]);
    CU(cudaMemcpy(nets.p, host_nets.data(), host_nets.size() * sizeof(dev::NetState), cudaMemcpyHostToDevice));
    h2d += host_nets.size() * sizeof(dev::NetState);

    stat_donated = stat_spilled = stat_overflow = 0;
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
      CU(cudaEventRecord(e0, st));
      launch(first, count, t, st);
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
      bump = std::min<uint64_t>(host_ctrl.bump, heap_bytes / 16);
      if (host_ctrl.error) {
        for (unsigned k = first; k < first + count; k++) host_nets[k].status = host_ctrl.error;
      }
    };
    if (mode == HVM64_BATCH_PLAIN) {
      for (unsigned i = 0; i < progs.size(); i++) one(i, 1);
    } else {
      one(0, unsigned(progs.size()));
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
    reduced = true;
  }

  void set_deadline(cudaStream_t st, uint64_t timeout_ms);
  uint64_t stat_donated = 0, stat_spilled = 0, stat_overflow = 0, heap_used = 0;

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
  }

  std::string readback(unsigned i) {
    if (!reduced) throw Error(HVM64_ERR_BAD_INPUT, "net not reduced yet");
    if (host_nets[i].status) throw Error(host_nets[i].status, status_name(host_nets[i].status));
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
};

namespace dev {
__global__ void set_deadline_kernel(Ctrl* c, ull timeout_ns) { c->deadline = globaltimer() + timeout_ns; }
}  // namespace dev

void Runner::set_deadline(cudaStream_t st, uint64_t timeout_ms) {
  dev::set_deadline_kernel<<<1, 1, 0, st>>>(ctrl.p, uint64_t(timeout_ms) * 1000000ull);
  CU(cudaGetLastError());
}

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
  if (s.status) return hvm::set_error(s.status, hvm::status_name(s.status));
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
int hvm64_batch_normal(hvm64_batch* b, int mode, const hvm64_tuning* t, hvm64_rewrites* per_net, int* status,
                       double* device_ms) {
  if (!b) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  if (mode != HVM64_BATCH_PERSISTENT && mode != HVM64_BATCH_PLAIN)
    return hvm::set_error(HVM64_ERR_BAD_INPUT, "unknown batch mode");
  int rc = guarded([&] { b->r.run(mode, t, device_ms); });
  if (rc) return rc;
  int worst = 0;
  for (size_t i = 0; i < b->r.host_nets.size(); i++) {
    const auto& s = b->r.host_nets[i];
    if (per_net) per_net[i] = hvm64_rewrites{s.rw[0], s.rw[1], s.rw[2], s.rw[3], s.rw[4]};
    if (status) status[i] = s.status;
    if (s.status && !worst) worst = s.status;
  }
  if (worst) return hvm::set_error(worst, hvm::status_name(worst));
  return HVM64_OK;
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
int hvm64_net_stats(const hvm64_net* n, hvm64_stats* out) {
  if (!n || !out) return hvm::set_error(HVM64_ERR_BAD_INPUT, "null argument");
  n->r.stats(out);
  return HVM64_OK;
}

}  // extern "C"
