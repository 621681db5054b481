/*
 * hvm64.h -- C ABI of the B200 interaction-net reducer.
 *
 * Drop-in boundary for HVM-64 net normalisation.  The reference's boundary is
 * a Rust API (no C ABI); each entry point below names the reference call it
 * replaces.  Paths are relative to the HigherOrderCO/hvm-64 checkout.
 *
 * Conventions
 *  - Every call returns an int status: HVM64_OK (0) or an HVM64_ERR_* code,
 *    where the reference would panic or abort.  hvm64_last_error() gives the
 *    message of the last failure on the calling thread.
 *  - Handles are owned by the caller and released with the *_free calls.
 *    One handle is used by one host thread at a time (the reference's
 *    `&mut Net`).  Different handles may be used from different threads:
 *    calls that run kernels on one device take turns (a run holds the
 *    device's launch parameters until its kernels finish; a persistent
 *    launch fills every SM, so runs would not overlap anyway).  A call that
 *    waits longer than its tuning's timeout_ms for its turn returns
 *    HVM64_ERR_TIMEOUT.  A running server holds its device until it is freed:
 *    calls from its own thread on that device return HVM64_ERR_BAD_INPUT.
 *  - A net's heap, redex queue and Book tables live in device memory behind
 *    the handle; buffers in these signatures are host memory.
 *  - No torch or CUDA types appear here; the library picks the current CUDA
 *    device at hvm64_net_create / hvm64_batch_create.
 */
#ifndef HVM64_H
#define HVM64_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HVM64_OK 0
#define HVM64_ERR_OOM 1       /* heap exhausted: runtime/src/allocator.rs:104 expect("OOM") */
#define HVM64_ERR_BAD_PAIR 2  /* no rule for the pair: runtime/src/interact.rs:39-42 */
#define HVM64_ERR_DIV0 3      /* integer / or % by zero: num/src/num.rs:183-186,209-212 */
#define HVM64_ERR_TIMEOUT 4   /* a bounded device wait or the run deadline ran out */
#define HVM64_ERR_BAD_INPUT 5 /* parse error, unknown reference, bad argument */
#define HVM64_ERR_CUDA 6      /* CUDA runtime error (no device, launch failure) */
#define HVM64_ERR_QUEUE 7     /* the device redex queue overflowed */
#define HVM64_ERR_BAD_ADDR 8  /* a heap address outside the arena (internal fault, caught) */
#define HVM64_ERR_OUTPUT 9    /* a served net's normal form did not fit its output buffer */
#define HVM64_ERR_LIMIT 10    /* a run passed its interaction limit (pre-reduce's max_rwts) */

/* Per-rule interaction counters: runtime/src/runtime.rs:72-79 (Rewrites). */
typedef struct hvm64_rewrites {
  uint64_t anni, comm, eras, dref, oper;
} hvm64_rewrites;

/* Device launch knobs (0 = default).  hvm-64_b200/autotune.py picks blocks_per_sm,
 * chunk_nodes, donate_min, queue_slots_log2 and max_warps_per_net for a batch. */
typedef struct hvm64_tuning {
  uint32_t blocks_per_sm;    /* resident reducer blocks per SM (2 warps each; 0: as many as fit) */
  uint32_t chunk_nodes;      /* nodes a lane takes from the global bump at once */
  uint32_t donate_min;       /* warp-stack depth above which a warp shares work (the steal threshold) */
  uint32_t queue_slots_log2; /* global redex-queue capacity, in 32-redex slots (0: 2^20) */
  uint32_t max_warps_per_net; /* warps (plus queued slots) one net's work may spread over (0: no cap) */
  uint32_t flags;            /* HVM64_TUNE_* bits */
  uint64_t timeout_ms;       /* run deadline; a longer run fails with TIMEOUT */
} hvm64_tuning;

/* A persistent batch run is captured once as a CUDA graph (uploads, queue
 * init, boot and reducer launches) and replayed by later runs of the same
 * batch and tuning. */
#define HVM64_TUNE_GRAPH 1u

typedef struct hvm64_book hvm64_book;
typedef struct hvm64_net hvm64_net;
typedef struct hvm64_batch hvm64_batch;

const char* hvm64_last_error(void);
const char* hvm64_version(void);

/* Book::from_str + Host::new (ast/src/parser.rs:464-469, host/src/host.rs:25-73):
 * parse `.hvm` text, compute label sets, encode every Def. */
int hvm64_book_load(const char* text, size_t len, hvm64_book** out);
/* Number of Defs, and the name of Def `i` (host/src/host.rs:19-21). */
uint32_t hvm64_book_def_count(const hvm64_book* book);
const char* hvm64_book_def_name(const hvm64_book* book, uint32_t i);
void hvm64_book_free(hvm64_book* book);

/* Heap::new(bytes) + Net::new (runtime/src/allocator.rs:22, runtime/src/net.rs:19).
 * heap_bytes = 0 picks a default sized from free device memory. */
int hvm64_net_create(const hvm64_book* book, uint64_t heap_bytes, hvm64_net** out);
/* Net::boot(&host.defs[name]) (runtime/src/net.rs:30-32): the root is bound to
 * a call of the named Def (counts one DREF). */
int hvm64_net_boot(hvm64_net* net, const char* def_name);
/* Host::encode_net(net, root, &ast_net) (host/src/encode.rs:116-120): the root
 * is bound to an expression net written in the text format. */
int hvm64_net_encode(hvm64_net* net, const char* net_text, size_t len);
/* Net::normal / Net::parallel_normal (runtime/src/net.rs:55-60,
 * runtime/src/parallel.rs:35-160): expand and reduce to normal form on the
 * device.  `out` receives net.rwts; `device_ms` (nullable) the device time. */
int hvm64_net_normal(hvm64_net* net, const hvm64_tuning* tuning, hvm64_rewrites* out, double* device_ms);
/* Host::readback + Display (host/src/readback.rs:23-33, ast/src/ast.rs:234-263).
 * Writes at most cap bytes (NUL-terminated when it fits) and sets *len to the
 * full text length; call with cap = 0 to size the buffer. */
int hvm64_net_readback(hvm64_net* net, char* buf, size_t cap, size_t* len);
void hvm64_net_free(hvm64_net* net);

/* Batched normalisation: `n` independent nets, each booted from Def
 * entries[i] (Net::boot) or, when entries[i] starts with '=', encoded from the
 * expression text after it (Host::encode_net), all reduced together in one
 * persistent launch.  No reference counterpart: the reference normalises one
 * net per call (src/main.rs:176-193). */
int hvm64_batch_create(const hvm64_book* book, uint32_t n, const char* const* entries, uint64_t heap_bytes,
                       hvm64_batch** out);
#define HVM64_BATCH_PERSISTENT 0 /* all nets in one persistent launch */
#define HVM64_BATCH_PLAIN 1      /* one net per launch, one after the other */
/* Reduce every net.  per_net (n entries, nullable) receives each net's
 * counters, status (n entries, nullable) each net's status code. */
int hvm64_batch_normal(hvm64_batch* batch, int mode, const hvm64_tuning* tuning, hvm64_rewrites* per_net,
                       int* status, double* device_ms);
/* The same for nets [first, first + count) only, in one launch (persistent)
 * or one per net (plain): per_net and status have `count` entries.  Only
 * these nets can be read back afterwards.  No reference counterpart (a caller
 * of the reference reduces one net per call). */
int hvm64_batch_normal_range(hvm64_batch* batch, int mode, const hvm64_tuning* tuning, uint32_t first,
                             uint32_t count, hvm64_rewrites* per_net, int* status, double* device_ms);
int hvm64_batch_readback(hvm64_batch* batch, uint32_t i, char* buf, size_t cap, size_t* len);
void hvm64_batch_free(hvm64_batch* batch);

/* Counters of the last run, summed over the batch (no reference counterpart;
 * the reference reports only Rewrites).  comm22 is the share of COMM done by
 * the binary-binary rule (runtime/src/interact.rs:118-141); dref_nodes and
 * dref_links count the nodes and links made by Def instantiation; the byte
 * counts are the host<->device copies of the last normal + readbacks. */
typedef struct hvm64_stats {
  uint64_t comm22, dref_nodes, dref_links;
  uint64_t heap_nodes_used, donated, spilled, overflowed;
  uint64_t h2d_bytes, d2h_bytes;
  uint64_t steps, step_lanes;        /* warp steps taken; redexes they started */
  uint64_t busy_cycles, idle_cycles; /* summed over warps: stepping vs waiting for work */
} hvm64_stats;
int hvm64_batch_stats(const hvm64_batch* batch, hvm64_stats* out);
int hvm64_net_stats(const hvm64_net* net, hvm64_stats* out);

/* `hvm64 compile` (src/compile.rs:110-161): CUDA source with one straight-line
 * device function per Def of `book` and their dispatch.  A library built with
 * it (hvm-64_b200/build.py build_compiled, or `hvm64 compile`) runs those
 * functions instead of the instruction VM for that Book; any other Book runs
 * on the VM as usual.  Buffer convention as hvm64_net_readback. */
int hvm64_book_compile_source(const hvm64_book* book, char* buf, size_t cap, size_t* out_len);
/* 1 when this library holds compiled functions for `book`'s Defs. */
int hvm64_book_is_compiled(const hvm64_book* book);
/* ast::Book::from_str + Display (ast/src/parser.rs, ast/src/ast.rs:221-232):
 * `book_text` as the reference prints a parsed Book.  References need not
 * resolve.  Buffer convention as hvm64_net_readback. */
int hvm64_book_format(const char* book_text, size_t len, char* buf, size_t cap, size_t* out_len);
/* Book::pre_reduce (transform/src/pre_reduce.rs:27-74, as `hvm64 transform
 * -O pre-reduce` runs it from src/main.rs:100-126) on the current device.
 * `book_text` may reference Defs it lacks; those become inert Defs whose
 * calls are kept as redexes.  Every Def not named in `skip` (names separated
 * by spaces or newlines; nullable) is booted without the expansion agent and
 * reduced, Defs it references first, one launch per Def on one heap of
 * `heap_bytes` (0: a default); the result replaces the Def.  `out` receives
 * the summed Rewrites, `buf` the pre-reduced Book's text (ast/src/ast.rs:
 * 221-232 Display) and `not_normal` the names, one per line, of Defs whose
 * reduction took `max_rwts` pops or more (UINT64_MAX: no limit).  Those keep
 * their original net and add no Rewrites, where the reference keeps the net
 * as it stood after max_rwts pops.  Buffers follow hvm64_net_readback's
 * convention (cap = 0 sizes them). */
int hvm64_pre_reduce(const char* book_text, size_t len, const char* skip, uint64_t max_rwts, uint64_t heap_bytes,
                     const hvm64_tuning* tuning, hvm64_rewrites* out, char* buf, size_t cap, size_t* out_len,
                     char* not_normal, size_t nn_cap, size_t* nn_len);

/* Serving: one reducer that stays on the device and admits requests while it
 * runs (continuous batching).  No reference counterpart: the reference reduces
 * one net per call (src/main.rs:176-193, runtime/src/net.rs:55-60).
 *
 * hvm64_server_create uploads the Book, allocates the heap (heap_bytes, 0 =
 * default) and `slots` net slots with an output buffer of `out_pairs`
 * (address, word) pairs each, and launches the persistent reducer on a stream
 * of its own.  hvm64_server_submit boots Def `def_name` in a free slot and
 * returns a ticket (HVM64_ERR_QUEUE when every slot is taken).
 * hvm64_server_poll writes up to `cap` finished tickets; hvm64_server_result
 * gives a finished request's Rewrites, status, device latency (admission to
 * completion, microseconds) and normal form (hvm64_net_readback's text
 * convention) and frees its slot.  hvm64_server_free stops the reducer at
 * once; requests still running are abandoned.
 *
 * A server holds its device while it runs: calls of other threads on that
 * device wait for it to be freed (see the conventions above).  An error in any request
 * (OOM, DIV0, BAD_PAIR, ...) stops the whole server; poll then returns it.
 * A server lives at most tuning->timeout_ms (default 10 minutes), then stops
 * with HVM64_ERR_TIMEOUT. */
typedef struct hvm64_server hvm64_server;
int hvm64_server_create(const hvm64_book* book, uint64_t heap_bytes, uint32_t slots, uint32_t out_pairs,
                        const hvm64_tuning* tuning, hvm64_server** out);
int hvm64_server_submit(hvm64_server* server, const char* def_name, uint64_t* ticket);
/* Admission by node budget: the request may hold up to `nodes` live heap
 * nodes (0: budget / slots, what hvm64_server_submit reserves).  The budget is
 * the heap less what the allocator can hold back (per-lane chunks and free
 * lists, per-warp pools); a request is admitted when a slot and `nodes` of the
 * budget are free (else HVM64_ERR_QUEUE: collect results and retry), and its
 * reservation returns with its result.  Nodes a finished request's normal
 * form used are recycled for later requests; once half the heap is in use,
 * free nodes also move between the reducer's warps, so a long-running
 * server's heap stops growing at about half its size. */
int hvm64_server_submit_nodes(hvm64_server* server, const char* def_name, uint64_t nodes, uint64_t* ticket);
/* The node budget, the part admitted requests hold, and the heap's high-water
 * mark (nodes ever taken from fresh memory). */
int hvm64_server_budget(hvm64_server* server, uint64_t* budget, uint64_t* reserved, uint64_t* heap_high);
int hvm64_server_poll(hvm64_server* server, uint64_t* tickets, size_t cap, size_t* n);
int hvm64_server_result(hvm64_server* server, uint64_t ticket, hvm64_rewrites* out, int* status,
                        double* device_us, char* buf, size_t cap, size_t* len);
void hvm64_server_free(hvm64_server* server);

/* Boot Def `def_name`, reduce it to normal form and read it back, without
 * allocating any device memory.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: a process where a framework's
 * caching allocator or a memory pool has already reserved the device memory
 * (a fresh cudaMalloc would fail or fragment it), a host under a fixed,
 * audited device-memory budget, or a request loop that must not pay
 * cudaMalloc's latency and implicit device-wide synchronisation per request.
 * hvm64_net_create allocates a heap of its own; this call instead uses one
 * array compiled into the library (64 MiB on every GPU that loads it, held
 * until the process exits): a 4 MiB region for the Book's device tables, a
 * redex queue of 2^13 slots, overflow stacks for a reducer grid of at most
 * 1184 warps (4 blocks of 2 warps per SM on 148 SMs), and a heap of
 * 3,350,416 nodes.  Lanes take allocator chunks of 8 nodes, so part-used
 * chunks tie up at most 303,104 of them; nodes a warp frees are reused by
 * that warp.  Limits: a Book whose tables exceed 4 MiB is refused with
 * HVM64_ERR_BAD_INPUT; a net that outgrows the heap stops with HVM64_ERR_OOM;
 * a net whose waiting redexes outgrow the overflow stacks and the queue stops
 * with HVM64_ERR_QUEUE; tuning->queue_slots_log2 must be 0 or 13 and
 * tuning->blocks_per_sm above 4 counts as 4.  Host memory is used only to
 * render the normal-form text.
 *
 * The first call on a device looks up the array's device address (with that
 * device current); make that first call before any stream capture.  Every call
 * on a device shares the array and starts by resetting the parts a run reads
 * (control block, net record, queue, Book tables), so two calls that overlapped
 * on the GPU would race on it; calls on one device take turns like every other
 * run (each call holds the device until its kernels finish and its results
 * are copied back), so calls from different host threads are serialised.
 * Outputs: `out` (nullable) receives the Rewrites; the normal form is
 * written as hvm64_net_readback writes it (buf/cap/len). */
int hvm64_net_normal_noalloc(const hvm64_book* book, const char* def_name, const hvm64_tuning* tuning,
                             hvm64_rewrites* out, char* buf, size_t cap, size_t* len);

#ifdef __cplusplus
}
#endif
#endif /* HVM64_H */
