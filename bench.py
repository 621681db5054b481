#!/usr/bin/env python
"""Benchmark: batched HVM-64 net normalisation on B200.

Workload (one step): a batch of independent nets (default 4096), each a
tree-sum or a bitonic sort chosen 50/50 by seed, depth drawn log-uniform in
[dmin, dmax], reduced to normal form in ONE persistent launch through the C
ABI (include/hvm64.h).  Metric: interactions (ANNI+COMM+ERAS+DREF+OPER, the
reference's Rewrites::total) per second, in G/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun the job reduces nets x N nets, split over the ranks by a
size-balanced partition (weak scaling: each GPU keeps about `nets` nets); no
collective on the data path (the nets are independent), only the step time
(max over ranks) and the interaction count (sum) are reduced.
`--impl reference` times the CPU evaluator (the oracle's restatement of the
reference's Net::parallel_normal; the Rust reference cannot be built without
a Rust toolchain) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hvm-64_b200"))

import workloads as W  # noqa: E402

METRIC = "GInteractions/s on 1 B200, batched-persistent vs per-net plain; p99 latency"
UNIT = "GInteractions/s"

# Algorithmic bytes per interaction (HBM model: one port word = 8 B, an
# exchange or CAS counts a read and a write).
BYTES = {"anni": 224, "comm22": 384, "comm02": 128, "eras": 0, "oper": 104}

# DRAM bytes (read + write) per interaction of reduce_kernel: ncu's
# dram__bytes_read.sum + dram__bytes_write.sum (68.06 + 151.11 GB) over the
# 1,414,382,623 interactions of one launch on a 4096-net batch of depth [8, 9]
# (the full workload is too long to capture); scaled by the interactions of a
# launch.
TRAFFIC_PER_INTERACTION = (68.06e9 + 151.11e9) / 1414382623


def dref_bytes(nodes, links, calls):
    return 32 * calls + 40 * nodes + 32 * links


def algorithmic_bytes(counts, stats):
    comm22 = stats["comm22"]
    comm02 = counts["comm"] - comm22
    return (counts["anni"] * BYTES["anni"] + comm22 * BYTES["comm22"] + comm02 * BYTES["comm02"] +
            counts["oper"] * BYTES["oper"] + dref_bytes(stats["dref_nodes"], stats["dref_links"], counts["dref"]))


# Global atomics per interaction of the same model (exchange or CAS); a Def
# call takes about one per link to its argument.
ATOMICS = {"anni": 8, "comm22": 8, "comm02": 4, "oper": 2}


def algorithmic_atomics(counts, stats):
    comm22 = stats["comm22"]
    comm02 = counts["comm"] - comm22
    return (counts["anni"] * ATOMICS["anni"] + comm22 * ATOMICS["comm22"] + comm02 * ATOMICS["comm02"] +
            counts["oper"] * ATOMICS["oper"] + stats["dref_links"])


def atomic_peak():
    """The measured L2 atomic rate (ops/s), if the microbenchmark's line was
    saved beside the measured peaks; else None."""
    try:
        p = json.load(open(os.path.join(ROOT, "profiles", "atomic_peak.json")))
        return min(float(p["atomic_exch_gops"]), float(p["atomic_cas_gops"])) * 1e9
    except Exception:
        return None


def peaks():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def pow2_threads():
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    t = 1
    while t * 2 <= n:
        t *= 2
    return t, n


class Clocks:
    """Samples nvidia-smi during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in self.rows if len(r) > 2 and num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if len(r) > 2 and num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def cpu_baseline(entries, budget, threads):
    """The oracle's parallel evaluator on the first nets of the batch whose
    estimated interactions fit `budget`; returns (interactions/s, sample)."""
    from oracle import oracle
    sample, est = [], 0.0
    for e in entries:
        c = W.est_interactions(e[0], e[1])
        if sample and est + c > budget:
            continue
        sample.append(e)
        est += c
    text = W.batch_book(sample)
    total, secs = 0, 0.0
    for kind, d, j in sample:
        _, rw, s = oracle.run_book(text, entry=f"main_{j}", mode=oracle.MODE_PARALLEL, threads=threads)
        total += sum(rw.values())
        secs += s
    desc = (f"{len(sample)} of the batch's nets ({total} interactions): the C++ restatement of "
            f"Net::parallel_normal, {threads} threads, timer around normal only")
    return total / secs / 1e9, desc


def _pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q * (len(xs) - 1)))))
    return xs[k]


def serve_leg(args, hvm64):
    """Serving at three offered loads: an open-loop Poisson stream of requests
    (tree-sum / bitonic sort / Church, sizes log-uniform 1e3..1e8
    interactions) served by the continuous-batching server, against the plain
    path that reduces one request per launch, first come first served."""
    import random
    reqs = W.serving_requests(args.serve_requests, seed=0)
    book = hvm64.Book.from_str(W.serving_book(reqs))
    names = [f"main_{j}" for _, _, j in reqs]
    # plain path: one Net, one boot + normal + readback per request
    net = hvm64.Net(book, 8 << 30)
    tune = hvm64.Tuning(timeout_ms=600000)
    net.boot(names[0])
    net.normal(tune)
    service, inter, bad = [], [], 0
    for (kind, param, j), name in zip(reqs, names):
        t0 = time.perf_counter()
        net.boot(name)
        rw = net.normal(tune)
        text = net.readback()
        service.append(time.perf_counter() - t0)
        inter.append(rw.total())
        bad += 0 if W.check_request(kind, param, j, text) else 1
    del net
    cap_rps = len(service) / sum(service)
    loads = []
    for frac in (1.0, 2.0, 4.0):
        rate = frac * cap_rps
        rng = random.Random(1234 + int(frac * 10))
        arr, t = [], 0.0
        for _ in names:
            t += rng.expovariate(rate)
            arr.append(t)
        # plain: one server, first come first served (measured service times)
        lat_plain, free_at = [], 0.0
        for a, sv_s in zip(arr, service):
            start = max(a, free_at)
            free_at = start + sv_s
            lat_plain.append(free_at - a)
        # continuous batching, in real time
        sv = hvm64.Server(book, slots=args.serve_slots, out_pairs=1 << 18, heap_bytes=16 << 30,
                          tuning=hvm64.Tuning(timeout_ms=600000))
        lat, owner, inflight, i = [], {}, 0, 0
        t_start = time.perf_counter()
        last = 0.0
        while len(lat) < len(names):
            now = time.perf_counter() - t_start
            if now > arr[-1] + args.serve_wait_s:
                sv.close()
                raise RuntimeError(f"serving: {len(names) - len(lat)} requests unfinished "
                                   f"{args.serve_wait_s} s after the last arrival")
            busy = False
            while i < len(names) and arr[i] <= now and inflight < args.serve_slots:
                owner[sv.submit(names[i])] = i
                inflight += 1
                i += 1
                busy = True
            for tk in sv.poll():
                k = owner.pop(tk)
                text, rw, us = sv.result(tk)
                last = time.perf_counter() - t_start
                lat.append(last - arr[k])
                inflight -= 1
                bad += 0 if W.check_request(*reqs[k], text) else 1
                busy = True
            if not busy:
                time.sleep(0.0002)
        sv.close()
        loads.append({
            "offered_rps": rate, "offered_frac_of_plain_capacity": frac,
            "served": {"p50_ms": 1e3 * _pct(lat, 0.5), "p99_ms": 1e3 * _pct(lat, 0.99),
                       "p999_ms": 1e3 * _pct(lat, 0.999), "sustained_gips": sum(inter) / last / 1e9},
            "plain": {"p50_ms": 1e3 * _pct(lat_plain, 0.5), "p99_ms": 1e3 * _pct(lat_plain, 0.99),
                      "p999_ms": 1e3 * _pct(lat_plain, 0.999),
                      "sustained_gips": sum(inter) / max(free_at, arr[-1]) / 1e9},
        })
    return {"requests": len(names), "bad": bad, "slots": args.serve_slots,
            "mix": "tree-sum / bitonic sort / Church 47/47/6, sizes log-uniform 1e3..1e8 interactions",
            "interactions": sum(inter), "plain_capacity_rps": cap_rps, "loads": loads,
            "note": "latency = completion seen by the host - arrival; plain = one boot+normal+readback per "
                    "request, first come first served, from measured service times; p999 of a few hundred "
                    "requests is close to the maximum"}


def config(args):
    return {"workload": f"batched {args.nets} nets: tree-sum / bitonic-sort 50-50 by seed, depth log-uniform "
                        f"[{args.dmin}, {args.dmax}], u24 keys",
            "nets": args.nets, "dmin": args.dmin, "dmax": args.dmax, "mode": "persistent, one launch per step",
            "l2": "flushed between steps (512 MiB write); heaps far above L2",
            "parallelism": f"weak: {args.gpus} x 1 GPU, size-balanced disjoint shares of nets x {args.gpus} nets"}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    t, n = pow2_threads()
    entries = W.batch_entries(args.nets, args.dmin, args.dmax, seed=0)
    vals = []
    for step in range(args.warmup + args.steps):
        v, desc = cpu_baseline(entries, args.cpu_budget / 4, t)
        if step >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": t, "kind": "port", "sample": desc,
                         "host_cpus": n},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nets", type=int, default=4096)
    ap.add_argument("--dmin", type=int, default=8)
    ap.add_argument("--dmax", type=int, default=14)
    ap.add_argument("--plain-nets", type=int, default=256, help="nets timed one-per-launch for the plain arm")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--cpu-budget", type=float, default=4e8, help="interactions in the CPU sample")
    ap.add_argument("--heap-gb", type=float, default=0)
    ap.add_argument("--device-only", action="store_true", help="skip the plain, e2e, serving and CPU legs")
    ap.add_argument("--serve-requests", type=int, default=96, help="requests per offered load (0: no serving leg)")
    ap.add_argument("--serve-slots", type=int, default=64)
    ap.add_argument("--serve-wait-s", type=float, default=120.0,
                    help="give up on a load this long after its last arrival")
    ap.add_argument("--autotune", type=int, default=1, help="pick the launch knobs on a sample first (0: defaults)")
    ap.add_argument("--tune-sample", type=int, default=1024)
    args = ap.parse_args()

    if args.impl == "reference":
        return run_reference(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local))

    import hvm64
    if world > 1:
        # one global batch of nets x world nets, split into size-balanced
        # shares (no communication while they reduce)
        import shard
        glob = W.batch_entries(args.nets * world, args.dmin, args.dmax, seed=0)
        entries = shard.rank_share(glob, lambda e: W.est_interactions(e[0], e[1]), rank, world)
    else:
        entries = W.batch_entries(args.nets, args.dmin, args.dmax, seed=0)
    text = W.batch_book(entries)
    book = hvm64.Book.from_str(text)
    names = [f"main_{j}" for _, _, j in entries]
    heap = int(args.heap_gb * (1 << 30))
    tune_report = None
    if args.autotune:
        import autotune
        tune, tune_report = autotune.autotune(book, names, heap, sample=args.tune_sample, timeout_ms=600000)
    else:
        tune = hvm64.Tuning(timeout_ms=600000)
    tune.flags |= hvm64.TUNE_GRAPH  # each step replays one captured CUDA graph
    batch = hvm64.Batch(book, names, heap)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        batch.normal(hvm64.PERSISTENT, tune)
    # every net's normal form, checked outside the timed region
    bad = sum(0 if W.check_result(kind, d, j, batch.readback(i)) else 1 for i, (kind, d, j) in enumerate(entries))
    total_per_step = sum(batch.rwts[i].total() for i in range(batch.n))
    counts = {k: sum(getattr(batch.rwts[i], k) for i in range(batch.n))
              for k in ("anni", "comm", "eras", "dref", "oper")}

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, kernel_ms = [], []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            batch.normal(hvm64.PERSISTENT, tune)
            e1.record()
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            kernel_ms.append(batch.device_ms)
    torch.cuda.synchronize()
    elapsed = sum(step_ms) / 1000.0
    stats = batch.stats()
    if dist:
        t = torch.tensor([elapsed], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        tot = torch.tensor([float(total_per_step)], device="cuda", dtype=torch.float64)
        dist.all_reduce(tot)
        total_all = float(tot.item())
    else:
        total_all = float(total_per_step)
    value = total_all * args.steps / elapsed / 1e9

    # roofline of reduce_kernel: algorithmic bytes of one launch over its
    # device time (CUDA events the library records on its launching stream)
    hbm, peak_kind = peaks()
    alg = algorithmic_bytes(counts, stats)
    atoms = algorithmic_atomics(counts, stats)
    arate = atomic_peak()
    kms = statistics.mean(kernel_ms)
    achieved = alg / (kms / 1000.0) / 1e9
    traffic = TRAFFIC_PER_INTERACTION * total_per_step if TRAFFIC_PER_INTERACTION else None
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed * 1000.0 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": config(args),
        "interactions_per_step": total_per_step, "counts_per_step": counts, "nets_bad": bad,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "peak_kind": f"{peak_kind} (copy bandwidth)",
                     "kernel": "reduce_kernel (+ boot_kernel) device time per launch", "kernel_ms": kms,
                     "algorithmic_bytes": alg, "algorithmic_atomics": atoms,
                     "atomic_rate_ops": arate,
                     "atomic_frac": (atoms / (kms / 1000.0)) / arate if arate else None},
        "gpu_launches": 4 * args.steps,
        "tuning": {"knobs": {k: getattr(tune, k) for k in ("blocks_per_sm", "chunk_nodes", "donate_min",
                                                            "queue_slots_log2")},
                   "cuda_graph": True, "autotune": tune_report},
        "clocks": clk.summary(),
        "device_stats": stats,
    }

    if not args.device_only:
        # plain arm: the batch's first `plain_nets` nets, one launch each
        plain_entries = entries[:args.plain_nets]
        if plain_entries:
            pbatch = hvm64.Batch(book, names[:len(plain_entries)], heap)
            ptune = hvm64.Tuning(timeout_ms=600000)
            pbatch.normal(hvm64.PLAIN, ptune)
            ptotal = sum(pbatch.rwts[i].total() for i in range(pbatch.n))
            torch.cuda.synchronize()
            p0 = time.perf_counter()
            pbatch.normal(hvm64.PLAIN, ptune)
            plain_s = time.perf_counter() - p0
            pdev = pbatch.device_ms
            del pbatch
            # the batched reducer on the same subset, for the like-for-like ratio
            sbatch = hvm64.Batch(book, names[:len(plain_entries)], heap)
            sbatch.normal(hvm64.PERSISTENT, tune)
            s0 = time.perf_counter()
            sbatch.normal(hvm64.PERSISTENT, tune)
            sub_s = time.perf_counter() - s0
            del sbatch
            out["plain"] = {"value": ptotal / plain_s / 1e9, "unit": UNIT, "nets": len(plain_entries),
                            "device_value": ptotal / (pdev / 1000.0) / 1e9,
                            "batched_same_nets": ptotal / sub_s / 1e9,
                            "note": "one net per launch (wall time incl. launch + sync) vs the batched "
                                    "reducer on the same nets, and the full batch's value"}

        # e2e through the public API from host memory: tables and net list to
        # the device, reduce, every net's normal form back to host text.
        e2e_s, h2d, d2h = 0.0, 0, 0
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            e0 = time.perf_counter()
            ebatch = hvm64.Batch(book, names, heap)
            ebatch.normal(hvm64.PERSISTENT, tune)
            for i in range(ebatch.n):
                ebatch.readback(i)
            e2e_s += time.perf_counter() - e0
            st = ebatch.stats()
            h2d, d2h = st["h2d_bytes"], st["d2h_bytes"]
            del ebatch
        if dist:
            t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        out["e2e"] = {"value": total_all * args.e2e_steps / e2e_s / 1e9, "unit": UNIT,
                      "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                      "note": "Batch create + normal + readback of every net, wall clock"}

        if rank == 0 and args.serve_requests > 0:
            del batch
            try:
                out["serving"] = serve_leg(args, hvm64)
            except Exception as e:  # the serving leg must not cost the benchmark line
                out["serving"] = {"error": f"{type(e).__name__}: {e}"}

        if rank == 0:
            t, n = pow2_threads()
            try:
                v, desc = cpu_baseline(entries, args.cpu_budget, t)
                out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": t, "kind": "port", "sample": desc,
                                       "host_cpus": n}
            except Exception as e:
                out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": t, "kind": "port",
                                       "error": f"{type(e).__name__}: {e}"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
