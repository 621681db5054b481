#!/usr/bin/env python
"""Benchmark: batched HVM-64 net normalisation on B200.

Workload (one step): a batch of independent nets (default 4096), each a
tree-sum or a bitonic sort chosen 50/50 by seed, depth drawn log-uniform in
[dmin, dmax], reduced to normal form in ONE persistent launch through the C
ABI (include/hvm64.h).  Metric: interactions (ANNI+COMM+ERAS+DREF+OPER, the
reference's Rewrites::total) per second, in G/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank reduces its own batch (seeded by rank): weak scaling.
`--impl reference` times the CPU evaluator (the oracle's restatement of the
reference's Net::parallel_normal, which cannot be built here) on a bounded
sample of the same workload.
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


def dref_bytes(nodes, links):
    return 32 + 40 * nodes + 32 * links


def peaks():
    try:
        p = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


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
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
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
    desc = f"{len(sample)} of the batch's nets ({total} interactions), Net::parallel_normal restated, {threads} threads"
    return total / secs / 1e9, desc, len(sample)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    t = 1
    while t * 2 <= threads:
        t *= 2
    entries = W.batch_entries(args.nets, args.dmin, args.dmax, seed=0)
    vals = []
    for step in range(args.warmup + args.steps):
        v, desc, n = cpu_baseline(entries, args.cpu_budget, t)
        if step >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": t, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def config(args):
    return {"workload": f"batched {args.nets} nets: tree-sum / bitonic-sort 50-50, depth log-uniform "
                        f"[{args.dmin}, {args.dmax}]",
            "nets": args.nets, "dmin": args.dmin, "dmax": args.dmax, "mode": "persistent, one launch per step",
            "l2": "flushed between steps (512 MiB write)", "parallelism": f"weak: {args.gpus} x 1 GPU"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nets", type=int, default=4096)
    ap.add_argument("--dmin", type=int, default=8)
    ap.add_argument("--dmax", type=int, default=12)
    ap.add_argument("--plain-nets", type=int, default=256, help="nets timed one-per-launch for the plain arm")
    ap.add_argument("--cpu-budget", type=float, default=4e8, help="interactions in the CPU sample")
    ap.add_argument("--heap-gb", type=float, default=0)
    ap.add_argument("--no-cpu", action="store_true")
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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import hvm64
    entries = W.batch_entries(args.nets, args.dmin, args.dmax, seed=rank)
    text = W.batch_book(entries)
    book = hvm64.Book.from_str(text)
    names = [f"main_{j}" for _, _, j in entries]
    heap = int(args.heap_gb * (1 << 30))
    batch = hvm64.Batch(book, names, heap)
    tune = hvm64.Tuning(timeout_ms=600000)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        batch.normal(hvm64.PERSISTENT, tune)
    # correctness of every net's normal form (outside the timed region)
    bad = 0
    for i, (kind, d, j) in enumerate(entries):
        if not W.check_result(kind, d, j, batch.readback(i)):
            bad += 1
    total_per_step = sum(batch.rwts[i].total() for i in range(batch.n))
    counts = {k: sum(getattr(batch.rwts[i], k) for i in range(batch.n)) for k in ("anni", "comm", "eras", "dref",
                                                                                    "oper")}

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = []
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
    torch.cuda.synchronize()
    elapsed = sum(step_ms) / 1000.0
    if dist:
        t = torch.tensor([elapsed], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        tot = torch.tensor([float(total_per_step)], device="cuda")
        dist.all_reduce(tot)
        total_all = tot.item()
    else:
        total_all = float(total_per_step)
    value = total_all * args.steps / elapsed / 1e9
    kernel_ms = statistics.mean(step_ms)

    # plain arm: the first `plain_nets` nets, one launch each
    plain_entries = entries[:args.plain_nets]
    pbatch = hvm64.Batch(book, names[:len(plain_entries)], heap)
    pbatch.normal(hvm64.PLAIN, tune)
    ptotal = sum(pbatch.rwts[i].total() for i in range(pbatch.n))
    p0 = time.perf_counter()
    pbatch.normal(hvm64.PLAIN, tune)
    plain_s = time.perf_counter() - p0
    plain_value = ptotal / plain_s / 1e9
    del pbatch

    # e2e: public API from host memory: batch creation (tables to HBM), reduce,
    # every net's normal form read back to host.
    e0 = time.perf_counter()
    ebatch = hvm64.Batch(book, names, heap)
    ebatch.normal(hvm64.PERSISTENT, tune)
    for i in range(ebatch.n):
        ebatch.readback(i)
    e2e_s = time.perf_counter() - e0
    stats = ebatch.stats()
    del ebatch

    hbm, peak_kind = peaks()
    comm22 = stats.get("comm22", counts["comm"])
    comm02 = counts["comm"] - comm22
    alg = (counts["anni"] * BYTES["anni"] + comm22 * BYTES["comm22"] + comm02 * BYTES["comm02"] +
           counts["oper"] * BYTES["oper"] + dref_bytes(stats.get("dref_nodes", 0), stats.get("dref_links", 0)) +
           counts["dref"] * 0)
    achieved = alg / (kernel_ms / 1000.0) / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kernel_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": config(args),
        "interactions_per_step": total_per_step, "counts_per_step": counts, "nets_bad": bad,
        "plain": {"value": plain_value, "unit": UNIT, "nets": len(plain_entries),
                  "note": "one net per launch, wall time incl. launch + sync"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "peak_kind": peak_kind},
        "e2e": {"value": total_per_step / e2e_s / 1e9, "unit": UNIT,
                "h2d_bytes_per_step": stats.get("h2d_bytes"), "d2h_bytes_per_step": stats.get("d2h_bytes")},
        "device_stats": stats,
        "gpu_launches": 4 * args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        t = 1
        while t * 2 <= threads:
            t *= 2
        v, desc, _ = cpu_baseline(entries, args.cpu_budget, t)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": t, "kind": "port", "sample": desc}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
