#!/usr/bin/env python
"""Benchmark: batched HVM-64 net normalisation on B200.

Workload: the batched configuration -- 4096 independent nets, each a tree-sum
or a bitonic sort chosen 50/50 by seed, depth drawn log-uniform in [8, 18]
(u24 keys from an in-net mixer), reduced to normal form through the C ABI
(include/hvm64.h).  Metric: interactions (ANNI+COMM+ERAS+DREF+OPER, the
reference's Rewrites::total) per second, in G/s.

Steps.  The batch is split into K size-balanced slices (longest-processing-
time on the predicted interaction count), K = --steps; step k reduces slice k
in ONE persistent launch (boot + reduce, replayed as a captured CUDA graph).
The K timed steps therefore reduce every net of the batch exactly once, and
`value` is the whole batch's interactions over the K steps' device time.
Warm-up steps reduce the first W slices first.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank takes a size-balanced share of a global batch of
nets x N nets (weak scaling); nothing crosses ranks while they reduce, only
the step time (max over ranks) and the interaction count (sum).
`--impl reference` times the CPU evaluator (the oracle's restatement of the
reference's Net::parallel_normal; the Rust reference cannot be built without
a Rust toolchain) on mass-weighted samples of the same batch.
"""
import argparse
import json
import os
import random
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hvm-64_b200"))

import workloads as W  # noqa: E402
import shard  # noqa: E402

METRIC = "GInteractions/s on 1 B200, batched-persistent vs per-net plain; p99 latency"
UNIT = "GInteractions/s"

# Algorithmic bytes per interaction (HBM model: one port word = 8 B, an
# exchange or CAS counts a read and a write).
BYTES = {"anni": 224, "comm22": 384, "comm02": 128, "eras": 0, "oper": 104}
# Global atomics per interaction of the same model (exchange or CAS); a Def
# call takes about one per link to its argument.
ATOMICS = {"anni": 8, "comm22": 8, "comm02": 4, "oper": 2}


def dref_bytes(nodes, links, calls):
    return 32 * calls + 40 * nodes + 32 * links


def algorithmic_bytes(counts, stats):
    comm22 = stats["comm22"]
    comm02 = counts["comm"] - comm22
    return (counts["anni"] * BYTES["anni"] + comm22 * BYTES["comm22"] + comm02 * BYTES["comm02"] +
            counts["oper"] * BYTES["oper"] + dref_bytes(stats["dref_nodes"], stats["dref_links"], counts["dref"]))


def algorithmic_atomics(counts, stats):
    comm22 = stats["comm22"]
    comm02 = counts["comm"] - comm22
    return (counts["anni"] * ATOMICS["anni"] + comm22 * ATOMICS["comm22"] + comm02 * ATOMICS["comm02"] +
            counts["oper"] * ATOMICS["oper"] + stats["dref_links"])


def _profile(name):
    try:
        return json.load(open(os.path.join(ROOT, "profiles", name)))
    except Exception:
        return None


def atomic_peak():
    """The measured L2 atomic rate (ops/s) of 64-bit exchange and CAS on random
    words (profiles/atomic_peak.json, hvm64_atomic_peak); else None."""
    p = _profile("atomic_peak.json")
    if not p:
        return None, None
    r = p.get("rate_for_roofline") or p
    return min(float(r["atomic_exch_gops"]), float(r["atomic_cas_gops"])) * 1e9, p.get("note")


def traffic_per_interaction():
    """DRAM bytes (read + write) per interaction of reduce_kernel from the
    current build's ncu capture summarised in profiles/ (None if absent)."""
    p = _profile("reduce_kernel_traffic.json")
    if not p:
        return None, None
    return float(p["dram_bytes_per_interaction"]), p.get("capture")


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


def est(e):
    return W.est_interactions(e[0], e[1])


def slices_of(entries, k):
    """The batch split into k size-balanced slices (lists of entries)."""
    parts = shard.lpt_partition([est(e) for e in entries], k)
    return [[entries[i] for i in p] for p in parts]


def mass_sample(entries, budget, seed, first_may_exceed=True):
    """Nets drawn with probability proportional to their predicted
    interactions (without replacement) until `budget` interactions: the
    sample's size distribution follows the batch's interaction mass, so big
    nets are represented as they weigh in the batch's time."""
    rng = random.Random(seed)
    pool = list(entries)
    out, tot = [], 0.0
    while pool and tot < budget:
        w = [est(e) for e in pool]
        e = rng.choices(pool, weights=w)[0]
        pool.remove(e)
        c = est(e)
        if out and tot + c > budget:
            continue
        if not out and c > budget and not first_may_exceed:
            continue
        out.append(e)
        tot += c
    return out


def cpu_run(sample, threads):
    """The oracle's parallel evaluator on each sampled net: (interactions,
    seconds inside normal, description)."""
    from oracle import oracle
    text = W.batch_book(sample)
    total, secs = 0, 0.0
    for kind, d, j in sample:
        _, rw, s = oracle.run_book(text, entry=f"main_{j}", mode=oracle.MODE_PARALLEL, threads=threads)
        total += sum(rw.values())
        secs += s
    depths = sorted(f"{k}{d}" for k, d, _ in sample)
    desc = (f"{len(sample)} nets drawn from the batch with probability proportional to their size "
            f"({', '.join(depths)}; {total} interactions): the C++ restatement of Net::parallel_normal, "
            f"{threads} threads, timer around normal only")
    return total, secs, desc


def cpu_baseline(entries, budget, threads, seed=0):
    total, secs, desc = cpu_run(mass_sample(entries, budget, seed), threads)
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
    interactions) served by the continuous-batching server (admission by slot
    and node budget), against the plain path -- one Net, one boot + normal +
    readback per request, first come first served -- run in real time on the
    same arrivals."""
    reqs = W.serving_requests(args.serve_requests, seed=0)
    book = hvm64.Book.from_str(W.serving_book(reqs))
    names = [f"main_{j}" for _, _, j in reqs]
    nodes = [W.est_request_nodes(k, p) for k, p, _ in reqs]
    net = hvm64.Net(book, 8 << 30)
    tune = hvm64.Tuning(timeout_ms=600000)
    net.boot(names[0])
    net.normal(tune)
    service, inter, bad = [], [], 0
    for (kind, param, j), name in zip(reqs, names):  # service times: the plain path's capacity
        t0 = time.perf_counter()
        net.boot(name)
        rw = net.normal(tune)
        text = net.readback()
        service.append(time.perf_counter() - t0)
        inter.append(rw.total())
        bad += 0 if W.check_request(kind, param, j, text) else 1
    cap_rps = len(service) / sum(service)
    loads = []
    for frac in (1.0, 2.0, 4.0):
        rate = frac * cap_rps
        rng = random.Random(1234 + int(frac * 10))
        arr, t = [], 0.0
        for _ in names:
            t += rng.expovariate(rate)
            arr.append(t)
        # plain, in real time: requests in arrival order, one launch each
        # (results are verified after the loop, so checking costs no latency)
        lat_plain, texts = [], []
        t_start = time.perf_counter()
        for k, name in enumerate(names):
            now = time.perf_counter() - t_start
            if now < arr[k]:
                time.sleep(arr[k] - now)
            net.boot(name)
            net.normal(tune)
            texts.append((k, net.readback()))
            lat_plain.append(time.perf_counter() - t_start - arr[k])
        plain_end = time.perf_counter() - t_start
        bad += sum(0 if W.check_request(*reqs[k], text) else 1 for k, text in texts)
        # continuous batching, in real time; the server's lifetime ends soon
        # after the last arrival's wait
        life_ms = int(1000 * (arr[-1] + args.serve_wait_s)) + 5000
        sv = hvm64.Server(book, slots=args.serve_slots, out_pairs=1 << 19, heap_bytes=16 << 30,
                          tuning=hvm64.Tuning(timeout_ms=life_ms))
        try:
            lat, owner, i, texts = [], {}, 0, []
            t_start = time.perf_counter()
            last = 0.0
            while len(lat) < len(names):
                now = time.perf_counter() - t_start
                if now > arr[-1] + args.serve_wait_s:
                    raise RuntimeError(f"serving: {len(names) - len(lat)} requests unfinished "
                                       f"{args.serve_wait_s} s after the last arrival")
                busy = False
                while i < len(names) and arr[i] <= now:
                    try:
                        owner[sv.submit(names[i], nodes=nodes[i])] = i
                    except hvm64.HvmError as e:  # no slot or node budget free: admit later
                        if e.code != hvm64.ERR_QUEUE:
                            raise
                        break
                    i += 1
                    busy = True
                for tk in sv.poll():
                    k = owner.pop(tk)
                    text, rw, us = sv.result(tk)
                    last = time.perf_counter() - t_start
                    lat.append(last - arr[k])
                    texts.append((k, text))
                    busy = True
                if not busy:
                    time.sleep(0.0002)
            heap = sv.budget()
        finally:  # a failed load still frees its server (and the device it holds)
            sv.close()
        bad += sum(0 if W.check_request(*reqs[k], text) else 1 for k, text in texts)
        loads.append({
            "offered_rps": rate, "offered_frac_of_plain_capacity": frac,
            "served": {"p50_ms": 1e3 * _pct(lat, 0.5), "p99_ms": 1e3 * _pct(lat, 0.99),
                       "p999_ms": 1e3 * _pct(lat, 0.999), "sustained_gips": sum(inter) / last / 1e9,
                       "heap_high_nodes": heap["heap_high"], "node_budget": heap["budget"]},
            "plain": {"p50_ms": 1e3 * _pct(lat_plain, 0.5), "p99_ms": 1e3 * _pct(lat_plain, 0.99),
                      "p999_ms": 1e3 * _pct(lat_plain, 0.999), "sustained_gips": sum(inter) / plain_end / 1e9},
        })
    del net
    return {"requests": len(names), "bad": bad, "slots": args.serve_slots,
            "mix": "tree-sum / bitonic sort / Church 47/47/6, sizes log-uniform 1e3..1e8 interactions",
            "interactions": sum(inter), "largest_request": max(inter), "plain_capacity_rps": cap_rps,
            "loads": loads,
            "note": "latency = completion seen by the host - arrival, both paths run in real time on the same "
                    "Poisson arrivals; plain = one Net, boot+normal+readback per request, first come first "
                    "served; served = admission by slot and declared node budget; p999 of a few hundred "
                    "requests is close to the maximum"}


def config(args, k):
    return {"workload": f"batched {args.nets} nets: tree-sum / bitonic-sort 50-50 by seed, depth log-uniform "
                        f"[{args.dmin}, {args.dmax}], u24 keys",
            "nets": args.nets, "dmin": args.dmin, "dmax": args.dmax,
            "steps_cover": f"the batch split into {k} size-balanced slices, one persistent launch (CUDA graph) "
                           f"per slice; the {k} timed steps reduce every net once",
            "l2": "flushed between steps (512 MiB write); heaps far above L2",
            "parallelism": f"weak: {args.gpus} x 1 GPU, size-balanced disjoint shares of nets x {args.gpus} nets"}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    t, n = pow2_threads()
    entries = W.batch_entries(args.nets, args.dmin, args.dmax, seed=0)
    k = max(1, args.steps)
    vals, descs = [], []
    for step in range(args.warmup + args.steps):
        sample = mass_sample(entries, args.ref_budget, seed=1000 + step)
        total, secs, desc = cpu_run(sample, t)
        if step >= args.warmup:
            vals.append((total, secs))
            descs.append(desc)
    value = sum(a for a, _ in vals) / sum(b for _, b in vals) / 1e9
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": config(args, k),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": t, "kind": "port",
                         "sample": f"per step: {descs[0] if descs else ''} (a fresh mass-weighted draw per step; "
                                   f"value = all timed steps' interactions over their normal() time)",
                         "host_cpus": n},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def roofline_record(alg, atoms, sec, hbm, peak_kind, arate, anote, traffic, tcap, kernel):
    """The kernel's roofline for one launch: `frac` is the HBM fraction of the
    algorithmic bytes (achieved GB/s over the measured copy bandwidth); the
    same launch's algorithmic atomics over the measured random-word atomic
    rate form the second bound (t_min = max(bytes / HBM, atomics / rate)),
    and `bound_frac` = t_min / t is the fraction of the binding one."""
    achieved = alg / sec / 1e9
    rec = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
           "traffic": traffic, "traffic_source": tcap, "peak_kind": f"{peak_kind} (copy bandwidth)",
           "kernel": kernel, "kernel_ms_per_launch": 1000.0 * sec, "algorithmic_bytes_per_launch": alg,
           "algorithmic_atomics_per_launch": atoms}
    if arate:
        a = atoms / sec
        rec["atomic"] = {"achieved": a / 1e9, "peak": arate / 1e9, "unit": "G atomics/s", "frac": a / arate,
                         "peak_kind": "measured (hvm64_atomic_peak, random 64-bit words of a 4 GiB array)",
                         "note": anote}
        t_min = max(alg / (hbm * 1e9), atoms / arate)
        rec["binding"] = "atomic" if atoms / arate > alg / (hbm * 1e9) else "hbm"
        rec["bound_frac"] = t_min / sec
    return rec


def single_net_leg(hvm64, args):
    """The single-net bitonic sort of 2^20 keys (8.8e9 interactions): device
    throughput and its own roofline record, checked against the golden
    counts."""
    text = W.bitonic(args.single_depth, 2)
    book = hvm64.Book.from_str(text)
    net = hvm64.Net(book, int(args.single_heap_gb * (1 << 30)))
    tune = hvm64.Tuning(timeout_ms=600000)
    net.boot("main")
    rw = net.normal(tune)
    ms = net.device_ms
    st = net.stats()
    counts = rw.as_dict()
    got = net.readback()
    ok = W.leaves(got) == sorted(W.sort_keys(args.single_depth, 2))
    gold = None
    try:
        gold = json.load(open(os.path.join(ROOT, "tests", "golden", "workload_counts.json")))[
            f"bitonic_{args.single_depth}_2"]["counts"]
    except Exception:
        pass
    alg = algorithmic_bytes(counts, st)
    atoms = algorithmic_atomics(counts, st)
    arate, anote = atomic_peak()
    tpi, tcap = traffic_per_interaction()
    hbm_peak, peak_kind = peaks()
    del net
    return {"workload": f"single net: bitonic sort of 2^{args.single_depth} u24 keys (seed 2)",
            "value": rw.total() / (ms / 1000.0) / 1e9, "unit": UNIT, "device_ms": ms,
            "interactions": rw.total(), "sorted": ok, "counts_match_golden": (counts == gold) if gold else None,
            "roofline": roofline_record(alg, atoms, ms / 1000.0, hbm_peak, peak_kind, arate, anote,
                                        tpi * rw.total() if tpi else None, tcap, "reduce_kernel, one launch"),
            "heap_nodes_used": st["heap_nodes_used"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nets", type=int, default=4096)
    ap.add_argument("--dmin", type=int, default=8)
    ap.add_argument("--dmax", type=int, default=18)
    ap.add_argument("--plain-nets", type=int, default=256, help="nets timed one-per-launch for the plain arm")
    ap.add_argument("--e2e-steps", type=int, default=2, help="slices timed end to end through the public API")
    ap.add_argument("--cpu-budget", type=float, default=2e9, help="interactions in the CPU-baseline sample")
    ap.add_argument("--ref-budget", type=float, default=5e8, help="interactions per reference-arm step")
    ap.add_argument("--count-check", type=float, default=3e8,
                    help="interactions of the nets whose per-rule counts are checked against the oracle")
    ap.add_argument("--heap-gb", type=float, default=48)
    ap.add_argument("--device-only", action="store_true", help="skip the plain, e2e, serving and CPU legs")
    ap.add_argument("--serve-requests", type=int, default=96, help="requests per offered load (0: no serving leg)")
    ap.add_argument("--serve-slots", type=int, default=64)
    ap.add_argument("--serve-wait-s", type=float, default=120.0,
                    help="give up on a load this long after its last arrival")
    ap.add_argument("--single-depth", type=int, default=20, help="single-net bitonic leg: 2^d keys (0: skip)")
    ap.add_argument("--single-heap-gb", type=float, default=32)
    ap.add_argument("--full-launch", action="store_true",
                    help="also time all nets in ONE launch (one step of the whole batch)")
    ap.add_argument("--autotune", type=int, default=1, help="pick the launch knobs on a sample first (0: defaults)")
    ap.add_argument("--tune-budget", type=float, default=3e9, help="interactions in the autotuner's sample")
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
        glob = W.batch_entries(args.nets * world, args.dmin, args.dmax, seed=0)
        entries = shard.rank_share(glob, est, rank, world)
    else:
        entries = W.batch_entries(args.nets, args.dmin, args.dmax, seed=0)
    K = max(1, args.steps)
    slices = slices_of(entries, K)
    order = [e for s in slices for e in s]  # the Batch holds the nets slice by slice
    bounds, o = [], 0
    for s in slices:
        bounds.append((o, len(s)))
        o += len(s)
    text = W.batch_book(order)
    book = hvm64.Book.from_str(text)
    names = [f"main_{j}" for _, _, j in order]
    heap = int(args.heap_gb * (1 << 30))
    tune_report = None
    if args.autotune:
        import autotune
        sample = mass_sample(entries, args.tune_budget, seed=7, first_may_exceed=False)
        tune, tune_report = autotune.autotune(book, [f"main_{j}" for _, _, j in sample], heap,
                                              sample=len(sample), timeout_ms=600000)
    else:
        tune = hvm64.Tuning(timeout_ms=600000)
    tune.flags |= hvm64.TUNE_GRAPH  # each step replays a captured CUDA graph
    batch = hvm64.Batch(book, names, heap)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def check_slice(k):
        f, c = bounds[k]
        bad = 0
        for i in range(f, f + c):
            kind, d, j = order[i]
            bad += 0 if W.check_result(kind, d, j, batch.readback(i)) else 1
        return bad

    for w in range(args.warmup):
        f, c = bounds[w % K]
        batch.normal(hvm64.PERSISTENT, tune, first=f, count=c)

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, kernel_ms, bad = [], [], 0
    agg_stats = {}
    with Clocks(local) as clk:
        for k in range(K):
            f, c = bounds[k]
            flush.fill_(1)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            batch.normal(hvm64.PERSISTENT, tune, first=f, count=c)
            e1.record()
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            kernel_ms.append(batch.device_ms)
            st = batch.stats()
            for key, v in st.items():
                agg_stats[key] = agg_stats.get(key, 0) + v
            bad += check_slice(k)  # every net's normal form, outside the step's events
    torch.cuda.synchronize()
    elapsed = sum(step_ms) / 1000.0
    total_per_rank = sum(batch.rwts[i].total() for i in range(batch.n))
    counts = {key: sum(getattr(batch.rwts[i], key) for i in range(batch.n))
              for key in ("anni", "comm", "eras", "dref", "oper")}
    if dist:
        elapsed = shard.max_over_ranks(elapsed, dist, "cuda")
        total_all = shard.sum_over_ranks(total_per_rank, dist, "cuda")
    else:
        total_all = float(total_per_rank)
    value = total_all / elapsed / 1e9

    # per-rule counts of a mass-weighted sample of nets against the oracle
    count_check = None
    if rank == 0 and not args.device_only and args.count_check > 0:
        from oracle import oracle
        t, _ = pow2_threads()
        sample = mass_sample(entries, args.count_check, seed=11, first_may_exceed=False)
        idx = {e: i for i, e in enumerate(order)}
        mism = 0
        for e in sample:
            _, want, _ = oracle.run_book(text, entry=f"main_{e[2]}", mode=oracle.MODE_PARALLEL, threads=t)
            mism += 0 if batch.rwts[idx[e]].as_dict() == want else 1
        count_check = {"nets": len(sample), "interactions": int(sum(est(e) for e in sample)),
                       "mismatches": mism, "sample": "mass-weighted draw of nets up to the budget"}

    # roofline of reduce_kernel: algorithmic bytes of the timed launches over
    # their device time (CUDA events the library records on its stream)
    hbm, peak_kind = peaks()
    alg = algorithmic_bytes(counts, agg_stats)
    atoms = algorithmic_atomics(counts, agg_stats)
    arate, anote = atomic_peak()
    ksec = sum(kernel_ms) / 1000.0
    tpi, tcap = traffic_per_interaction()
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed * 1000.0 / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": config(args, K),
        "interactions": total_all, "counts": counts, "nets_bad": bad, "count_check": count_check,
        "roofline": roofline_record(alg / K, atoms / K, ksec / K, hbm, peak_kind, arate, anote,
                                    tpi * total_per_rank / K if tpi else None, tcap,
                                    "reduce_kernel (+ boot_kernel) device time per launch (one launch per step)"),
        "gpu_launches": 4 * K,
        "tuning": {"knobs": {key: getattr(tune, key) for key in ("blocks_per_sm", "chunk_nodes", "donate_min",
                                                                  "queue_slots_log2", "max_warps_per_net")},
                   "cuda_graph": True, "autotune": tune_report},
        "clocks": clk.summary(),
        "device_stats": agg_stats,
    }

    if args.full_launch:
        # the whole batch in ONE persistent launch (no slicing)
        batch.normal(hvm64.PERSISTENT, tune)
        fl = batch.device_ms
        tot = sum(batch.rwts[i].total() for i in range(batch.n))
        out["full_launch"] = {"value": tot / (fl / 1000.0) / 1e9, "unit": UNIT, "device_ms": fl,
                              "interactions": tot, "nets": batch.n}

    if not args.device_only:
        # plain arm: the batch's first `plain_nets` nets, one launch each
        plain_entries = entries[:args.plain_nets]
        if plain_entries:
            pnames = [f"main_{j}" for _, _, j in plain_entries]
            pbatch = hvm64.Batch(book, pnames, heap)
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
            sbatch = hvm64.Batch(book, pnames, heap)
            sbatch.normal(hvm64.PERSISTENT, tune)
            s0 = time.perf_counter()
            sbatch.normal(hvm64.PERSISTENT, tune)
            sub_s = time.perf_counter() - s0
            del sbatch
            out["plain"] = {"value": ptotal / plain_s / 1e9, "unit": UNIT, "nets": len(plain_entries),
                            "device_value": ptotal / (pdev / 1000.0) / 1e9,
                            "batched_same_nets": ptotal / sub_s / 1e9,
                            "note": "one net per launch (wall time incl. launch + sync) vs the batched "
                                    "reducer on the same nets in one launch"}

        # e2e through the public API from host memory, per slice: net list to
        # the device, reduce, every net's normal form back to host text.  One
        # untimed slice first (the process's first batch pays one-time costs:
        # allocations, the page-locked readback staging).
        e2e_s, e2e_tot, h2d, d2h = 0.0, 0, 0, 0
        ne = max(1, min(args.e2e_steps, K))
        for it, k in enumerate([ne % K] + list(range(ne))):
            warm = it == 0
            f, c = bounds[k]
            torch.cuda.synchronize()
            e0 = time.perf_counter()
            ebatch = hvm64.Batch(book, names[f:f + c], heap)
            ebatch.normal(hvm64.PERSISTENT, tune)
            for i in range(ebatch.n):
                ebatch.readback(i)
            dt = time.perf_counter() - e0
            if warm:
                del ebatch
                continue
            e2e_s += dt
            e2e_tot += sum(ebatch.rwts[i].total() for i in range(ebatch.n))
            st = ebatch.stats()
            h2d += st["h2d_bytes"]
            d2h += st["d2h_bytes"]
            del ebatch
        if dist:
            e2e_s = shard.max_over_ranks(e2e_s, dist, "cuda")
        out["e2e"] = {"value": e2e_tot * (world if dist else 1) / e2e_s / 1e9, "unit": UNIT,
                      "h2d_bytes_per_step": h2d // ne, "d2h_bytes_per_step": d2h // ne,
                      "steps": ne,
                      "note": "per slice: Batch create (Book tables + net list to the device) + normal + "
                              "readback of every net's normal form to host text, wall clock; after one "
                              "untimed slice"}

        if rank == 0:
            del batch
            if args.single_depth:
                try:
                    out["single_net"] = single_net_leg(hvm64, args)
                except Exception as e:
                    out["single_net"] = {"error": f"{type(e).__name__}: {e}"}
            if args.serve_requests > 0:
                # the serving leg must not cost the benchmark line; a failed
                # attempt is reported and the leg runs once more
                failed = []
                for attempt in range(2):
                    try:
                        out["serving"] = serve_leg(args, hvm64)
                        if failed:
                            out["serving"]["failed_attempts"] = failed
                        break
                    except Exception as e:
                        failed.append(f"{type(e).__name__}: {e}")
                        out["serving"] = {"error": failed[-1], "failed_attempts": failed}
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
