"""Autotuner for the batched reducer's launch knobs (hvm64_tuning).

The knobs trade against each other per workload: resident reducer blocks per
SM (occupancy vs. shared memory per warp), allocator chunk size (bump-pointer
traffic vs. nodes stranded in half-used chunks), the stack depth above which a
warp donates work (the steal threshold: load balance vs. queue traffic), the
queue capacity, and how many warps one net's work may spread over (warps per
net: locality in one net's heap vs. parallelism).
`autotune` runs a sample of the batch (the nets are independent, so a sample
has the batch's mix) under candidate settings and keeps the fastest by device
time, one knob at a time (coordinate descent from the defaults), so the search
costs a few runs per knob instead of the whole grid.
"""
import time

import hvm64

# Candidate values per knob; 0 is the library default.
SPACE = {
    "blocks_per_sm": (0, 6, 5),
    "chunk_nodes": (0, 64, 1024, 4096),
    "donate_min": (0, 32, 128, 256),
    "queue_slots_log2": (0, 18, 22),
    "max_warps_per_net": (0, 64, 512),
}
ORDER = ("blocks_per_sm", "chunk_nodes", "donate_min", "queue_slots_log2", "max_warps_per_net")


def coordinate_search(measure, space=SPACE, order=ORDER, rounds=1):
    """Minimise measure(settings) -> seconds (None for a failed setting) one
    knob at a time.  Returns (best settings, best seconds, trials)."""
    best = {k: space[k][0] for k in order}
    best_t = measure(dict(best))
    trials = [(dict(best), best_t)]
    if best_t is None:
        raise RuntimeError("the default settings failed")
    for _ in range(rounds):
        for k in order:
            for v in space[k]:
                if v == best[k]:
                    continue
                cand = dict(best)
                cand[k] = v
                t = measure(dict(cand))
                trials.append((cand, t))
                if t is not None and t < best_t:
                    best, best_t = cand, t
    return best, best_t, trials


def autotune(book, names, heap_bytes=0, sample=512, timeout_ms=120000, flags=0, repeats=1):
    """Pick hvm64_tuning knobs for a batch of Def entries `names` by timing a
    sample of it (every len/sample-th net).  Returns (Tuning, report dict)."""
    step = max(1, len(names) // sample)
    picked = names[::step][:sample]
    batch = hvm64.Batch(book, picked, heap_bytes)

    def measure(settings):
        t = hvm64.Tuning(timeout_ms=timeout_ms, flags=flags, **settings)
        best = None
        for _ in range(repeats):
            rc = batch.normal(hvm64.PERSISTENT, t, check=False)
            if rc != hvm64.OK:
                return None
            ms = batch.device_ms / 1000.0
            best = ms if best is None else min(best, ms)
        return best

    batch.normal(hvm64.PERSISTENT, hvm64.Tuning(timeout_ms=timeout_ms, flags=flags))  # warm-up
    t0 = time.perf_counter()
    best, best_s, trials = coordinate_search(measure)
    interactions = sum(batch.rwts[i].total() for i in range(batch.n))
    del batch
    report = {"sample_nets": len(picked), "trials": len(trials), "search_s": time.perf_counter() - t0,
              "chosen": best, "sample_gips": interactions / best_s / 1e9 if best_s else None,
              "default_gips": interactions / trials[0][1] / 1e9 if trials[0][1] else None}
    return hvm64.Tuning(timeout_ms=timeout_ms, flags=flags, **best), report
