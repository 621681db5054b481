"""Writes tests/golden/workload_counts.json: the oracle's normal-form checks
and per-rule counts for workload instances too large to run through the
oracle inside a GPU test (minutes of CPU time each).

    python tests/golden/make_workload_counts.py

The oracle is the C++ restatement of the reference evaluator (oracle/), run
in its Net::parallel_normal mode on this machine's cores; counts do not
depend on the thread count (strong confluence), which tests/test_oracle.py
checks on the reference's own fixtures.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "hvm-64_b200"))

import workloads as W  # noqa: E402
from oracle import oracle  # noqa: E402

OUT = os.path.join(HERE, "workload_counts.json")

# (key, book text builder, check of the read-back normal form)
CASES = [
    ("bitonic_20_2", lambda: W.bitonic(20, 2),
     lambda t: W.leaves(t) == sorted(W.sort_keys(20, 2))),
    ("church_big", lambda: W.church_big(),
     lambda t: t == W.CHURCH_BIG_NORMAL_FORM),
]


def main(only=None):
    try:
        out = json.load(open(OUT))
    except FileNotFoundError:
        out = {}
    threads = os.cpu_count() or 1
    for key, build, check in CASES:
        if only and key not in only:
            continue
        t0 = time.time()
        text, rw, secs = oracle.run_book(build(), mode=oracle.MODE_PARALLEL, threads=threads)
        assert check(text), f"{key}: oracle normal form failed its check"
        out[key] = {"counts": rw, "total": sum(rw.values()), "oracle_threads": threads,
                    "oracle_normal_s": round(secs, 2)}
        print(key, out[key], f"{time.time() - t0:.1f} s", flush=True)
        json.dump(out, open(OUT, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main(set(sys.argv[1:]) or None)
