"""Extract the reference's own golden vectors into JSON fixtures.

Run once in a container where the reference checkout is mounted:

    python tests/golden/make_golden.py /path/to/hvm-64

It reads, as text, and writes under tests/golden/:
  programs.json   every `{examples,tests/programs}/**/*.hvm` program with its
                  `tests/snapshots/run@<name>.snap` normal form and the
                  ANNI/COMM/ERAS/DREF/OPER counts (tests/tests.rs:28-42)
  lists.json      tests/lists.rs: list_put_got.hvm and the pinned RWTS totals
  cli.json        tests/cli.rs: `reduce`/`run` outputs and apply_tree cases
  labels.json     host/src/calc_labels.rs:196-234 label-set expectations
  pre_reduce.json tests/snapshots/pre_reduce_run@<name>.snap (pre-reduce then
                  run)
  transform.json  tests/transform.rs: per-rule counts of pre-reduce + run

Nothing at test time reads the reference checkout; only these fixtures.
"""
import json
import os
import re
import sys


def snap_body(path):
    text = open(path).read()
    # insta header: ---\n...\n---\n
    parts = text.split("---\n", 2)
    return parts[2] if len(parts) == 3 else text


def parse_counts(lines):
    out = {}
    for ln in lines:
        m = re.match(r"^(RWTS|- ANNI|- COMM|- ERAS|- DREF|- OPER)\s*:\s*([\d_]+)", ln)
        if m:
            key = m.group(1).replace("- ", "").lower()
            out[key] = int(m.group(2).replace("_", ""))
    return out


def programs(ref):
    out = []
    for top in ("examples", "tests/programs"):
        for dirpath, _, files in os.walk(os.path.join(ref, top)):
            for f in sorted(files):
                if not f.endswith(".hvm"):
                    continue
                full = os.path.join(dirpath, f)
                rel = os.path.relpath(full, ref)
                name = rel[:-4].replace("/", "::")
                snap = os.path.join(ref, "tests/snapshots", f"run@{name}.snap")
                if not os.path.exists(snap):
                    continue
                body = snap_body(snap).rstrip("\n").split("\n")
                # the normal form may span lines (redexes print as "\n  & a ~ b")
                idx = next(i for i, ln in enumerate(body) if ln.startswith("RWTS"))
                counts = parse_counts(body[idx:])
                out.append({
                    "name": name,
                    "path": rel,
                    "source": open(full).read(),
                    "text": "\n".join(body[:idx]),
                    "anni": counts["anni"], "comm": counts["comm"], "eras": counts["eras"],
                    "dref": counts["dref"], "oper": counts["oper"], "total": counts["rwts"],
                })
    out.sort(key=lambda p: p["name"])
    return out


def pre_reduce(ref):
    """tests/tests.rs:44-55: each program pre-reduced (`main` skipped, no
    rewrite limit) then run: `pre_reduce_run@<name>.snap` holds the normal
    form, the pre-reduce Rewrites and the run's Rewrites."""
    progs = []
    for p in programs(ref):
        snap = os.path.join(ref, "tests/snapshots", f"pre_reduce_run@{p['name']}.snap")
        if not os.path.exists(snap):
            continue
        body = snap_body(snap).rstrip("\n").split("\n")
        if "pre-reduce:" in body:
            i, j = body.index("pre-reduce:"), body.index("run:")
            text, pre, run = "\n".join(body[:i]), parse_counts(body[i + 1:j]), parse_counts(body[j + 1:])
        else:  # no run (tests.rs:47-50): only the pre-reduce Rewrites
            text, pre, run = None, parse_counts(body), None
        progs.append({"name": p["name"], "source": p["source"], "text": text, "pre": pre, "run": run})
    return progs


def transform(ref):
    """tests/transform.rs:14-47 (test_fast_pre_reduce): heavy_pre_reduction.hvm
    without `black_box` is pre-reduced keeping only the listed defs' reduction
    (every other def is skipped), `black_box` is put back, the entry is run
    with normal(), and the pre-reduce plus run counts are pinned."""
    src = open(os.path.join(ref, "tests/transform.rs")).read()
    body = src[src.index("fn test_fast_pre_reduce"):]
    lists = re.findall(r"!\[([^\]]*)\]\.contains", body)[:2]
    only = [re.findall(r'"(\w+)"', x) for x in lists]
    snap = re.search(r'@r###"(.*?)"###', body, re.S).group(1)
    lines = [ln.strip() for ln in snap.strip("\n").split("\n")]
    i = lines.index("Slow:")
    return {
        "source": open(os.path.join(ref, "tests/programs/heavy_pre_reduction.hvm")).read(),
        "removed": "black_box",
        "cases": [
            {"only": only[0], "entry": "main_fast", "total": parse_counts(lines[1:i])},
            {"only": only[1], "entry": "main_slow", "total": parse_counts(lines[i + 1:])},
        ],
    }


def lists(ref):
    src = open(os.path.join(ref, "tests/lists.rs")).read()
    got_idx = [int(x) for x in re.search(r"for index in \[([^\]]*)\]", src).group(1).split(",")]
    put_pairs = [tuple(int(y) for y in p) for p in re.findall(r"\((\d+),\s*(\d+)\)", re.search(
        r"for \(index, value\) in \[([^\]]*)\]", src).group(1))]
    fns = re.split(r"fn test_list_put", src)
    got_expect = [int(x) for x in re.findall(r'@"(\d+)"', fns[0])]
    put_expect = [int(x) for x in re.findall(r'@"(\d+)"', fns[1])]
    return {
        "source": open(os.path.join(ref, "tests/programs/list_put_got.hvm")).read(),
        "got": [{"index": i, "total": t} for i, t in zip(got_idx, got_expect)],
        "put": [{"index": i, "value": v, "total": t} for (i, v), t in zip(put_pairs, put_expect)],
    }


def cli(ref):
    src = open(os.path.join(ref, "tests/cli.rs")).read()
    apply = []
    for m in re.finditer(r'eval_with_args\("((?:[^"\\]|\\.)*)",\s*&\[((?:"[^"]*",?\s*)*)\]\),\s*@"([^"]*)"', src):
        args = re.findall(r'"([^"]*)"', m.group(2))
        apply.append({"fun": m.group(1), "args": args, "expect": m.group(3)})
    runs = []
    pat = re.compile(r'execute_hvm64\(&\[(.*?)\]\)\.unwrap\(\)\.1,\s*@r###"\n(.*?)"###', re.S)
    for m in pat.finditer(src):
        raw_args = m.group(1)
        toks = re.findall(r'"((?:[^"\\]|\\.)*)"|(&arithmetic_program)', raw_args)
        args = [a if a else "{arithmetic}" for a, b in toks]
        expect = "\n".join(ln.strip() for ln in m.group(2).strip("\n").split("\n")).strip()
        runs.append({"args": args, "expect": expect})
    return {
        "arithmetic": open(os.path.join(ref, "examples/arithmetic.hvm")).read(),
        "apply_tree": apply,
        "runs": runs,
    }


def labels(ref):
    src = open(os.path.join(ref, "host/src/calc_labels.rs")).read()
    body = re.search(r'&"(.*?)"\s*\.parse\(\)', src, re.S).group(1)
    sets = {}
    for name, labs in re.findall(r'\("(\w+)",\s*\[([^\]]*)\]', src):
        sets[name] = [int(x) for x in labs.split(",") if x.strip()]
    return {"book": body, "sets": sets}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HVM64_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: make_golden.py <reference checkout>")
    here = os.path.dirname(os.path.abspath(__file__))
    for fname, data in (("programs.json", programs(ref)), ("lists.json", lists(ref)),
                        ("cli.json", cli(ref)), ("labels.json", labels(ref)),
                        ("pre_reduce.json", pre_reduce(ref)), ("transform.json", transform(ref))):
        with open(os.path.join(here, fname), "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
            f.write("\n")
        print(fname, len(data) if isinstance(data, list) else "ok")


if __name__ == "__main__":
    main()
