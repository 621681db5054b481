"""The `hvm64` command line (hvm-64_b200/csrc/cli.cpp) on the CPU: argument
handling, the net that `run` builds from its arguments (apply_tree), and
failing loudly without a GPU.  The nets it would reduce are reduced by the
oracle here and must give the reference CLI's outputs (tests/cli.rs cases)."""
import json
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CLI = os.path.join(ROOT, "hvm-64_b200", "build", "hvm64")
CASES = json.load(open(os.path.join(HERE, "golden", "cli.json")))


def _cli():
    if not os.path.exists(CLI):
        import build
        build.build()
    return CLI


def _run(args, cwd):
    return subprocess.run([_cli()] + args, capture_output=True, text=True, cwd=cwd, timeout=120)


RUNS = [c for c in CASES["runs"] if c["args"][0] in ("run", "reduce")]


@pytest.mark.parametrize("case", RUNS, ids=[" ".join(c["args"]) for c in RUNS])
def test_cli_nets_reduce_to_reference_outputs(case, tmp_path):
    from oracle import oracle
    path = tmp_path / "arithmetic.hvm"
    path.write_text(CASES["arithmetic"])
    args = [str(path) if a == "{arithmetic}" else a for a in case["args"]]
    if "not found" in case["expect"]:
        r = _run(args, tmp_path)
        assert r.returncode != 0
        assert (r.stdout + r.stderr).strip() == case["expect"]
        return
    r = _run(args + ["--print-net"] if "--" not in args else args[:args.index("--")] + ["--print-net"] +
             args[args.index("--"):], tmp_path)
    assert r.returncode == 0, r.stderr
    nets = r.stdout.strip().split("\n")
    book = CASES["arithmetic"] if "{arithmetic}" in case["args"] else ""
    got = [oracle.run_expr(book, n)[0] for n in nets]
    assert "\n".join(got) == case["expect"]


def test_cli_usage_and_bad_memory(tmp_path):
    assert _run([], tmp_path).returncode == 2
    assert _run(["frobnicate"], tmp_path).returncode == 2
    assert _run(["run"], tmp_path).returncode == 2
    r = _run(["reduce", "-m", "12Q", "--", "1"], tmp_path)
    assert r.returncode == 2 and "memory" in r.stderr


def test_cli_without_gpu_fails_loudly(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = _run(["reduce", "--", "1"], tmp_path)
    assert r.returncode == 101
    assert "error" in r.stderr and "CUDA" in r.stderr


GPU_RUNS = [c for c in RUNS if "not found" not in c["expect"]]
STATS = [r"RWTS   : +[\d_]+", r"- ANNI : +[\d_]+", r"- COMM : +[\d_]+", r"- ERAS : +[\d_]+", r"- DREF : +[\d_]+",
         r"- OPER : +[\d_]+", r"TIME   : \d+\.\d{3}(s|ms|µs|ns)", r"RPS    : (\d+\.\d{3}|inf|NaN) M"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GPU_RUNS, ids=[" ".join(c["args"]) for c in GPU_RUNS])
def test_cli_on_gpu_prints_reference_outputs(case, tmp_path):
    """`hvm64 run` / `hvm64 reduce` reduce on the GPU and print the reference
    CLI's normal forms (tests/cli.rs:40-131), and with -s the statistics block
    of src/main.rs:195-204 (RWTS and per-rule lines with the reference's
    pretty numbers and widths, TIME as a Duration, RPS) once per expression;
    the counts equal the oracle's for the same net."""
    import re
    from oracle import oracle
    path = tmp_path / "arithmetic.hvm"
    path.write_text(CASES["arithmetic"])
    args = [str(path) if a == "{arithmetic}" else a for a in case["args"]]
    cut = args.index("--") if "--" in args else len(args)
    r = _run(args[:cut] + ["-s"] + args[cut:], tmp_path)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == case["expect"]
    lines = r.stderr.strip().split("\n")
    outs = case["expect"].split("\n")
    assert len(lines) == 8 * len(outs), r.stderr
    nets = _run(args[:cut] + ["--print-net"] + args[cut:], tmp_path).stdout.strip().split("\n")
    book = CASES["arithmetic"] if "{arithmetic}" in case["args"] else ""
    for k, net in enumerate(nets):
        block = lines[8 * k:8 * k + 8]
        for line, pat in zip(block, STATS):
            assert re.fullmatch(pat, line), (line, pat)
        _, want = oracle.run_expr(book, net)
        got = [int(l.split(":")[1].replace("_", "")) for l in block[1:6]]
        assert got == [want[x] for x in ("anni", "comm", "eras", "dref", "oper")]
        assert int(block[0].split(":")[1].replace("_", "")) == sum(want.values())
