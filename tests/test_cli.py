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
