"""Pre-reduce (transform/src/pre_reduce.rs) -- the Book pass that reduces
every Def ahead of time with the reducer.

- The oracle's restatement is pinned against the reference's own vectors:
  the pre_reduce_run@*.snap snapshots (tests/tests.rs:44-55: pre-reduce with
  `main` skipped, then run main), test_fast_pre_reduce (tests/transform.rs:
  14-47: a Book with a missing Def, so inert Defs capture redexes) and the CLI
  `transform -Opre-reduce` outputs (tests/cli.rs:133-182).
- The device runtime compiled for the host (tests/emu) runs the same host
  driver as the CUDA library, on many threads, and must give the oracle's
  Book text and counts.
- On the GPU, hvm64.pre_reduce and `hvm64 transform` give the same.
"""
import json
import os
import re
import subprocess
import sys

import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")
PRE = json.load(open(os.path.join(GOLD, "pre_reduce.json")))
TRANSFORM = json.load(open(os.path.join(GOLD, "transform.json")))
CLI = json.load(open(os.path.join(GOLD, "cli.json")))
KEYS = oracle.COUNT_KEYS

RUN_LIMIT = 5_000_000   # run the pre-reduced Book on the oracle up to this many interactions
EMU_LIMIT = 60_000      # pre-reduce interactions the emulator does in a few seconds


def with_total(rw):
    d = {k: rw[k] for k in KEYS}
    d["rwts"] = sum(d.values())
    return d


def split_defs(text):
    """Def name -> its text, in source order (a Def starts at `@name =`)."""
    defs, cur = {}, None
    for ln in text.split("\n"):
        m = re.match(r"@(\S+)\s*=", ln)
        if m:
            cur = m.group(1)
            defs[cur] = ln
        elif ln.strip() and cur:
            defs[cur] += "\n" + ln
    return defs


def fast_case(case):
    """tests/transform.rs:14-29: the Book without `black_box`, every Def but
    case["only"] skipped; returns (book text, skip list, removed Def's text)."""
    defs = split_defs(TRANSFORM["source"])
    removed = defs.pop(TRANSFORM["removed"])
    return "\n".join(defs.values()), [n for n in defs if n not in case["only"]], removed


def cli_transform_cases():
    out = []
    for r in CLI["runs"]:
        if r["args"][0] != "transform":
            continue
        a = r["args"]
        skip = a[a.index("--pre-reduce-skip") + 1].split(" ") if "--pre-reduce-skip" in a else []
        out.append(pytest.param(r, skip, id=" ".join(a)))
    return out


def norm_lines(text):
    return "\n".join(ln.strip() for ln in text.strip("\n").split("\n")).strip()


# ---- the oracle against the reference's vectors ---------------------------------

@pytest.mark.parametrize("prog", PRE, ids=[p["name"] for p in PRE])
def test_oracle_pre_reduce_snapshot(prog):
    text, rw, not_normal = oracle.pre_reduce(prog["source"], skip=("main",))
    assert with_total(rw) == prog["pre"]
    assert not_normal == []
    if prog["run"] and prog["run"]["rwts"] <= RUN_LIMIT:
        nf, run, _ = oracle.run_book(text, "main", mode=oracle.MODE_PARALLEL, threads=1)
        assert nf == prog["text"]
        assert with_total(run) == prog["run"]


@pytest.mark.parametrize("case", TRANSFORM["cases"], ids=[c["entry"] for c in TRANSFORM["cases"]])
def test_oracle_fast_pre_reduce(case):
    book, skip, removed = fast_case(case)
    text, pre, _ = oracle.pre_reduce(book, skip=skip)
    _, run, _ = oracle.run_book(text + "\n" + removed, case["entry"], mode=oracle.MODE_NORMAL)
    assert with_total({k: pre[k] + run[k] for k in KEYS}) == case["total"]


@pytest.mark.parametrize("run,skip", cli_transform_cases())
def test_oracle_cli_transform(run, skip):
    text, _, _ = oracle.pre_reduce(CLI["arithmetic"], skip=skip)
    assert norm_lines(text) == run["expect"]


def test_oracle_rewrite_limit_reports_not_normal():
    """Net::reduce(limit) stops after `limit` popped redexes (net.rs:41-52):
    such Defs are listed, the others reach normal form."""
    src = next(p for p in PRE if p["name"] == "tests::programs::dec_bits_tree")["source"]
    _, _, nn_all = oracle.pre_reduce(src, skip=("main",))
    _, _, nn_small = oracle.pre_reduce(src, skip=("main",), max_rwts=50)
    assert nn_all == [] and nn_small


# ---- the device runtime on host threads ---------------------------------------

def _emu():
    sys.path.insert(0, HERE)
    import test_emu
    L = test_emu._lib()
    import ctypes as c
    L.hvm64emu_pre_reduce.argtypes = [c.c_char_p, c.c_char_p, c.c_uint64, c.c_uint, c.c_uint, c.c_uint,
                                      c.c_uint64, c.c_uint64, c.POINTER(c.c_char_p), c.POINTER(c.c_uint64),
                                      c.POINTER(c.c_char_p), c.c_char_p, c.c_size_t]
    return L


def emu_pre_reduce(text, skip=("main",), max_rwts=(1 << 64) - 1, threads=8, ring=2, spill=24):
    import ctypes
    L = _emu()
    out, nn = ctypes.c_char_p(), ctypes.c_char_p()
    rw = (ctypes.c_uint64 * 5)()
    err = ctypes.create_string_buffer(256)
    rc = L.hvm64emu_pre_reduce(text.encode(), "\n".join(skip).encode(), max_rwts, threads, ring, spill, 4 << 20,
                               32, ctypes.byref(out), rw, ctypes.byref(nn), err, 256)
    assert rc == 0, err.value.decode()
    return out.value.decode(), dict(zip(KEYS, list(rw))), [x for x in nn.value.decode().split("\n") if x]


EMU_PROGS = [p for p in PRE if p["pre"]["rwts"] <= EMU_LIMIT]


@pytest.mark.parametrize("prog", EMU_PROGS, ids=[p["name"] for p in EMU_PROGS])
def test_emu_pre_reduce_matches_oracle(prog):
    want_text, want_rw, _ = oracle.pre_reduce(prog["source"], skip=("main",))
    text, rw, not_normal = emu_pre_reduce(prog["source"])
    assert with_total(rw) == prog["pre"]
    assert text == want_text
    assert not_normal == []


@pytest.mark.parametrize("case", TRANSFORM["cases"], ids=[c["entry"] for c in TRANSFORM["cases"]])
def test_emu_fast_pre_reduce(case):
    """Defs missing from the Book become inert Defs: their calls come back as
    redexes of the pre-reduced net (`& @black_box ~ ...`)."""
    book, skip, removed = fast_case(case)
    want_text, _, _ = oracle.pre_reduce(book, skip=skip)
    text, pre, _ = emu_pre_reduce(book, skip=skip, threads=1)
    assert text == want_text
    _, run, _ = oracle.run_book(text + "\n" + removed, case["entry"], mode=oracle.MODE_NORMAL)
    assert with_total({k: pre[k] + run[k] for k in KEYS}) == case["total"]


@pytest.mark.parametrize("limit", [10, 50, 400, 5000])
def test_emu_rewrite_limit_lists_the_oracles_defs(limit):
    """A Def whose reduction pops `limit` redexes or more is not normal in
    both; the device keeps its original net.  (The lists agree while no Def
    that stopped short is called by one reduced after it: the reference's
    later Defs then call the partly reduced net, the device's the original.)"""
    src = next(p for p in PRE if p["name"] == "tests::programs::dec_bits_tree")["source"]
    _, _, want = oracle.pre_reduce(src, skip=("main",), max_rwts=limit)
    _, _, got = emu_pre_reduce(src, max_rwts=limit)
    assert got == want


def test_emu_limit_zero_leaves_defs_without_redexes_normal():
    """Net::reduce(0) pops once before it checks the limit, so a Def with no
    redex after its boot is normal under any limit (net.rs:41-52)."""
    src = "@add = ($([+] $(a b)) (a b))\n@main = a & @add ~ (1 (2 a))\n@two = a & @add ~ (1 (1 a))"
    for limit in (0, 1):
        want_text, want_rw, want = oracle.pre_reduce(src, skip=("main",), max_rwts=limit)
        text, rw, got = emu_pre_reduce(src, max_rwts=limit)
        assert want == got == ["two"]


# ---- on the GPU --------------------------------------------------------------------

# (apelacion and burn pre-reduce one long sequential chain of 18-33 million
# interactions each: a single-warp workload, left to the oracle tests)
GPU_PROGS = [p for p in PRE if p["pre"]["rwts"] <= 100_000]


@pytest.mark.gpu
@pytest.mark.parametrize("prog", GPU_PROGS, ids=[p["name"] for p in GPU_PROGS])
def test_gpu_pre_reduce_matches_snapshot(prog):
    import hvm64
    want_text, _, _ = oracle.pre_reduce(prog["source"], skip=("main",))
    text, rw, not_normal = hvm64.pre_reduce(prog["source"], skip=("main",))
    assert with_total(rw.as_dict()) == prog["pre"]
    assert text == want_text
    assert not_normal == []
    if prog["run"] and prog["run"]["rwts"] <= 2_000_000:
        book = hvm64.Book.from_str(text)
        net = hvm64.Net(book, heap_bytes=1 << 30)
        net.boot("main")
        run = net.normal()
        assert net.readback() == prog["text"]
        assert with_total(run.as_dict()) == prog["run"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", TRANSFORM["cases"], ids=[c["entry"] for c in TRANSFORM["cases"]])
def test_gpu_fast_pre_reduce(case):
    import hvm64
    book, skip, removed = fast_case(case)
    text, pre, _ = hvm64.pre_reduce(book, skip=skip)
    net = hvm64.Net(hvm64.Book.from_str(text + "\n" + removed), heap_bytes=1 << 30)
    net.boot(case["entry"])
    run = net.normal()
    total = {k: pre.as_dict()[k] + run.as_dict()[k] for k in KEYS}
    assert with_total(total) == case["total"]


@pytest.mark.gpu
@pytest.mark.parametrize("limit", [10, 400])
def test_gpu_rewrite_limit_lists_the_oracles_defs(limit):
    import hvm64
    src = next(p for p in PRE if p["name"] == "tests::programs::dec_bits_tree")["source"]
    _, _, want = oracle.pre_reduce(src, skip=("main",), max_rwts=limit)
    _, _, got = hvm64.pre_reduce(src, skip=("main",), max_rwts=limit)
    assert got == want


@pytest.mark.gpu
@pytest.mark.parametrize("run,skip", cli_transform_cases())
def test_gpu_cli_transform(run, skip, tmp_path):
    """`hvm64 transform -Opre-reduce` prints the reference CLI's Book
    (tests/cli.rs:133-182)."""
    path = tmp_path / "arithmetic.hvm"
    path.write_text(CLI["arithmetic"])
    args = [str(path) if a == "{arithmetic}" else a for a in run["args"]]
    exe = os.path.join(ROOT, "hvm-64_b200", "build", "hvm64")
    p = subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert norm_lines(p.stdout) == run["expect"]


def test_cli_transform_without_passes_prints_the_book(tmp_path):
    """`hvm64 transform FILE` with no -O prints the parsed Book (src/main.rs:
    71-74): host code only."""
    path = tmp_path / "arithmetic.hvm"
    path.write_text(CLI["arithmetic"])
    exe = os.path.join(ROOT, "hvm-64_b200", "build", "hvm64")
    if not os.path.exists(exe):
        sys.path.insert(0, os.path.join(ROOT, "hvm-64_b200"))
        import build
        build.build()
    p = subprocess.run([exe, "transform", str(path)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 0, p.stderr
    assert p.stdout == oracle.book_roundtrip(CLI["arithmetic"]) + "\n"
    bad = subprocess.run([exe, "transform", "-O", "inline", str(path)], capture_output=True, text=True, timeout=60)
    assert bad.returncode == 2 and "pre-reduce" in bad.stderr
