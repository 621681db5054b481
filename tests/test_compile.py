"""Ahead-of-time Def specialisation -- the analogue of `hvm64 compile`
(src/compile.rs:110-161): a Book's Defs emitted as straight-line device
functions and compiled into the reducer in place of its instruction VM.

- CPU: the generated source, compiled into the host emulation of the device
  runtime, must reduce the reference fixtures to their snapshot normal forms
  and counts (the emulation reports that the compiled functions are the ones
  running).
- GPU: a library built by build.build_compiled runs the fixtures and the
  bitonic workload through the compiled functions, equal to the oracle and the
  snapshots; a Book it was not built for runs on the VM and is still right.
"""
import ctypes
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "hvm-64_b200"))
PROGRAMS = {p["name"]: p for p in json.load(open(os.path.join(HERE, "golden", "programs.json")))}
EMU_BUILD = os.path.join(HERE, "emu", "build")
KEYS = ("anni", "comm", "eras", "dref", "oper")

# fixtures whose Defs cover every instruction kind: constructors and wires
# (bitonic), numeric operators (numeric_casts), switches (dec_bits), labels
# (church_exp)
CPU_CASES = ["examples::sort::bitonic::bitonic_sort_lam", "tests::programs::numeric_casts",
             "tests::programs::dec_bits", "tests::programs::church_exp"]


def _source(text):
    import hvm64
    return hvm64.Book.from_str(text).compile_source()


def _emu_lib(text):
    """The emulation built with `text`'s compiled Defs."""
    import build
    src = _source(text)
    h = build.compiled_source_hash(src)
    os.makedirs(EMU_BUILD, exist_ok=True)
    hdr = os.path.join(EMU_BUILD, f"defs_{h}.cuh")
    so = os.path.join(EMU_BUILD, f"libemu_{h}.so")
    with open(hdr, "w") as f:
        f.write(src)
    srcs = [os.path.join(HERE, "emu", "emu.cpp"), os.path.join(ROOT, "hvm-64_b200", "csrc", "host.cpp")]
    subprocess.run(["g++", "-std=c++20", "-O2", "-pthread", "-fPIC", "-shared", "-DHVM_EMU_STRESS",
                    f'-DHVM_GEN_INCLUDE="{hdr}"', "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "hvm-64_b200", "csrc"), *srcs, "-o", so], check=True)
    L = ctypes.CDLL(so)
    c = ctypes
    L.hvm64emu_run.argtypes = [c.c_char_p, c.c_char_p, c.c_uint, c.c_uint, c.c_uint, c.c_uint, c.c_uint64,
                               c.c_uint64, c.POINTER(c.c_char_p), c.POINTER(c.c_uint64), c.c_char_p, c.c_size_t]
    L.hvm64emu_compiled_for.argtypes = [c.c_char_p]
    return L


@pytest.mark.parametrize("name", CPU_CASES)
def test_generated_defs_on_the_emulation(name):
    prog = PROGRAMS[name]
    L = _emu_lib(prog["source"])
    assert L.hvm64emu_compiled_for(prog["source"].encode()) == 1
    assert L.hvm64emu_compiled_for(b"@main = *") == 0  # another Book runs on the VM
    out = ctypes.c_char_p()
    rw = (ctypes.c_uint64 * 5)()
    err = ctypes.create_string_buffer(256)
    rc = L.hvm64emu_run(prog["source"].encode(), b"main", 8, 2, 24, 16, 256 << 20, 32, ctypes.byref(out), rw, err, 256)
    assert rc == 0, err.value.decode()
    assert out.value.decode() == prog["text"]
    assert dict(zip(KEYS, list(rw))) == {k: prog[k] for k in KEYS}


def test_generated_source_shape():
    """One function per Def, the dispatch, and the Book hash; every
    instruction kind becomes a direct call."""
    src = _source(PROGRAMS["examples::arithmetic"]["source"])
    assert "#define HVM_GEN_NDEFS 6u" in src
    assert src.count("HVM_COLD void gen_def_") == 6
    assert "HVM_INL bool gen_call(" in src
    assert "do_op_num(" in src or "do_op(" in src
    assert "switch (k)" not in src  # no instruction loop


# ---- on the GPU ------------------------------------------------------------------
GPU_SCRIPT = r"""
import json, sys
sys.path.insert(0, "hvm-64_b200")
import hvm64, workloads as W
from oracle import oracle
case = json.loads(sys.argv[1])
text = case["text"]
book = hvm64.Book.from_str(text)
out = {"compiled": book.is_compiled()}
net = hvm64.Net(book, heap_bytes=4 << 30)
net.boot("main")
rw = net.normal(hvm64.Tuning(timeout_ms=120000))
out["text"] = net.readback()
out["rw"] = rw.as_dict()
other = hvm64.Book.from_str("@main = a & @f ~ (1 a)\n@f = (a a)")
out["other_compiled"] = other.is_compiled()
n2 = hvm64.Net(other, heap_bytes=1 << 28)
n2.boot("main")
n2.normal()
out["other_text"] = n2.readback()
print(json.dumps(out))
"""


def _run_compiled(text):
    import build
    lib = build.build_compiled(_source(text))
    env = dict(os.environ, HVM64_LIB=lib)
    p = subprocess.run([sys.executable, "-c", GPU_SCRIPT, json.dumps({"text": text})], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


@pytest.mark.gpu
# (each case builds a library: about 40 s of nvcc on the GPU machine when absent)
@pytest.mark.parametrize("name", ["examples::sort::bitonic::bitonic_sort_lam", "tests::programs::numeric_casts",
                                  "tests::programs::dec_bits"])
def test_compiled_library_matches_snapshot(name):
    prog = PROGRAMS[name]
    got = _run_compiled(prog["source"])
    assert got["compiled"] is True
    assert got["text"] == prog["text"]
    assert got["rw"] == {k: prog[k] for k in KEYS}
    assert got["other_compiled"] is False and got["other_text"] == "1"


@pytest.mark.gpu
def test_compiled_bitonic_matches_oracle():
    import workloads as W
    from oracle import oracle
    text = W.bitonic(12, 5)
    want, want_rw, _ = oracle.run_book(text, mode=oracle.MODE_PARALLEL, threads=8)
    got = _run_compiled(text)
    assert got["compiled"] is True
    assert got["text"] == want
    assert got["rw"] == want_rw
