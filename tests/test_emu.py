"""The device runtime (hvm-64_b200/csrc/device.cuh) compiled for the host and
run on many threads with random jitter in its memory operations: the link /
redirect protocol, the allocator (with free-node batches published to the
shared stack after every 4 nodes) and the instruction VM must give the
reference's normal forms and counts under contention.  CPU-only."""
import ctypes
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO = os.path.join(HERE, "emu", "libhvm64_emu.so")
SRC = [os.path.join(HERE, "emu", "emu.cpp"), os.path.join(ROOT, "hvm-64_b200", "csrc", "host.cpp")]
DEPS = SRC + [os.path.join(ROOT, "hvm-64_b200", "csrc", f) for f in ("device.cuh", "host.hpp", "num.h")]
PROGRAMS = json.load(open(os.path.join(HERE, "golden", "programs.json")))


def _lib():
    if not os.path.exists(SO) or any(os.path.getmtime(d) > os.path.getmtime(SO) for d in DEPS):
        subprocess.run(["g++", "-std=c++20", "-O2", "-pthread", "-fPIC", "-shared", "-DHVM_EMU_STRESS",
                        "-DHVM_OVF_FLUSH=4",
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "hvm-64_b200", "csrc"),
                        *SRC, "-o", SO], check=True)
    L = ctypes.CDLL(SO)
    c = ctypes
    L.hvm64emu_run.argtypes = [c.c_char_p, c.c_char_p, c.c_uint, c.c_uint, c.c_uint, c.c_uint, c.c_uint64,
                               c.c_uint64, c.POINTER(c.c_char_p), c.POINTER(c.c_uint64), c.c_char_p, c.c_size_t]
    return L


def emu_run(text, threads=16, ring=2, spill=24, heap=256 << 20, chunk=32):
    """Reduce `text`'s @main on `threads` host threads.  A step may push into
    at most `ring` stack slots; the rest go to a `spill`-redex overflow stack
    and, past that, to the shared queue."""
    L = _lib()
    out = ctypes.c_char_p()
    rw = (ctypes.c_uint64 * 5)()
    err = ctypes.create_string_buffer(256)
    rc = L.hvm64emu_run(text.encode(), b"main", threads, ring, spill, 16, heap, chunk, ctypes.byref(out), rw,
                        err, 256)
    assert rc == 0, err.value.decode()
    return out.value.decode(), dict(zip(("anni", "comm", "eras", "dref", "oper"), list(rw)))


@pytest.mark.parametrize("prog", [p for p in PROGRAMS if p["total"] <= 3_000_000], ids=lambda p: p["name"])
def test_emu_snapshot(prog):
    text, rw = emu_run(prog["source"])
    assert text == prog["text"]
    assert rw == {k: prog[k] for k in rw}


def test_emu_workloads():
    sys.path.insert(0, os.path.join(ROOT, "hvm-64_b200"))
    import workloads as W
    text, _ = emu_run(W.tree_sum(12, 3), threads=32)
    assert text == str(W.expected_sum(12, 3))
    text, _ = emu_run(W.bitonic(9, 4), threads=32)
    assert W.leaves(text) == sorted(W.sort_keys(9, 4))


def test_emu_deep_literal_def():
    """A Def whose literal tree is 300 levels deep on one side needs more live
    wires than the device register file in the reference's emission order;
    the encoder emits it smaller-child-first, with the same normal form and
    counts as the oracle's."""
    from oracle import oracle
    for left in (True, False):
        t = "*"
        for i in range(300):
            t = f"({t} {i % 7})" if left else f"({i % 7} {t})"
        src = f"@deep = {t}\n@main = x & @deep ~ x\n"
        want, want_rw, _ = oracle.run_book(src)
        text, rw = emu_run(src, threads=4)
        assert text == want
        assert rw == want_rw


@pytest.mark.parametrize("ring,spill", [(2, 24), (512, 64), (512, 0)])
def test_emu_radix_bursts(ring, spill):
    """The radix-sort fixture at 2^9 keys: each @radix call pushes about 60
    redexes at once, so the stack, the overflow stack and the shared queue
    all take pushes; normal form and counts equal the oracle's."""
    from oracle import oracle
    src = next(p for p in PROGRAMS if p["name"] == "examples::sort::radix::radix_sort_ctr")["source"]
    s = src.replace("& @gen ~ (20 (0 d))", "& @gen ~ (9 (0 d))")
    assert s != src
    want, want_rw, _ = oracle.run_book(s)
    text, rw = emu_run(s, threads=16, ring=ring, spill=spill)
    assert text == want
    assert rw == want_rw


def test_emu_def_with_many_live_wires():
    """A Def whose two halves each hold the same 120 variables needs more
    than 120 live wires in either emission order: more than a thread's local
    register file, so its calls use the warp's register file in device
    memory.  Normal form and counts equal the oracle's."""
    from oracle import oracle
    vs = [f"x{i}" for i in range(120)]

    def chain(names):
        t = "*"
        for v in reversed(names):
            t = f"({v} {t})"
        return t
    src = f"@wide = ({chain(vs)} {chain(vs[::-1])})\n@main = x & @wide ~ x\n"
    want, want_rw, _ = oracle.run_book(src)
    text, rw = emu_run(src, threads=4)
    assert text == want
    assert rw == want_rw


CHECK_SO = os.path.join(HERE, "emu", "build", "libhvm64_emu_check.so")


def _check_lib():
    """The emulation built with allocator bookkeeping (HVM_EMU_CHECK_ALLOC):
    every node handed out is marked, and handing out a marked node or
    reclaiming an unmarked one is counted and fails the run."""
    if not os.path.exists(CHECK_SO) or any(os.path.getmtime(d) > os.path.getmtime(CHECK_SO) for d in DEPS):
        os.makedirs(os.path.dirname(CHECK_SO), exist_ok=True)
        subprocess.run(["g++", "-std=c++20", "-O2", "-pthread", "-fPIC", "-shared", "-DHVM_EMU_STRESS",
                        "-DHVM_OVF_FLUSH=4", "-DHVM_EMU_CHECK_ALLOC",
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "hvm-64_b200", "csrc"),
                        *SRC, "-o", CHECK_SO], check=True)
    L = ctypes.CDLL(CHECK_SO)
    c = ctypes
    L.hvm64emu_run.argtypes = [c.c_char_p, c.c_char_p, c.c_uint, c.c_uint, c.c_uint, c.c_uint, c.c_uint64,
                               c.c_uint64, c.POINTER(c.c_char_p), c.POINTER(c.c_uint64), c.c_char_p, c.c_size_t]
    return L


@pytest.mark.parametrize("prog", [p for p in PROGRAMS if p["total"] <= 3_000_000], ids=lambda p: p["name"])
def test_emu_never_hands_out_a_node_twice(prog):
    """Under jittered contention (16 host threads, free lists published to
    the shared stack after 4 nodes, half the lanes without a reuse pool), no
    node is handed out while already out and none is reclaimed twice: the
    free / claim / recycle protocol and the shared free stack keep each node
    with one owner at a time."""
    L = _check_lib()
    out = ctypes.c_char_p()
    rw = (ctypes.c_uint64 * 5)()
    err = ctypes.create_string_buffer(256)
    rc = L.hvm64emu_run(prog["source"].encode(), b"main", 16, 2, 24, 16, 1 << 30, 32, ctypes.byref(out), rw, err, 256)
    assert rc == 0, err.value.decode()
    assert out.value.decode() == prog["text"]
