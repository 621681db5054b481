"""Pins the CPU oracle against the reference's own golden vectors.

Fixtures come from tests/golden/make_golden.py (run against the reference
checkout): the run@*.snap snapshots (tests/tests.rs:28-42), tests/lists.rs,
tests/cli.rs and host/src/calc_labels.rs:196-234.
"""
import json
import os
import subprocess

import pytest

from oracle import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PROGRAMS = json.load(open(os.path.join(GOLD, "programs.json")))
LISTS = json.load(open(os.path.join(GOLD, "lists.json")))
CLI = json.load(open(os.path.join(GOLD, "cli.json")))
LABELS = json.load(open(os.path.join(GOLD, "labels.json")))

FAST_LIMIT = 5_000_000      # interactions; larger programs are marked slow
ORDER_LIMIT = 3_000_000


def counts(p):
    return {k: p[k] for k in oracle.COUNT_KEYS}


def prog_params(limit, slow_marks=True):
    out = []
    for p in PROGRAMS:
        marks = [pytest.mark.slow] if (p["total"] > limit and slow_marks) else []
        if p["total"] > limit and not slow_marks:
            continue
        out.append(pytest.param(p, id=p["name"], marks=marks))
    return out


@pytest.mark.parametrize("prog", prog_params(FAST_LIMIT))
def test_snapshot_normal(prog):
    """Net::normal reproduces the snapshot's normal form and all five counts."""
    text, rw, _ = oracle.run_book(prog["source"], mode=oracle.MODE_NORMAL)
    assert text == prog["text"]
    assert rw == counts(prog)


@pytest.mark.parametrize("prog", prog_params(ORDER_LIMIT, slow_marks=False))
@pytest.mark.parametrize("mode,threads", [(oracle.MODE_PARALLEL, 4), (oracle.MODE_PARALLEL, 8),
                                          (oracle.MODE_FIFO, 0), (oracle.MODE_RANDOM, 0)])
def test_snapshot_other_orders(prog, mode, threads):
    """parallel_normal and reordered normal() give identical forms and counts:
    the counts the device must match do not depend on reduction order."""
    text, rw, _ = oracle.run_book(prog["source"], mode=mode, threads=threads)
    assert text == prog["text"]
    assert rw == counts(prog)


def _list_book(kind, item):
    src = LISTS["source"]
    if kind == "got":
        book = oracle.book_apply(src, "GenGotIndex", f"@S{item['index']}")
        book = oracle.book_apply(book, "main", "@GenGotIndex")
    else:
        book = oracle.book_apply(src, "GenPutIndexValue", f"@S{item['index']}")
        book = oracle.book_apply(book, "GenPutIndexValue", f"@S{item['value']}")
        book = oracle.book_apply(book, "main", "@GenPutIndexValue")
    return book


@pytest.mark.parametrize("kind", ["got", "put"])
def test_lists(kind):
    """tests/lists.rs: RWTS totals and their linearity in the index."""
    totals = []
    for item in LISTS[kind]:
        _, rw, _ = oracle.run_book(_list_book(kind, item), mode=oracle.MODE_NORMAL)
        totals.append(sum(rw.values()))
        assert totals[-1] == item["total"]
    d = totals[1] - totals[0]
    for k in range(1, 5):
        assert totals[k] + d * 2 ** k == totals[k + 1]


@pytest.mark.parametrize("case", CLI["apply_tree"], ids=lambda c: f"{c['fun']}|{','.join(c['args'])}")
def test_cli_apply_tree(case):
    """tests/cli.rs:205-251 on a 16-word heap (Heap::new_exact(16))."""
    assert oracle.eval_with_args(case["fun"], case["args"], heap_bytes=16 * 8) == case["expect"]


def _cli_cases():
    out = []
    for c in CLI["runs"]:
        if c["args"][0] in ("reduce", "run"):
            out.append(pytest.param(c, id=" ".join(c["args"])))
    return out


@pytest.mark.parametrize("case", _cli_cases())
def test_cli_outputs(case, tmp_path):
    """tests/cli.rs:40-131,184-203: `run` / `reduce` stdout and errors."""
    oracle.lib()
    path = tmp_path / "arithmetic.hvm"
    path.write_text(CLI["arithmetic"])
    args = [str(path) if a == "{arithmetic}" else a for a in case["args"]]
    r = subprocess.run([oracle.CLI] + args, capture_output=True, text=True, cwd=tmp_path)
    assert (r.stdout + r.stderr).strip() == case["expect"]


def _labels_book():
    """The calc_labels unit test writes `{n a b}` for a combinator with label
    n (an older surface syntax); restate it with today's `#k(..)`/`#k{..}`
    (label = 2k + kind, ast/src/parser.rs:353)."""
    import re
    txt = LABELS["book"]

    def ctr(m):
        n = int(m.group(1))
        return f"#{n // 2}" + ("{" if n % 2 else "(")
    txt = re.sub(r"\{(\d+) ", ctr, txt)
    # closing brackets: rebuild by scanning the opened kinds
    out, stack = [], []
    for ch in txt:
        if ch in "({":
            stack.append(ch)
            out.append(ch)
        elif ch in ")}":
            o = stack.pop()
            out.append(")" if o == "(" else "}")
        else:
            out.append(ch)
    return "".join(out)


def test_calc_labels():
    sets = oracle.label_sets(_labels_book())
    for name, labs in LABELS["sets"].items():
        assert sets[name][1] == sorted(labs), name
        assert sets[name][0] == max(labs) + 1


def test_book_roundtrip():
    for p in PROGRAMS:
        once = oracle.book_roundtrip(p["source"])
        assert oracle.book_roundtrip(once) == once


# ---- num crate edge cases (num/src/num.rs) --------------------------------
ADD, SUB, MUL, DIV, REM, SHL, SHR, EQ, LT = 4, 5, 7, 8, 10, 15, 17, 19, 21


def test_num_u24():
    u = oracle.num_parse
    assert oracle.num_print(oracle.num_binary(u("0"), SUB, u("1"))) == "16777215"
    assert oracle.num_print(oracle.num_binary(u("16777215"), ADD, u("1"))) == "0"
    assert oracle.num_print(oracle.num_binary(u("16777215"), SHR, u("22"))) == "3"
    assert oracle.num_print(oracle.num_binary(u("1"), SHL, u("33"))) == "2"  # wrapping_shl masks by 31
    with pytest.raises(oracle.OracleError) as e:
        oracle.num_binary(u("1"), DIV, u("0"))
    assert e.value.code == 3


def test_num_i24_f24():
    u = oracle.num_parse
    assert oracle.num_print(oracle.num_binary(u("-8388608"), SUB, u("+1"))) == "+8388607"
    assert oracle.num_print(oracle.num_binary(u("-3"), REM, u("+2"))) == "-1"
    assert oracle.num_print(oracle.num_binary(u("0.5"), ADD, u("2.0"))) == "2.5"
    assert oracle.num_print(oracle.num_binary(u("0.5"), MUL, u("2.3"))) == "1.1499939"
    assert oracle.num_print(oracle.num_binary(u("0.0"), DIV, u("0.0"))) == "+NaN"
    assert oracle.num_print(u("[u24]")) == "[u24]"
    assert oracle.num_print(u("[*2]")) == "[*2]"
    # new_f24 rounds the low byte to nearest even (num.rs:81-90)
    import struct
    for bits, want in ((0x3F800080, 0x3F8000), (0x3F800180, 0x3F8002), (0x3F80007F, 0x3F8000),
                       (0x3F800081, 0x3F8001)):
        f = struct.unpack("<f", struct.pack("<I", bits))[0]
        assert oracle.num_f24(f) >> 8 == want
