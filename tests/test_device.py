"""Parity of the CUDA reducer against the oracle and the reference's golden
vectors, through the C ABI.  GPU tests are marked `gpu`."""
import json
import os

import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PROGRAMS = json.load(open(os.path.join(GOLD, "programs.json")))
DEVICE_LIMIT = 50_000_000  # interactions; bigger fixtures run under HVM64_SLOW=1


def _hvm():
    import hvm64
    return hvm64


def prog_params(limit):
    out = []
    for p in PROGRAMS:
        marks = [pytest.mark.gpu] + ([pytest.mark.slow] if p["total"] > limit else [])
        out.append(pytest.param(p, id=p["name"], marks=marks))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prog", prog_params(DEVICE_LIMIT))
def test_device_snapshot(prog):
    """Normal form and all five per-rule counts equal the reference snapshot."""
    hvm64 = _hvm()
    t = hvm64.Tuning(timeout_ms=60000)
    text, rw = hvm64.run_book(prog["source"], heap_bytes=1 << 30, tuning=t)
    assert text == prog["text"]
    assert rw == {k: prog[k] for k in ("anni", "comm", "eras", "dref", "oper")}
