"""hvm64_net_normal_noalloc: normalisation for callers that cannot allocate
device memory (a caching allocator or pool already owns it, a fixed device
memory budget, a request loop that must not pay cudaMalloc's latency and
device-wide synchronisation).  The entry point runs out of one array built
into the library, so it is checked here against the allocating entry point
(hvm64_net_create + boot + normal + readback) on the same nets, twice in a
row, since each call reuses what the previous one left in that array.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""
import pytest

import workloads as W


def _hvm():
    import hvm64
    return hvm64


def _radix(keys_log2):
    import json
    import os
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "programs.json")
    src = next(p for p in json.load(open(gold)) if p["name"] == "examples::sort::radix::radix_sort_ctr")["source"]
    out = src.replace("& @gen ~ (20 (0 d))", f"& @gen ~ ({keys_log2} (0 d))")
    assert out != src
    return out


CASES = [
    ("tree_sum_10", lambda: W.tree_sum(10, 4)),
    ("bitonic_8", lambda: W.bitonic(8, 5)),
    ("church_4", lambda: W.church(4)),
    # wide nets: their work spreads over every warp of the grid, so every
    # lane's allocator chunk is taken at once
    ("tree_sum_16", lambda: W.tree_sum(16, 6)),
    ("bitonic_12", lambda: W.bitonic(12, 7)),
    # Def calls that push about 60 redexes each: the warps' overflow stacks
    # and the queue take the bursts
    ("radix_2^12", lambda: _radix(12)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_allocating_entry_point(case):
    hvm64 = _hvm()
    text = case[1]()
    book = hvm64.Book.from_str(text)
    tune = hvm64.Tuning(timeout_ms=60000)
    want_text, want_rw = hvm64.run_book(text, heap_bytes=1 << 30, tuning=tune)
    for _ in range(2):  # two calls in a row share the built-in array
        got_text, got_rw = hvm64.normal_noalloc(book, "main", tune)
        assert got_text == want_text
        assert got_rw.as_dict() == want_rw


@pytest.mark.gpu
def test_noalloc_alternating_books():
    """Two different Books one after the other, then the first again: each
    call resets what it reads, so no result depends on the previous call."""
    hvm64 = _hvm()
    texts = [W.tree_sum(9, 1), W.bitonic(7, 2)]
    books = [hvm64.Book.from_str(t) for t in texts]
    want = [hvm64.run_book(t, heap_bytes=1 << 28) for t in texts]
    for k in (0, 1, 0, 1):
        got_text, got_rw = hvm64.normal_noalloc(books[k])
        assert (got_text, got_rw.as_dict()) == want[k]


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_limits():
    hvm64 = _hvm()
    book = hvm64.Book.from_str(W.tree_sum(6, 0))
    with pytest.raises(hvm64.HvmError) as e:
        hvm64.normal_noalloc(book, "main", hvm64.Tuning(queue_slots_log2=16))
    assert e.value.code == hvm64.ERR_BAD_INPUT and "queue_slots_log2" in str(e.value)
    # a Book whose device tables exceed the 4 MiB region: one Def holding a
    # literal tree of 2^18 numbers (one instruction per node)
    def tree(d, k=[0]):
        if d == 0:
            k[0] += 1
            return str(k[0] & 0xFFFF)
        return f"({tree(d - 1)} {tree(d - 1)})"
    big = hvm64.Book.from_str(f"@main = {tree(18)}\n")
    with pytest.raises(hvm64.HvmError) as e:
        hvm64.normal_noalloc(big, "main")
    assert e.value.code == hvm64.ERR_BAD_INPUT and "too large" in str(e.value)
    # a Def needing more registers than a thread's local register file (the
    # allocating entry points give it a register file in device memory)
    wide = hvm64.Book.from_str("@main = (" + "".join(f"(x{i} " for i in range(60)) + "*" + ")" * 60 + " "
                               + "".join(f"(x{i} " for i in reversed(range(60))) + "*" + ")" * 60 + ")\n")
    with pytest.raises(hvm64.HvmError) as e:
        hvm64.normal_noalloc(wide, "main")
    assert e.value.code == hvm64.ERR_BAD_INPUT and "registers" in str(e.value)
    # a net that outgrows the built-in heap (a generated tree of 2^22 leaves,
    # kept whole: far more than its 3.35 million nodes) stops with OOM, and
    # the next call works
    gen_only = W.tree_sum(22, 0).replace("@main = a\n& @sum ~ (b a)\n& @gen ~ (22 (0 b))",
                                         "@main = a\n& @gen ~ (22 (0 a))")
    assert "& @gen ~ (22 (0 a))" in gen_only
    with pytest.raises(hvm64.HvmError) as e:
        hvm64.normal_noalloc(hvm64.Book.from_str(gen_only), "main", hvm64.Tuning(timeout_ms=60000))
    assert e.value.code == hvm64.ERR_OOM
    text = W.tree_sum(8, 3)
    got_text, _ = hvm64.normal_noalloc(hvm64.Book.from_str(text))
    assert got_text == str(W.expected_sum(8, 3))
