"""Parity of the CUDA reducer against the oracle and the reference's golden
vectors, through the C ABI.  GPU tests are marked `gpu`."""
import json
import os

import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PROGRAMS = json.load(open(os.path.join(GOLD, "programs.json")))
DEVICE_LIMIT = 50_000_000  # interactions; bigger fixtures get a 16 GiB heap and a 5-minute deadline
# Fixtures that keep only a handful of redexes alive at any time (tail loops,
# rotations, label-heavy Church towers).  The GPU reduces them at the latency
# of one chain of L2 round trips per interaction (about 0.1-1 M interactions/s),
# so at full size they run for many minutes; they are checked on the CPU
# emulation and at reduced sizes instead.  (apelacion, 1.5·10^9 interactions,
# is wide enough to run at about 13 M interactions/s: about two minutes.)
SEQUENTIAL = {
    "tests::programs::stress_tests::sum_tail",
    "tests::programs::stress_tests::tuple_rots",
    "tests::programs::stress_tests::boom",
    "tests::programs::stress_tests::burn",
}
LONG = {"tests::programs::stress_tests::apelacion"}  # given a 10-minute deadline


def _hvm():
    import hvm64
    return hvm64


def prog_params(limit):
    out = []
    for p in PROGRAMS:
        marks = [pytest.mark.gpu]
        if p["name"] in SEQUENTIAL and p["total"] > limit:
            marks += [pytest.mark.slow,
                      pytest.mark.skip(reason="sequential net: latency-bound on the GPU, runs for minutes")]
        out.append(pytest.param(p, id=p["name"], marks=marks))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prog", prog_params(DEVICE_LIMIT))
def test_device_snapshot(prog):
    """Normal form and all five per-rule counts equal the reference snapshot,
    for every fixture at its full size (the 2^20-key radix sorts included:
    1.4-1.5·10^9 interactions, Def calls that push about 60 redexes each)."""
    hvm64 = _hvm()
    big = prog["total"] > DEVICE_LIMIT
    t = hvm64.Tuning(timeout_ms=600000 if prog["name"] in LONG else 300000 if big else 60000)
    text, rw = hvm64.run_book(prog["source"], heap_bytes=(16 << 30) if big else (1 << 30), tuning=t)
    assert text == prog["text"]
    assert rw == {k: prog[k] for k in ("anni", "comm", "eras", "dref", "oper")}


# ---------------------------------------------------------------------------
# Workload families (tree-sum, bitonic sort, Church) against the oracle
# ---------------------------------------------------------------------------
def _oracle():
    from oracle import oracle
    return oracle


COUNTS = ("anni", "comm", "eras", "dref", "oper")


@pytest.mark.gpu
def test_batch_families_match_oracle():
    """A ragged batch of tree-sum and bitonic nets in one persistent launch:
    every net's normal form and counts equal the oracle's run of that net."""
    import workloads as W
    hvm64, oracle = _hvm(), _oracle()
    entries = W.batch_entries(24, 4, 10, seed=3)
    text = W.batch_book(entries)
    batch = hvm64.Batch(hvm64.Book.from_str(text), [f"main_{j}" for _, _, j in entries], 1 << 30)
    batch.normal(hvm64.PERSISTENT, hvm64.Tuning(timeout_ms=60000))
    for i, (kind, d, j) in enumerate(entries):
        want, want_rw, _ = oracle.run_book(text, entry=f"main_{j}")
        got = batch.readback(i)
        assert got == want, (kind, d, j)
        assert batch.rwts[i].as_dict() == want_rw, (kind, d, j)
        assert W.check_result(kind, d, j, got)


@pytest.mark.gpu
def test_plain_equals_persistent_and_repeats():
    """One-net-per-launch and persistent runs give the same forms and
    counts, and a second persistent run of the same batch repeats them."""
    import workloads as W
    hvm64 = _hvm()
    entries = W.batch_entries(12, 4, 9, seed=5)
    book = hvm64.Book.from_str(W.batch_book(entries))
    names = [f"main_{j}" for _, _, j in entries]
    runs = []
    for mode in (hvm64.PLAIN, hvm64.PERSISTENT, hvm64.PERSISTENT):
        b = hvm64.Batch(book, names, 1 << 30)
        b.normal(mode, hvm64.Tuning(timeout_ms=60000))
        runs.append([(b.readback(i), b.rwts[i].as_dict()) for i in range(b.n)])
    assert runs[0] == runs[1] == runs[2]


@pytest.mark.gpu
def test_graph_replay_equals_direct_launch():
    """A persistent batch captured as a CUDA graph and replayed gives the
    same forms and counts as the direct launches, on every replay."""
    import workloads as W
    hvm64 = _hvm()
    entries = W.batch_entries(16, 4, 9, seed=13)
    book = hvm64.Book.from_str(W.batch_book(entries))
    names = [f"main_{j}" for _, _, j in entries]
    b = hvm64.Batch(book, names, 1 << 30)
    b.normal(hvm64.PERSISTENT, hvm64.Tuning(timeout_ms=60000))
    want = [(b.readback(i), b.rwts[i].as_dict()) for i in range(b.n)]
    g = hvm64.Tuning(timeout_ms=60000, flags=hvm64.TUNE_GRAPH)
    for _ in range(3):
        b.normal(hvm64.PERSISTENT, g)
        assert [(b.readback(i), b.rwts[i].as_dict()) for i in range(b.n)] == want


@pytest.mark.gpu
def test_batch_expression_and_trivial_entries():
    """Entries may be expression nets ('=' prefix), nets with no redex at
    all, and Def boots, mixed in one batch."""
    hvm64, oracle = _hvm(), _oracle()
    src = "@two = (a (* a))\n@main = x & @two ~ (1 x)\n"
    exprs = ["main", "=*", "=(a a)", "=x & 3 ~ $([+] $(4 x))", "two", "main"]
    b = hvm64.Batch(hvm64.Book.from_str(src), exprs, 1 << 28)
    b.normal(hvm64.PERSISTENT, hvm64.Tuning(timeout_ms=20000))
    want_main, rw_main, _ = oracle.run_book(src, entry="main")
    assert b.readback(0) == want_main and b.rwts[0].as_dict() == rw_main
    assert b.readback(5) == want_main
    for i in (1, 2, 3):  # expression nets: Host::encode_net, no boot call
        want, want_rw = oracle.run_expr(src, exprs[i][1:])
        assert b.readback(i) == want and b.rwts[i].as_dict() == want_rw
    assert b.readback(1) == "*" and b.readback(2) == "(a a)" and b.readback(3) == "7"
    want_two, rw_two, _ = oracle.run_book(src, entry="two")
    assert b.readback(4) == want_two and b.rwts[4].as_dict() == rw_two


@pytest.mark.gpu
def test_tree_sum_depth18_full_size():
    """The tree-sum workload at its full size (262,144 leaves): normal form is
    the host-computed wrapping sum; counts equal the oracle's."""
    import workloads as W
    hvm64, oracle = _hvm(), _oracle()
    text = W.tree_sum(18, 0)
    got, rw = hvm64.run_book(text, heap_bytes=4 << 30, tuning=hvm64.Tuning(timeout_ms=60000))
    assert got == str(W.expected_sum(18, 0))
    _, want_rw, _ = oracle.run_book(text, mode=oracle.MODE_PARALLEL, threads=8)
    assert rw == want_rw


@pytest.mark.gpu
def test_repeated_runs_identical():
    """The same net reduced eight times on one heap (which keeps the previous
    run's words) gives the same normal form and counts every time: a check
    against scheduling-dependent races, which show up as occasional wrong
    results."""
    import workloads as W
    hvm64 = _hvm()
    text = W.tree_sum(18, 0)
    net = hvm64.Net(hvm64.Book.from_str(text), 4 << 30)
    seen = set()
    for _ in range(8):
        net.boot("main")
        rw = net.normal(hvm64.Tuning(timeout_ms=60000))
        seen.add((net.readback(), tuple(sorted(rw.as_dict().items()))))
    assert len(seen) == 1
    assert next(iter(seen))[0] == str(W.expected_sum(18, 0))


@pytest.mark.gpu
def test_bitonic_depth15_sorted():
    """Bitonic sort of 2^15 keys: the read-back leaves are the sorted input
    multiset (size-independent check), counts equal the oracle's."""
    import workloads as W
    hvm64, oracle = _hvm(), _oracle()
    text = W.bitonic(15, 2)
    got, rw = hvm64.run_book(text, heap_bytes=4 << 30, tuning=hvm64.Tuning(timeout_ms=120000))
    assert W.leaves(got) == sorted(W.sort_keys(15, 2))
    _, want_rw, _ = oracle.run_book(text, mode=oracle.MODE_PARALLEL, threads=8)
    assert rw == want_rw


@pytest.mark.gpu
def test_church_labels():
    """The label-heavy Church net (numeral 2 with one DUP label per copy,
    applied to itself 5 times, collapsed): normal form and counts equal the
    oracle's."""
    import workloads as W
    hvm64, oracle = _hvm(), _oracle()
    text = W.church(5)
    want, want_rw, _ = oracle.run_book(text)
    got, rw = hvm64.run_book(text, heap_bytes=1 << 30, tuning=hvm64.Tuning(timeout_ms=60000))
    assert got == want
    assert rw == want_rw


# ---------------------------------------------------------------------------
# Failure statuses: where the reference panics, the C ABI returns a code and
# the context stays usable.  None of these faults the GPU: each ends in the
# kernel's own checks (division, dispatch, allocator bound, run deadline).
# ---------------------------------------------------------------------------
ERROR_CASES = [
    ("div0", "@main = x & 10 ~ $([/] $(0 x))\n", "ERR_DIV0", 1 << 26, 20000),
    ("bad_pair", "@main = (a b) & ?(a b) ~ (c c)\n", "ERR_BAD_PAIR", 1 << 26, 20000),
    ("oom", None, "ERR_OOM", 1 << 16, 20000),
    ("timeout", "@L = (a b) & @L ~ (a b)\n@main = x & @L ~ (x *)\n", "ERR_TIMEOUT", 1 << 26, 300),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", ERROR_CASES, ids=[c[0] for c in ERROR_CASES])
def test_error_status(case):
    import workloads as W
    hvm64 = _hvm()
    name, src, code, heap, timeout = case
    if src is None:
        src = W.tree_sum(12, 0)
    net = hvm64.Net(hvm64.Book.from_str(src), heap)
    net.boot("main")
    with pytest.raises(hvm64.HvmError) as e:
        net.normal(hvm64.Tuning(timeout_ms=timeout))
    assert e.value.code == getattr(hvm64, code)
    # the device is still usable afterwards
    got, _ = hvm64.run_book("@main = x & 3 ~ $([*] $(5 x))\n", heap_bytes=1 << 24)
    assert got == "15"


@pytest.mark.gpu
def test_deep_normal_form_reads_back():
    """A normal form nested deeper than the device gather's stack (a
    left-nested tree of depth 300) is read back through the heap image
    instead, with the same text as the oracle's."""
    hvm64, oracle = _hvm(), _oracle()
    t = "*"
    for i in range(300):
        t = f"({t} {i % 7})"
    src = f"@deep = {t}\n@main = x & @deep ~ x\n"
    want, want_rw, _ = oracle.run_book(src)
    got, rw = hvm64.run_book(src, heap_bytes=1 << 28)
    assert got == want
    assert rw == want_rw


@pytest.mark.gpu
def test_radix_sort_reduced_sizes():
    """The radix-sort fixture at 2^12 and 2^16 keys: normal form and counts
    equal the oracle's."""
    hvm64, oracle = _hvm(), _oracle()
    src = next(p for p in PROGRAMS if p["name"] == "examples::sort::radix::radix_sort_ctr")["source"]
    for n in (12, 16):
        s = src.replace("& @gen ~ (20 (0 d))", f"& @gen ~ ({n} (0 d))")
        want, want_rw, _ = oracle.run_book(s, mode=oracle.MODE_PARALLEL, threads=8)
        got, rw = hvm64.run_book(s, heap_bytes=16 << 30, tuning=hvm64.Tuning(timeout_ms=60000))
        assert got == want
        assert rw == want_rw


@pytest.mark.gpu
def test_bitonic_depth20_full_size():
    """The single-net bitonic sort of 2^20 u24 keys (about 5% duplicates) at
    its full size, 8.9·10^9 interactions: the read-back leaves are the sorted
    key multiset, and all five counts equal the oracle's (precomputed by
    tests/golden/make_workload_counts.py, minutes of CPU time)."""
    import workloads as W
    hvm64 = _hvm()
    gold = json.load(open(os.path.join(GOLD, "workload_counts.json")))["bitonic_20_2"]
    got, rw = hvm64.run_book(W.bitonic(20, 2), heap_bytes=32 << 30, tuning=hvm64.Tuning(timeout_ms=300000))
    assert W.leaves(got) == sorted(W.sort_keys(20, 2))
    assert rw == gold["counts"]


@pytest.mark.gpu
def test_concurrent_handles_two_threads():
    """Two nets on one device, reduced from two host threads at the same
    time (ctypes releases the GIL around each C call): the runs take turns on
    the device's launch parameters, so both normal forms and all counts equal
    the oracle's, on every round."""
    import threading
    import workloads as W
    hvm64, oracle = _hvm(), _oracle()
    texts = [W.tree_sum(14, 1), W.bitonic(11, 3)]
    want = [oracle.run_book(t, mode=oracle.MODE_PARALLEL, threads=8)[:2] for t in texts]
    got = [[], []]
    errs = []

    def work(k):
        try:
            net = hvm64.Net(hvm64.Book.from_str(texts[k]), 1 << 30)
            for _ in range(4):
                net.boot("main")
                rw = net.normal(hvm64.Tuning(timeout_ms=60000))
                got[k].append((net.readback(), rw.as_dict()))
        except Exception as e:  # reported on the main thread
            errs.append(e)

    th = [threading.Thread(target=work, args=(k,)) for k in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for k in (0, 1):
        assert got[k] == [want[k]] * 4


@pytest.mark.gpu
def test_def_with_many_live_wires():
    """A Def needing more live wires than a thread's local register file (121
    in either emission order) runs through the warp's register file in device
    memory: normal form and counts equal the oracle's."""
    hvm64, oracle = _hvm(), _oracle()
    vs = [f"x{i}" for i in range(120)]

    def chain(names):
        t = "*"
        for v in reversed(names):
            t = f"({v} {t})"
        return t
    src = f"@wide = ({chain(vs)} {chain(vs[::-1])})\n@main = x & @wide ~ x\n"
    want, want_rw, _ = oracle.run_book(src)
    got, rw = hvm64.run_book(src, heap_bytes=1 << 28)
    assert got == want
    assert rw == want_rw
