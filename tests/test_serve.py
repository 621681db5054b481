"""The serving reducer (hvm64_server_*): requests admitted while others are
on the device give the same normal forms and counts as each request reduced
alone.  GPU tests."""
import time

import pytest

import workloads as W


def _hvm():
    import hvm64
    return hvm64


def _alone(hvm64, book, names):
    """Each request reduced by itself through the one-net entry points."""
    net = hvm64.Net(book, 2 << 30)
    out = {}
    for name in names:
        net.boot(name)
        rw = net.normal(hvm64.Tuning(timeout_ms=60000))
        out[name] = (net.readback(), rw.as_dict())
    del net
    return out


def _drain(sv, want, done, deadline):
    while len(done) < want and time.time() < deadline:
        for t in sv.poll():
            done[t] = sv.result(t)
        time.sleep(0.001)


@pytest.mark.gpu
def test_server_mix_matches_alone():
    hvm64 = _hvm()
    reqs = W.serving_requests(48, seed=7, hi=3e6)
    book = hvm64.Book.from_str(W.serving_book(reqs))
    names = [f"main_{j}" for _, _, j in reqs]
    alone = _alone(hvm64, book, names)
    for (kind, param, j), name in zip(reqs, names):
        assert W.check_request(kind, param, j, alone[name][0]), name

    sv = hvm64.Server(book, slots=64, out_pairs=1 << 16, heap_bytes=4 << 30, tuning=hvm64.Tuning(timeout_ms=120000))
    try:
        tickets = {}
        done = {}
        # the first half goes in at once; the rest arrives while it runs
        for name in names[:24]:
            tickets[sv.submit(name)] = name
        for name in names[24:]:
            time.sleep(0.0005)
            for t in sv.poll():
                done[t] = sv.result(t)
            tickets[sv.submit(name)] = name
        _drain(sv, len(names), done, time.time() + 60)
    finally:
        sv.close()
    assert len(done) == len(names)
    for t, (text, rw, us) in done.items():
        name = tickets[t]
        assert text == alone[name][0], name
        assert rw.as_dict() == alone[name][1], name
        assert us > 0


@pytest.mark.gpu
def test_server_slots_and_reuse():
    """A full server refuses a request (HVM64_ERR_QUEUE); slots freed by
    collected results take new requests, many times over."""
    hvm64 = _hvm()
    reqs = [("sum", 8, j) for j in range(6)]
    book = hvm64.Book.from_str(W.serving_book(reqs))
    sv = hvm64.Server(book, slots=4, out_pairs=1 << 10, heap_bytes=1 << 30, tuning=hvm64.Tuning(timeout_ms=120000))
    try:
        owner = {sv.submit(f"main_{j}"): j for j in range(4)}
        with pytest.raises(hvm64.HvmError) as e:
            sv.submit("main_4")
        assert e.value.code == hvm64.ERR_QUEUE
        for round_ in range(10):
            got = {}
            _drain(sv, 4, got, time.time() + 20)
            assert len(got) == 4
            for t, (text, rw, us) in got.items():
                assert text == str(W.expected_sum(8, owner.pop(t)))
            for k in range(4):
                j = (round_ + k) % 6
                owner[sv.submit(f"main_{j}")] = j
        got = {}
        _drain(sv, 4, got, time.time() + 20)
        assert len(got) == 4
    finally:
        sv.close()


@pytest.mark.gpu
def test_server_error_stops_it_cleanly():
    """A request that divides by zero stops the whole server; poll reports
    the error, close returns, and the device stays usable."""
    hvm64 = _hvm()
    src = "@bad = x & 10 ~ $([/] $(0 x))\n@ok = x & 3 ~ $([*] $(5 x))\n"
    book = hvm64.Book.from_str(src)
    sv = hvm64.Server(book, slots=4, out_pairs=1 << 10, heap_bytes=1 << 30, tuning=hvm64.Tuning(timeout_ms=60000))
    try:
        sv.submit("bad")
        deadline = time.time() + 30
        with pytest.raises(hvm64.HvmError) as e:  # from poll, or from the failed request's result
            while time.time() < deadline:
                for t in sv.poll():
                    sv.result(t)
                time.sleep(0.001)
        assert e.value.code == hvm64.ERR_DIV0
    finally:
        sv.close()
    got, _ = hvm64.run_book(src.replace("@ok", "@main"), heap_bytes=1 << 24)
    assert got == "15"


@pytest.mark.gpu
def test_server_long_run_heap_stays_bounded():
    """600 bitonic-sort requests (2^12 keys each; about 12,000 nodes of
    normal form per request) through one server, 32 at a time, each admitted
    against the node budget: every result is right, the reservation returns
    to zero, and once half the heap is in use (the point from which free
    nodes move between warps; a 1 GiB heap reaches it in the first half of
    the run) the heap's high-water mark stops growing: the last 300 requests
    add far less than the 3.6 million nodes their normal forms alone would
    hold if finished requests' nodes were not recycled."""
    hvm64 = _hvm()
    reqs = [("sort", 12, j) for j in range(8)]
    book = hvm64.Book.from_str(W.serving_book(reqs))
    sv = hvm64.Server(book, slots=32, out_pairs=1 << 18, heap_bytes=1 << 30,
                      tuning=hvm64.Tuning(timeout_ms=300000))
    try:
        owner, done, submitted, high = {}, 0, 0, {}
        per_req = 200_000
        deadline = time.time() + 240
        while done < 600 and time.time() < deadline:
            while submitted < 600:
                try:
                    t = sv.submit(f"main_{submitted % 8}", nodes=per_req)
                except hvm64.HvmError as e:
                    assert e.code == hvm64.ERR_QUEUE
                    break
                owner[t] = submitted % 8
                submitted += 1
            for t in sv.poll():
                text, rw, us = sv.result(t)
                j = owner.pop(t)
                assert W.leaves(text) == sorted(W.sort_keys(12, j))
                done += 1
                if done in (300, 600):
                    high[done] = sv.budget()["heap_high"]
            time.sleep(0.001)
        assert done == 600
        b = sv.budget()
        assert b["reserved"] == 0
        assert high[600] - high[300] < 2_000_000, (high, b)
    finally:
        sv.close()


@pytest.mark.gpu
def test_server_admits_by_node_budget():
    """With slots to spare, requests are admitted only while their declared
    node needs fit the free budget: the third of three requests that each
    hold 40% of the budget is refused until a result is collected, and a
    request larger than the whole budget is refused outright."""
    hvm64 = _hvm()
    reqs = [("sum", 10, j) for j in range(4)]
    book = hvm64.Book.from_str(W.serving_book(reqs))
    sv = hvm64.Server(book, slots=16, out_pairs=1 << 10, heap_bytes=1 << 30, tuning=hvm64.Tuning(timeout_ms=120000))
    try:
        budget = sv.budget()["budget"]
        big = int(budget * 0.4)
        owner = {sv.submit("main_0", nodes=big): 0, sv.submit("main_1", nodes=big): 1}
        assert sv.budget()["reserved"] == 2 * big
        with pytest.raises(hvm64.HvmError) as e:
            sv.submit("main_2", nodes=big)
        assert e.value.code == hvm64.ERR_QUEUE and "budget" in str(e.value)
        with pytest.raises(hvm64.HvmError) as e:
            sv.submit("main_3", nodes=budget + 1)
        assert e.value.code == hvm64.ERR_BAD_INPUT
        got = {}
        _drain(sv, 1, got, time.time() + 30)
        for t, (text, rw, us) in got.items():
            assert text == str(W.expected_sum(10, owner.pop(t)))
        owner[sv.submit("main_2", nodes=big)] = 2
        got = {}
        _drain(sv, 2, got, time.time() + 30)
        for t, (text, rw, us) in got.items():
            assert text == str(W.expected_sum(10, owner.pop(t)))
        assert sv.budget()["reserved"] == 0
    finally:
        sv.close()


@pytest.mark.gpu
def test_server_holds_its_device():
    """A running server holds its device's launch parameters: a reduction
    started from the server's own thread on that device is refused (it could
    only wait for itself) instead of hanging, and works once the server is
    freed."""
    hvm64 = _hvm()
    src = "@main = x & 3 ~ $([*] $(5 x))\n"
    sv = hvm64.Server(hvm64.Book.from_str(src), slots=4, out_pairs=1 << 10, heap_bytes=1 << 30,
                      tuning=hvm64.Tuning(timeout_ms=60000))
    try:
        with pytest.raises(hvm64.HvmError) as e:
            hvm64.run_book(src, heap_bytes=1 << 24)
        assert e.value.code == hvm64.ERR_BAD_INPUT and "server" in str(e.value)
    finally:
        sv.close()
    got, _ = hvm64.run_book(src, heap_bytes=1 << 24)
    assert got == "15"
