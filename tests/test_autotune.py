"""The autotuner's search (CPU) and its use on a small batch (GPU)."""
import pytest


def test_coordinate_search_finds_the_best_setting():
    import autotune
    space = {"a": (0, 1, 2, 3), "b": (0, 10, 20)}
    cost = {0: 5.0, 1: 3.0, 2: 1.0, 3: 4.0}
    calls = []

    def measure(s):
        calls.append(dict(s))
        if s["b"] == 20:
            return None  # a setting that fails is skipped
        return cost[s["a"]] + (0.5 if s["b"] == 0 else 0.0)

    best, t, trials = autotune.coordinate_search(measure, space=space, order=("a", "b"))
    assert best == {"a": 2, "b": 10}
    assert t == 1.0
    assert len(trials) == len(calls) == 1 + 3 + 2


def test_coordinate_search_rejects_failing_defaults():
    import autotune
    with pytest.raises(RuntimeError):
        autotune.coordinate_search(lambda s: None, space={"a": (0, 1)}, order=("a",))


@pytest.mark.gpu
def test_autotune_on_a_batch_keeps_results():
    import hvm64
    import autotune
    import workloads as W
    entries = W.batch_entries(64, 4, 9, seed=9)
    book = hvm64.Book.from_str(W.batch_book(entries))
    names = [f"main_{j}" for _, _, j in entries]
    tune, report = autotune.autotune(book, names, heap_bytes=1 << 30, sample=32, timeout_ms=60000)
    assert report["trials"] >= 1 and report["sample_gips"] > 0
    b = hvm64.Batch(book, names, 1 << 30)
    b.normal(hvm64.PERSISTENT, tune)
    for i, (kind, d, j) in enumerate(entries):
        assert W.check_result(kind, d, j, b.readback(i))
