"""The C ABI without a GPU: the library loads, exports every function that
include/hvm64.h declares, parses Books on the host, and fails loudly (a
status code, not a crash and not a CPU fallback) when asked for device work
with no GPU present."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hvm64.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hvm64_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_python_exports():
    import hvm64
    assert sorted(hvm64.EXPORTS) == declared()


def test_library_exports_every_declared_symbol():
    import hvm64
    lib = hvm64.lib()
    for name in declared():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.hvm64_version()


def test_book_load_on_host():
    import hvm64
    book = hvm64.Book.from_str("@main = x & @id ~ (x *)\n@id = (a a)\n")
    assert sorted(book.names()) == ["id", "main"]
    with pytest.raises(hvm64.HvmError) as e:
        hvm64.Book.from_str("@main = (a")
    assert e.value.code == hvm64.ERR_BAD_INPUT


def test_rewrites_display_matches_reference_format():
    import hvm64
    rw = hvm64.Rewrites(anni=1234567, comm=2, eras=0, dref=30, oper=4000)
    lines = str(rw).splitlines()
    assert lines[0] == "RWTS   :       1_238_599"
    assert lines[1] == "- ANNI :       1_234_567"
    assert lines[5] == "- OPER :           4_000"


def test_device_work_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import hvm64
    book = hvm64.Book.from_str("@main = *\n")
    with pytest.raises(hvm64.HvmError) as e:
        hvm64.Net(book, 1 << 20)
    assert e.value.code == hvm64.ERR_CUDA
