"""ctypes binding for the CPU oracle (oracle.cpp).  TEST INFRASTRUCTURE ONLY:
imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
never by the product.

The oracle restates the reference evaluator (HigherOrderCO/hvm-64) and is
pinned against the reference's own snapshots by tests/test_oracle.py.
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "build")
LIB = os.path.join(BUILD, "liboracle.so")
CLI = os.path.join(BUILD, "hvm64-oracle")

MODE_NORMAL = 0      # Net::normal (runtime/src/net.rs:55-60)
MODE_PARALLEL = 1    # Net::parallel_normal (runtime/src/parallel.rs:35-160)
MODE_FIFO = 2        # normal() popping redexes first-in-first-out
MODE_RANDOM = 3      # normal() popping redexes in seeded random order


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not (os.path.exists(LIB) and os.path.exists(CLI)):
            build()
        L = ctypes.CDLL(LIB)
        c = ctypes
        L.hvo_last_error.restype = c.c_char_p
        L.hvo_free.argtypes = [c.c_void_p]
        L.hvo_run_book.argtypes = [c.c_char_p, c.c_char_p, c.c_int, c.c_int, c.c_uint64, c.c_uint64, c.c_int,
                                   c.POINTER(c.c_void_p), c.POINTER(c.c_uint64), c.POINTER(c.c_double)]
        L.hvo_run_expr.argtypes = [c.c_char_p, c.c_char_p, c.c_int, c.c_int, c.c_uint64, c.c_int,
                                   c.POINTER(c.c_void_p), c.POINTER(c.c_uint64)]
        L.hvo_eval_with_args.argtypes = [c.c_char_p, c.c_char_p, c.c_uint64, c.POINTER(c.c_void_p)]
        L.hvo_label_sets.argtypes = [c.c_char_p, c.POINTER(c.c_void_p)]
        L.hvo_book_apply.argtypes = [c.c_char_p, c.c_char_p, c.c_char_p, c.POINTER(c.c_void_p)]
        L.hvo_book_roundtrip.argtypes = [c.c_char_p, c.POINTER(c.c_void_p)]
        L.hvo_num_binary.argtypes = [c.c_uint32, c.c_uint32, c.c_uint32, c.POINTER(c.c_uint32)]
        L.hvo_num_unary.argtypes = [c.c_uint32, c.c_uint32]
        L.hvo_num_unary.restype = c.c_uint32
        L.hvo_num_parse.argtypes = [c.c_char_p, c.POINTER(c.c_uint32)]
        L.hvo_num_print.argtypes = [c.c_uint32, c.POINTER(c.c_void_p)]
        L.hvo_num_f24.argtypes = [c.c_float]
        L.hvo_num_f24.restype = c.c_uint32
        L.hvo_pre_reduce.argtypes = [c.c_char_p, c.c_char_p, c.c_uint64, c.c_uint64, c.POINTER(c.c_void_p),
                                     c.POINTER(c.c_uint64), c.POINTER(c.c_void_p)]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


def _take(ptr):
    s = ctypes.cast(ptr, ctypes.c_char_p).value.decode()
    lib().hvo_free(ptr)
    return s


def _check(rc):
    if rc != 0:
        raise OracleError(rc, lib().hvo_last_error().decode())


COUNT_KEYS = ("anni", "comm", "eras", "dref", "oper")


def run_book(text, entry="main", mode=MODE_NORMAL, threads=0, seed=7, heap_bytes=0, resolve=True):
    """Boot `entry` and normalise (tests/tests.rs:28-35).  Returns
    (normal-form text, {anni, comm, eras, dref, oper}, seconds)."""
    out = ctypes.c_void_p()
    rw = (ctypes.c_uint64 * 5)()
    sec = ctypes.c_double()
    _check(lib().hvo_run_book(text.encode(), entry.encode(), mode, threads, seed, heap_bytes, int(resolve),
                              ctypes.byref(out), rw, ctypes.byref(sec)))
    return _take(out), dict(zip(COUNT_KEYS, list(rw))), sec.value


def pre_reduce(text, skip=("main",), max_rwts=(1 << 64) - 1, heap_bytes=0):
    """Book::pre_reduce (transform/src/pre_reduce.rs:27-74) with the names in
    `skip` left as they are.  Returns (pre-reduced Book text, {anni, comm,
    eras, dref, oper}, names of defs that stopped at max_rwts)."""
    out, nn = ctypes.c_void_p(), ctypes.c_void_p()
    rw = (ctypes.c_uint64 * 5)()
    _check(lib().hvo_pre_reduce(text.encode(), "\n".join(skip).encode(), max_rwts, heap_bytes, ctypes.byref(out),
                                rw, ctypes.byref(nn)))
    return _take(out), dict(zip(COUNT_KEYS, rw)), [n for n in _take(nn).split("\n") if n]


def run_expr(book_text, expr, mode=MODE_NORMAL, threads=0, heap_bytes=0):
    out = ctypes.c_void_p()
    rw = (ctypes.c_uint64 * 5)()
    _check(lib().hvo_run_expr(book_text.encode(), expr.encode(), mode, threads, heap_bytes, 1,
                              ctypes.byref(out), rw))
    return _take(out), dict(zip(COUNT_KEYS, list(rw)))


def eval_with_args(fun, args, heap_bytes=0):
    out = ctypes.c_void_p()
    _check(lib().hvo_eval_with_args(fun.encode(), "\n".join(args).encode(), heap_bytes, ctypes.byref(out)))
    return _take(out)


def label_sets(text):
    out = ctypes.c_void_p()
    _check(lib().hvo_label_sets(text.encode(), ctypes.byref(out)))
    res = {}
    for ln in _take(out).strip().split("\n"):
        parts = ln.split()
        res[parts[0]] = (int(parts[1]), [int(x) for x in parts[2:]])
    return res


def book_apply(text, def_name, arg_tree):
    out = ctypes.c_void_p()
    _check(lib().hvo_book_apply(text.encode(), def_name.encode(), arg_tree.encode(), ctypes.byref(out)))
    return _take(out)


def book_roundtrip(text):
    out = ctypes.c_void_p()
    _check(lib().hvo_book_roundtrip(text.encode(), ctypes.byref(out)))
    return _take(out)


def num_binary(a, op, b):
    out = ctypes.c_uint32()
    _check(lib().hvo_num_binary(a, op, b, ctypes.byref(out)))
    return out.value


def num_unary(op, a):
    return lib().hvo_num_unary(op, a)


def num_parse(text):
    out = ctypes.c_uint32()
    _check(lib().hvo_num_parse(text.encode(), ctypes.byref(out)))
    return out.value


def num_print(raw):
    out = ctypes.c_void_p()
    _check(lib().hvo_num_print(raw, ctypes.byref(out)))
    return _take(out)


def num_f24(v):
    return lib().hvo_num_f24(v)
