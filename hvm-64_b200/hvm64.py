"""Python mirror of the reference's host API over the B200 reducer's C ABI.

    book = Book.from_str(text)          # ast::Book::from_str + Host::new
    net = Net(book)                     # Heap::new + Net::new
    net.boot("main")                    # Net::boot(&host.defs["main"])
    rwts = net.normal()                 # Net::normal / parallel_normal, on the GPU
    print(net.readback())               # Host::readback + Display
    print(rwts)                         # Rewrites (runtime/src/runtime.rs:131-141)

`Batch` reduces many nets in one persistent launch (or one launch per net with
mode=PLAIN).  Every call goes through include/hvm64.h; there is no CPU
fallback: without the CUDA library or a GPU the calls raise.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HVM64_LIB") or os.path.join(HERE, "build", "libhvm64.so")

OK, ERR_OOM, ERR_BAD_PAIR, ERR_DIV0, ERR_TIMEOUT, ERR_BAD_INPUT, ERR_CUDA, ERR_QUEUE, ERR_BAD_ADDR, ERR_OUTPUT, \
    ERR_LIMIT = range(11)
PERSISTENT, PLAIN = 0, 1
TUNE_GRAPH = 1  # Tuning.flags: persistent runs replay one captured CUDA graph

# Every symbol include/hvm64.h declares.
EXPORTS = (
    "hvm64_last_error", "hvm64_version", "hvm64_book_load", "hvm64_book_def_count", "hvm64_book_def_name",
    "hvm64_book_free", "hvm64_net_create", "hvm64_net_boot", "hvm64_net_encode", "hvm64_net_normal",
    "hvm64_net_readback", "hvm64_net_free", "hvm64_batch_create", "hvm64_batch_normal", "hvm64_batch_readback",
    "hvm64_batch_free", "hvm64_batch_stats", "hvm64_net_stats", "hvm64_net_normal_noalloc",
    "hvm64_batch_normal_range",
    "hvm64_server_create", "hvm64_server_submit", "hvm64_server_poll", "hvm64_server_result", "hvm64_server_free",
    "hvm64_server_submit_nodes", "hvm64_server_budget", "hvm64_pre_reduce", "hvm64_book_format",
    "hvm64_book_compile_source", "hvm64_book_is_compiled",
)


class HvmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hvm64 error {code}: {msg}")
        self.code = code


class Rewrites(ctypes.Structure):
    _fields_ = [("anni", ctypes.c_uint64), ("comm", ctypes.c_uint64), ("eras", ctypes.c_uint64),
                ("dref", ctypes.c_uint64), ("oper", ctypes.c_uint64)]

    def total(self):
        return self.anni + self.comm + self.eras + self.dref + self.oper

    def as_dict(self):
        return {k: getattr(self, k) for k in ("anni", "comm", "eras", "dref", "oper")}

    def __str__(self):  # runtime/src/runtime.rs:131-141
        def pretty(n):  # util/src/pretty_num.rs
            s = str(n)
            head = len(s) % 3
            parts = ([s[:head]] if head else []) + [s[i:i + 3] for i in range(head, len(s), 3)]
            return "_".join(parts)
        rows = [("RWTS   ", self.total()), ("- ANNI ", self.anni), ("- COMM ", self.comm), ("- ERAS ", self.eras),
                ("- DREF ", self.dref), ("- OPER ", self.oper)]
        return "".join(f"{k}: {pretty(v):>15}\n" for k, v in rows)


class Tuning(ctypes.Structure):
    _fields_ = [("blocks_per_sm", ctypes.c_uint32), ("chunk_nodes", ctypes.c_uint32),
                ("donate_min", ctypes.c_uint32), ("queue_slots_log2", ctypes.c_uint32),
                ("max_warps_per_net", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("timeout_ms", ctypes.c_uint64)]


class Stats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("comm22", "dref_nodes", "dref_links", "heap_nodes_used", "donated",
                                                "spilled", "overflowed", "h2d_bytes", "d2h_bytes", "steps",
                                                "step_lanes", "busy_cycles", "idle_cycles")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib(build_if_missing=True):
    """Loads build/libhvm64.so (building it first if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and build_if_missing:
        import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    c = ctypes
    P = c.c_void_p
    L.hvm64_last_error.restype = c.c_char_p
    L.hvm64_version.restype = c.c_char_p
    L.hvm64_book_load.argtypes = [c.c_char_p, c.c_size_t, c.POINTER(P)]
    L.hvm64_book_def_count.argtypes = [P]
    L.hvm64_book_def_count.restype = c.c_uint32
    L.hvm64_book_def_name.argtypes = [P, c.c_uint32]
    L.hvm64_book_def_name.restype = c.c_char_p
    L.hvm64_book_free.argtypes = [P]
    L.hvm64_net_create.argtypes = [P, c.c_uint64, c.POINTER(P)]
    L.hvm64_net_boot.argtypes = [P, c.c_char_p]
    L.hvm64_net_encode.argtypes = [P, c.c_char_p, c.c_size_t]
    L.hvm64_net_normal.argtypes = [P, c.POINTER(Tuning), c.POINTER(Rewrites), c.POINTER(c.c_double)]
    L.hvm64_net_readback.argtypes = [P, c.c_char_p, c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_net_free.argtypes = [P]
    L.hvm64_batch_create.argtypes = [P, c.c_uint32, c.POINTER(c.c_char_p), c.c_uint64, c.POINTER(P)]
    L.hvm64_batch_normal.argtypes = [P, c.c_int, c.POINTER(Tuning), c.POINTER(Rewrites), c.POINTER(c.c_int),
                                     c.POINTER(c.c_double)]
    L.hvm64_batch_normal_range.argtypes = [P, c.c_int, c.POINTER(Tuning), c.c_uint32, c.c_uint32,
                                           c.c_void_p, c.c_void_p, c.POINTER(c.c_double)]
    L.hvm64_batch_readback.argtypes = [P, c.c_uint32, c.c_char_p, c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_batch_free.argtypes = [P]
    L.hvm64_batch_stats.argtypes = [P, c.POINTER(Stats)]
    L.hvm64_net_stats.argtypes = [P, c.POINTER(Stats)]
    L.hvm64_net_normal_noalloc.argtypes = [P, c.c_char_p, c.POINTER(Tuning), c.POINTER(Rewrites), c.c_char_p,
                                           c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_server_create.argtypes = [P, c.c_uint64, c.c_uint32, c.c_uint32, c.POINTER(Tuning), c.POINTER(P)]
    L.hvm64_server_submit.argtypes = [P, c.c_char_p, c.POINTER(c.c_uint64)]
    L.hvm64_server_submit_nodes.argtypes = [P, c.c_char_p, c.c_uint64, c.POINTER(c.c_uint64)]
    L.hvm64_server_budget.argtypes = [P, c.POINTER(c.c_uint64), c.POINTER(c.c_uint64), c.POINTER(c.c_uint64)]
    L.hvm64_server_poll.argtypes = [P, c.POINTER(c.c_uint64), c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_server_result.argtypes = [P, c.c_uint64, c.POINTER(Rewrites), c.POINTER(c.c_int),
                                      c.POINTER(c.c_double), c.c_char_p, c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_server_free.argtypes = [P]
    L.hvm64_pre_reduce.argtypes = [c.c_char_p, c.c_size_t, c.c_char_p, c.c_uint64, c.c_uint64, c.POINTER(Tuning),
                                   c.POINTER(Rewrites), c.c_char_p, c.c_size_t, c.POINTER(c.c_size_t), c.c_char_p,
                                   c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_book_format.argtypes = [c.c_char_p, c.c_size_t, c.c_char_p, c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_book_compile_source.argtypes = [P, c.c_char_p, c.c_size_t, c.POINTER(c.c_size_t)]
    L.hvm64_book_is_compiled.argtypes = [P]
    _lib = L
    return L


def _check(rc):
    if rc != OK:
        raise HvmError(rc, lib().hvm64_last_error().decode())


def _read_text(fn, *args):
    n = ctypes.c_size_t()
    _check(fn(*args, None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    _check(fn(*args, buf, n.value + 1, ctypes.byref(n)))
    return buf.value.decode()


class Book:
    """A loaded `.hvm` Book (ast::Book + host::Host)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_str(cls, text):
        h = ctypes.c_void_p()
        data = text.encode()
        _check(lib().hvm64_book_load(data, len(data), ctypes.byref(h)))
        return cls(h)

    def compile_source(self):
        """CUDA source of this Book's Defs as straight-line device functions
        (the analogue of `hvm64 compile`); build.build_compiled turns it into
        a library."""
        return _read_text(lib().hvm64_book_compile_source, self._h)

    def is_compiled(self):
        """True when the loaded library runs compiled functions for this Book."""
        return bool(lib().hvm64_book_is_compiled(self._h))

    def names(self):
        L = lib()
        return [L.hvm64_book_def_name(self._h, i).decode() for i in range(L.hvm64_book_def_count(self._h))]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.hvm64_book_free(self._h)
            self._h = None


class Net:
    """One net on the device (runtime::Net)."""

    def __init__(self, book, heap_bytes=0):
        self.book = book
        h = ctypes.c_void_p()
        _check(lib().hvm64_net_create(book._h, heap_bytes, ctypes.byref(h)))
        self._h = h
        self.rwts = Rewrites()
        self.device_ms = 0.0

    def boot(self, name="main"):
        _check(lib().hvm64_net_boot(self._h, name.encode()))

    def encode(self, net_text):
        data = net_text.encode()
        _check(lib().hvm64_net_encode(self._h, data, len(data)))

    def normal(self, tuning=None):
        ms = ctypes.c_double()
        t = ctypes.byref(tuning) if tuning is not None else None
        _check(lib().hvm64_net_normal(self._h, t, ctypes.byref(self.rwts), ctypes.byref(ms)))
        self.device_ms = ms.value
        return self.rwts

    def readback(self):
        return _read_text(lib().hvm64_net_readback, self._h)

    def stats(self):
        st = Stats()
        _check(lib().hvm64_net_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.hvm64_net_free(self._h)
            self._h = None


class Batch:
    """Many independent nets reduced together.  Each entry is a Def name
    (booted) or '=' followed by an expression net (encoded)."""

    def __init__(self, book, entries, heap_bytes=0):
        self.book = book
        self.n = len(entries)
        arr = (ctypes.c_char_p * self.n)(*[e.encode() for e in entries])
        h = ctypes.c_void_p()
        _check(lib().hvm64_batch_create(book._h, self.n, arr, heap_bytes, ctypes.byref(h)))
        self._h = h
        self.rwts = (Rewrites * self.n)()
        self.status = (ctypes.c_int * self.n)()
        self.device_ms = 0.0

    def normal(self, mode=PERSISTENT, tuning=None, check=True, first=0, count=None):
        """Reduce every net, or only nets [first, first + count) (one launch;
        only those can be read back afterwards).  self.rwts[i] and
        self.status[i] hold net i's results."""
        ms = ctypes.c_double()
        t = ctypes.byref(tuning) if tuning is not None else None
        if count is None:
            count = self.n - first
        rsz, isz = ctypes.sizeof(Rewrites), ctypes.sizeof(ctypes.c_int)
        per_net = ctypes.addressof(self.rwts) + first * rsz
        status = ctypes.addressof(self.status) + first * isz
        rc = lib().hvm64_batch_normal_range(self._h, mode, t, first, count, per_net, status, ctypes.byref(ms))
        self.device_ms = ms.value
        if check:
            _check(rc)
        return rc

    def readback(self, i):
        return _read_text(lib().hvm64_batch_readback, self._h, i)

    def stats(self):
        st = Stats()
        _check(lib().hvm64_batch_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.hvm64_batch_free(self._h)
            self._h = None


class Server:
    """A reducer that stays on the device and admits requests while it runs.
    `submit(name, nodes=0)` boots Def `name` when a slot and `nodes` of the
    node budget are free (ERR_QUEUE otherwise) and returns a ticket; `poll()`
    lists finished tickets; `result(ticket)` returns (text, Rewrites,
    device_us); `budget()` the node budget, its reserved part and the heap's
    high-water mark.  `close()` stops the reducer at once."""

    def __init__(self, book, slots=256, out_pairs=1 << 16, heap_bytes=0, tuning=None):
        self.book = book
        self.slots = slots
        h = ctypes.c_void_p()
        t = ctypes.byref(tuning) if tuning is not None else None
        _check(lib().hvm64_server_create(book._h, heap_bytes, slots, out_pairs, t, ctypes.byref(h)))
        self._h = h
        self._buf = (ctypes.c_uint64 * slots)()

    def submit(self, name, nodes=0):
        t = ctypes.c_uint64()
        _check(lib().hvm64_server_submit_nodes(self._h, name.encode(), nodes, ctypes.byref(t)))
        return t.value

    def budget(self):
        b, r, h = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().hvm64_server_budget(self._h, ctypes.byref(b), ctypes.byref(r), ctypes.byref(h)))
        return {"budget": b.value, "reserved": r.value, "heap_high": h.value}

    def poll(self):
        n = ctypes.c_size_t()
        _check(lib().hvm64_server_poll(self._h, self._buf, self.slots, ctypes.byref(n)))
        return [self._buf[i] for i in range(n.value)]

    def result(self, ticket, cap=1 << 22):
        rw = Rewrites()
        st = ctypes.c_int()
        us = ctypes.c_double()
        n = ctypes.c_size_t()
        buf = ctypes.create_string_buffer(cap)
        _check(lib().hvm64_server_result(self._h, ticket, ctypes.byref(rw), ctypes.byref(st), ctypes.byref(us), buf,
                                         cap, ctypes.byref(n)))
        if n.value >= cap:
            raise HvmError(ERR_BAD_INPUT, f"normal form needs {n.value + 1} bytes; pass a larger cap")
        return buf.value.decode(), rw, us.value

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.hvm64_server_free(self._h)
            self._h = None

    def __del__(self):
        self.close()


def book_format(text):
    """ast::Book::from_str + Display: the Book as the reference prints it
    (host-only; no device work)."""
    data = text.encode()
    return _read_text(lib().hvm64_book_format, data, len(data))


def pre_reduce(text, skip=(), max_rwts=(1 << 64) - 1, heap_bytes=0, tuning=None):
    """Book::pre_reduce (transform/src/pre_reduce.rs:27-74) on the GPU: every
    Def not in `skip` is reduced (no expansion) and replaced by its result.
    Returns (pre-reduced Book text, Rewrites, names of the Defs that did not
    reach normal form within max_rwts popped redexes)."""
    L = lib()
    data = text.encode()
    sk = " ".join(skip).encode()
    rw = Rewrites()
    n, nn = ctypes.c_size_t(), ctypes.c_size_t()
    t = ctypes.byref(tuning) if tuning is not None else None
    cap, ncap = max(8 * len(data), 1 << 16), max(len(data), 1 << 12)
    while True:
        buf, nbuf = ctypes.create_string_buffer(cap), ctypes.create_string_buffer(ncap)
        _check(L.hvm64_pre_reduce(data, len(data), sk, max_rwts, heap_bytes, t, ctypes.byref(rw), buf, cap,
                                  ctypes.byref(n), nbuf, ncap, ctypes.byref(nn)))
        if n.value < cap and nn.value < ncap:
            return buf.value.decode(), rw, [x for x in nbuf.value.decode().split("\n") if x]
        cap, ncap = n.value + 1, nn.value + 1  # rare: the results outgrew the buffers


def normal_noalloc(book, entry="main", tuning=None, cap=1 << 20):
    """hvm64_net_normal_noalloc: boot `entry`, normalise and read back using
    only the library's built-in device array (no device allocation).
    Returns (text, Rewrites)."""
    rw = Rewrites()
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_size_t()
    t = ctypes.byref(tuning) if tuning is not None else None
    _check(lib().hvm64_net_normal_noalloc(book._h, entry.encode(), t, ctypes.byref(rw), buf, cap, ctypes.byref(n)))
    if n.value >= cap:
        raise HvmError(ERR_BAD_INPUT, f"normal form needs {n.value + 1} bytes; pass a larger cap")
    return buf.value.decode(), rw


def run_book(text, entry="main", heap_bytes=0, tuning=None):
    """Boot `entry`, normalise on the GPU, read back: (text, counts dict)."""
    book = Book.from_str(text)
    net = Net(book, heap_bytes)
    net.boot(entry)
    rw = net.normal(tuning)
    return net.readback(), rw.as_dict()
