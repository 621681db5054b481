"""Build recipe for the B200 reducer (nvcc for sm_100a + g++ for the host layer).

    python hvm-64_b200/build.py          # builds build/libhvm64.so, build/hvm64 (CLI)
                                         # and build/hvm64_atomic_peak

Outputs stay in-tree (hvm-64_b200/build/) so they travel with the repository
snapshot to the GPU machine.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "build")
INC = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(OUT, "libhvm64.so")
CLI = os.path.join(OUT, "hvm64")
PEAK = os.path.join(OUT, "hvm64_atomic_peak")  # L2 atomic-rate microbenchmark

SOURCES = ["hvm64.cu", "host.cpp", "host.hpp", "device.cuh", "num.h", "cli.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]}")
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    os.makedirs(OUT, exist_ok=True)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(INC, "hvm64.h"), __file__]
    if force or _stale(LIB, deps):
        host_o = os.path.join(OUT, "host.o")
        _run(["g++", "-std=c++20", "-O2", "-fPIC", "-Wall", "-I", INC, "-c", os.path.join(CSRC, "host.cpp"),
              "-o", host_o])
        dev_o = os.path.join(OUT, "hvm64.o")
        log = _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xptxas", "-v",
                    "-Xcompiler", "-fPIC", "-I", INC, "-c", os.path.join(CSRC, "hvm64.cu"), "-o", dev_o])
        if verbose:
            sys.stderr.write(log)
        _run([NVCC, *ARCH, "-shared", "-o", LIB, dev_o, host_o, "-lcudart"])
    peak_src = os.path.join(CSRC, "atomic_peak.cu")
    if os.path.exists(peak_src) and (force or _stale(PEAK, [peak_src, __file__])):
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", peak_src, "-o", PEAK])
    if os.path.exists(os.path.join(CSRC, "cli.cpp")) and (force or _stale(CLI, deps + [LIB])):
        _run(["g++", "-std=c++20", "-O2", "-I", INC, os.path.join(CSRC, "cli.cpp"), "-o", CLI,
              "-L", OUT, "-lhvm64", "-Wl,-rpath,$ORIGIN"])
    return LIB


GEN = os.path.join(OUT, "gen")


def compiled_source_hash(source):
    """The Book hash a generated source was made for (its HVM_GEN_HASH)."""
    for line in source.splitlines():
        if line.startswith("#define HVM_GEN_HASH "):
            return line.split()[2].removesuffix("ull")
    raise ValueError("not a generated Def source")


def build_compiled(source, verbose=False):
    """`hvm64 compile` for a Book: `source` is its generated Def functions
    (hvm64.Book.compile_source, hvm64_book_compile_source).  Builds
    build/gen/libhvm64_<hash>.so, the reducer library with those functions in
    place of the instruction VM for that Book (any other Book still runs on
    the VM), and returns its path.  Rebuilt only when missing or stale."""
    build()
    os.makedirs(GEN, exist_ok=True)
    h = compiled_source_hash(source)
    hdr = os.path.join(GEN, f"defs_{h}.cuh")
    lib = os.path.join(GEN, f"libhvm64_{h}.so")
    if not os.path.exists(hdr) or open(hdr).read() != source:
        with open(hdr, "w") as f:
            f.write(source)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(INC, "hvm64.h"), hdr, __file__]
    if _stale(lib, deps):
        obj = os.path.join(GEN, f"hvm64_{h}.o")
        log = _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xptxas", "-v",
                    "-Xcompiler", "-fPIC", "-I", INC, f'-DHVM_GEN_INCLUDE="{hdr}"', "-c",
                    os.path.join(CSRC, "hvm64.cu"), "-o", obj])
        if verbose:
            sys.stderr.write(log)
        _run([NVCC, *ARCH, "-shared", "-o", lib, obj, os.path.join(OUT, "host.o"), "-lcudart"])
        os.remove(obj)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
