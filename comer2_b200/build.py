"""Build the sm_100a shared library ``_lib/libcomer2_b200.so`` in-tree, and
the search program ``_lib/comer2`` on top of it.

nvcc compiles the CUDA sources for ``sm_100a`` only (Blackwell B200); the
library exports the C ABI declared in ``include/comer2_b200.h``.  The program
(``host/comer2.cpp``, the reference ``comer``'s command line and file formats)
is plain C++ linked against the library.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libcomer2_b200.so")
PROG = os.path.join(HERE, "_lib", "comer2")
PROG_SRC = os.path.join(HERE, "host", "comer2.cpp")
SOURCES = ["c2_host.cu", "c2_kernels.cu", "c2_stats.cu", "c2_map.cu", "c2_adj.cu", "c2_dbio.cpp", "c2_report.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-I", os.path.join(ROOT, "include"),
]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    if not os.path.exists(PROG):
        return True
    t = min(os.path.getmtime(OUT), os.path.getmtime(PROG))
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "comer2_b200.h"),
                                                                 PROG_SRC]
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra=None) -> str:
    if not force and not needs_build():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [NVCC] + FLAGS + (extra or []) + ["-o", OUT] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building %s" % OUT)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    build_program(verbose)
    return OUT


def build_program(verbose: bool = False) -> str:
    """The comer2 search program, linked against the library (found next to
    it at run time)."""
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
           "-o", PROG, PROG_SRC, "-L", os.path.dirname(OUT), "-lcomer2_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("g++ failed building %s" % PROG)
    return PROG


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "-v" in sys.argv else None
    print(build(verbose=True, force=True, extra=extra))
