"""Build the sm_100a shared library ``_lib/libcomer2_b200.so`` in-tree.

nvcc compiles the CUDA sources for ``sm_100a`` only (Blackwell B200); the
library exports the C ABI declared in ``include/comer2_b200.h``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libcomer2_b200.so")
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
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "comer2_b200.h")]
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
    return OUT


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "-v" in sys.argv else None
    print(build(verbose=True, force=True, extra=extra))
