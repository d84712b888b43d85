"""Build libdftk.so for sm_100a (in-tree, next to the package).

    python -m dft_b200.csrc.build          # or: python dft_b200/csrc/build.py
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libdftk.so")
SOURCES = ["dftk.cu", "jk_noalloc.cu"]
HEADERS = ["common.cuh", "boys.cuh", "eri_classes.cuh", "jk.cuh", "generic.cuh", "onee.cuh", "grad.cuh", "grid.cuh", "hl.cuh",
           "hl_classes.cuh", "hlc.cuh", "gen_hl.py"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, f) for f in SOURCES + HEADERS] + [os.path.join(REPO, "include", "dftk.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def generate_hl_classes() -> None:
    """Write hl_classes.cuh (the generated d classes, ~10 MB, not committed)
    from gen_hl.py when it is missing or differs from the generator's output."""
    sys.path.insert(0, HERE)
    try:
        import gen_hl
    finally:
        sys.path.remove(HERE)
    text = gen_hl.render()
    path = os.path.join(HERE, "hl_classes.cuh")
    if os.path.exists(path):
        with open(path) as fh:
            if fh.read() == text:
                return
    with open(path, "w") as fh:
        fh.write(text)


def build(verbose: bool = False, force: bool = False, extra=()) -> str:
    generate_hl_classes()
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", HERE, "-I", os.path.join(REPO, "include"),
           "-o", LIB] + [os.path.join(HERE, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v, force=True, extra=extra))
