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
SOURCES = ["dftk.cu", "jk_noalloc.cu", "hlc_part_a.cu", "hlc_part_b.cu", "hlc_part_c.cu", "hlc_part_d.cu"]
HEADERS = ["common.cuh", "boys.cuh", "eri_classes.cuh", "jk.cuh", "generic.cuh", "onee.cuh", "grad.cuh", "grid.cuh", "hl.cuh",
           "hl_classes.cuh", "hlc.cuh", "gen_hl.py", "hlc_parts.h", "hlc_part.cuh"]

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
    """Compile every source to an object in parallel (the generated d-class
    kernels sit in four hlc_part_*.cu units, the bulk of the compile time),
    then link libdftk.so."""
    generate_hl_classes()
    if not force and not needs_build():
        return LIB
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(obj_dir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *flags, *extra, "-I", HERE, "-I", os.path.join(REPO, "include"), "-c", "-o", obj,
               os.path.join(HERE, src)]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [src for src, pr in procs if pr.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, f"nvcc {' '.join(failed)}")
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v, force=True, extra=extra))
