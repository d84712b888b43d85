"""Compile the reference's own integral kernels as host C++ into ``oracle/_ref/``.

TEST INFRASTRUCTURE ONLY.  The shared object built here is a checker and the
timed CPU baseline of ``bench.py --impl reference``; nothing in the product
(``dft_b200/``) loads it.

The reference keeps its integral kernels as CUDA C source inside a Python
f-string (``shelled.py:166-533``) that CuPy hands to NVRTC at run time
(``shelled.py:923-931``).  The string has no ``{}`` placeholders, so it is
plain C++ once ``{{``/``}}`` are unescaped (the AST constant already holds the
unescaped text).  This recipe reads that string where it lies under the
reference tree, prepends a shim that turns ``__global__``/``__device__`` into
ordinary host functions with thread-local ``blockIdx``/``threadIdx``, and
appends launch loops that walk the flat thread index ``q`` exactly as the
kernels compute it (``blockIdx.x * blockDim.x + threadIdx.x`` with
``blockDim.x = 1``).  Only ``#include <math_constants.h>`` is dropped; the
shim defines ``CUDART_PI`` instead.

No reference source is written anywhere but ``oracle/_ref/`` (git-ignored).

Usage: ``python oracle/build_ref.py [--reference DIR]``.
"""
from __future__ import annotations

import argparse
import ast
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libref.so")

SHIM = r"""
// Host shim for the reference kernel string (generated by oracle/build_ref.py).
#include <cmath>
#include <cstdint>
using std::exp; using std::erf; using std::sqrt;
#define __device__
#define __global__
#define CUDART_PI 3.141592653589793115997963468544185161590576171875
struct ref_uint3 { unsigned int x, y, z; };
static thread_local ref_uint3 blockIdx = {0, 0, 0};
static thread_local ref_uint3 threadIdx = {0, 0, 0};
static thread_local ref_uint3 blockDim = {1, 1, 1};
"""

DRIVER = r"""
// Launch loops: one host iteration per CUDA thread of the original launch.
extern "C" void ref_run_nuclear_kernel(long long n_threads,
    const double* exp_a, const double* exp_b, const double* cen_a, const double* cen_b,
    const int* pow_a, const int* pow_b, const int* atoms, const double* atom_centers,
    int num_atoms, int num_funcs_a, int num_funcs_b, double* V, double* Ex, double* Ey,
    double* Ez, double* p, double* P, int* nx, int* ny, int* nz) {
    #pragma omp parallel for schedule(static)
    for (long long q = 0; q < n_threads; ++q) {
        blockDim.x = 1; threadIdx.x = 0; blockIdx.x = (unsigned int)q;
        nuclear_kernel(exp_a, exp_b, cen_a, cen_b, pow_a, pow_b, atoms, atom_centers,
                       num_atoms, num_funcs_a, num_funcs_b, V, Ex, Ey, Ez, p, P, nx, ny, nz);
    }
}

extern "C" void ref_run_eri_kernel(long long n_threads,
    int K_ab, const double* p_ab, const double* P_ab, const double* Exab, const double* Eyab,
    const double* Ezab, const int* nxab, const int* nyab, const int* nzab,
    int K_cd, const double* p_cd, const double* P_cd, const double* Excd, const double* Eycd,
    const double* Ezcd, const int* nxcd, const int* nycd, const int* nzcd, double* out) {
    #pragma omp parallel for schedule(static) if (n_threads > 4096)
    for (long long q = 0; q < n_threads; ++q) {
        blockDim.x = 1; threadIdx.x = 0; blockIdx.x = (unsigned int)q;
        eri_kernel(K_ab, p_ab, P_ab, Exab, Eyab, Ezab, nxab, nyab, nzab,
                   K_cd, p_cd, P_cd, Excd, Eycd, Ezcd, nxcd, nycd, nzcd, out);
    }
}

// One call per shell quartet, many quartets per call: the reference launches
// eri_kernel once per quartet (shelled.py:642); batching the host loop here
// only removes Python overhead, each quartet still runs the reference kernel.
extern "C" void ref_run_eri_batch(int n_quartets, const long long* ab_off, const long long* cd_off,
    const int* K_ab, const int* K_cd, const double* p, const double* P, const double* Ex,
    const double* Ey, const double* Ez, const int* nx, const int* ny, const int* nz,
    const long long* out_off, double* out) {
    #pragma omp parallel for schedule(dynamic, 4)
    for (int t = 0; t < n_quartets; ++t) {
        long long a = ab_off[t], c = cd_off[t];
        long long n = (long long)K_ab[t] * K_cd[t];
        for (long long q = 0; q < n; ++q) {
            blockDim.x = 1; threadIdx.x = 0; blockIdx.x = (unsigned int)q;
            eri_kernel(K_ab[t], p + a, P + 3 * a, Ex + 7 * a, Ey + 7 * a, Ez + 7 * a,
                       nx + a, ny + a, nz + a, K_cd[t], p + c, P + 3 * c, Ex + 7 * c,
                       Ey + 7 * c, Ez + 7 * c, nx + c, ny + c, nz + c, out + out_off[t]);
        }
    }
}
"""


def extract_kernel_source(reference_dir: str) -> str:
    """Return the CUDA C string assigned to ``source`` in shelled.py (:166-533)."""
    path = os.path.join(reference_dir, "shelled.py")
    with open(path) as fh:
        tree = ast.parse(fh.read(), filename=path)
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(
            getattr(t, "id", None) == "source" for t in node.targets
        ):
            value = node.value
            if isinstance(value, ast.JoinedStr):
                if not all(isinstance(v, ast.Constant) for v in value.values):
                    raise RuntimeError("kernel f-string has placeholders; cannot build")
                return "".join(v.value for v in value.values)
            if isinstance(value, ast.Constant):
                return value.value
    raise RuntimeError(f"no `source = ...` assignment found in {path}")


# Where this recipe looks for the reference checkout when DFT_REFERENCE is not
# set (the build container's read-only copy; absent on machines that only run
# the prebuilt files).
_CONTAINER_REFERENCE = "/root/reference"


def reference_dir():
    """The reference checkout to compile from: $DFT_REFERENCE, else the build
    container's copy; None when neither exists (nothing to build)."""
    for d in (os.environ.get("DFT_REFERENCE"), _CONTAINER_REFERENCE):
        if d and os.path.isfile(os.path.join(d, "shelled.py")):
            return d
    return None


def build(reference_dir: str, quiet: bool = False) -> str:
    src = extract_kernel_source(reference_dir)
    lines = [ln for ln in src.splitlines() if "#include <math_constants.h>" not in ln]
    os.makedirs(OUT_DIR, exist_ok=True)
    cpp = os.path.join(OUT_DIR, "ref_kernels.cpp")
    with open(cpp, "w") as fh:
        fh.write(SHIM)
        fh.write("\n".join(lines))
        fh.write("\n")
        fh.write(DRIVER)
    cmd = ["g++", "-O2", "-fopenmp", "-shared", "-fPIC", "-std=c++17", "-o", LIB, cpp]
    subprocess.run(cmd, check=True, capture_output=quiet)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference checkout (default: $DFT_REFERENCE)")
    args = ap.parse_args()
    ref = args.reference or reference_dir()
    if ref is None:
        ap.error("no reference checkout: pass --reference or set DFT_REFERENCE")
    print(build(ref))


if __name__ == "__main__":
    sys.exit(main())
