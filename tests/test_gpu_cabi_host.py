"""libdftk.so driven from C (tests/cabi/jk_host.c): dftk_prepare + dftk_jk
with only include/dftk.h and the CUDA runtime give the Python engine's J/K
(needs a GPU and gcc)."""
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

from conftest import REPO

pytestmark = pytest.mark.gpu

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_host(out_dir):
    exe = os.path.join(out_dir, "jk_host")
    lib_dir = os.path.join(REPO, "dft_b200")
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-I", os.path.join(REPO, "include"), "-I",
                    os.path.join(CUDA, "include"), os.path.join(REPO, "tests", "cabi", "jk_host.c"), "-o", exe,
                    "-L", lib_dir, "-ldftk", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
                    f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"], check=True)
    return exe


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not found")
def test_c_host_jk_matches_engine(tmp_path):
    from dft_b200 import basis, geometry
    from dft_b200.engine import IntegralEngine

    atoms, centers = geometry.water_cluster((2, 2, 1))
    shells = basis.build_shells(basis.load_basis(), atoms, centers)
    eng = IntegralEngine(shells)
    N = eng.n_ao
    rng = np.random.default_rng(4)
    A = rng.standard_normal((N, N))
    Da = 0.05 * (A + A.T)
    host = lambda t: t.detach().cpu().numpy()
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as fh:
        np.array([eng.ns, N, host(eng.d_exp).size], dtype=np.int32).tofile(fh)
        host(eng.d_xyz).astype(np.float64).tofile(fh)
        for t in (eng.d_l, eng.d_nprim, eng.d_prim_off, eng.d_ao):
            host(t).astype(np.int32).tofile(fh)
        host(eng.d_exp).astype(np.float64).tofile(fh)
        host(eng.d_cn).astype(np.float64).tofile(fh)
        (2 * Da).astype(np.float64).tofile(fh)
        Da.astype(np.float64).tofile(fh)
    exe = build_host(str(tmp_path))
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    JK = np.fromfile(out, dtype=np.float64).reshape(2, N, N)
    J0, K0, _ = eng.jk(torch.as_tensor(2 * Da, device=eng.device), torch.as_tensor(Da, device=eng.device), tau=1e-14)
    assert np.abs(JK[0] - host(J0)).max() < 1e-12
    assert np.abs(JK[1] - host(K0)).max() < 1e-12
    assert f"quartets {' '.join(str(t) for t in eng.quartet_totals())}" in r.stdout
