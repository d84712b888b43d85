"""Generate golden fixtures by running the reference's own ``shelled.py``.

Run in a container that has the reference tree (default ``/root/reference``);
the fixtures it writes (``tests/golden/*.npz``) are committed and are all the
tests ever read.

How the reference is run without CuPy or a GPU:

* ``cupy`` is replaced by a module that forwards to NumPy, with
  ``asnumpy``/``RawModule``/``cuda.runtime`` stand-ins; ``cupyx.scipy.special``
  is ``scipy.special``.
* ``RawModule`` checks that the source string it is given is the one
  ``oracle/build_ref.py`` compiled, then launches the host-compiled kernels
  from ``oracle/_ref/libref.so`` (one host iteration per CUDA thread).
* A copy of ``shelled.py`` is patched in memory -- basis file, molecule,
  multiplicity, integer electron counts for NumPy indexing, optional tighter
  convergence -- and executed in a temporary working directory, so the
  reference's own ``compute_eri/*.npy`` files land there.  The patched text is
  never written into this repository.

Usage::

    python tests/golden/make_golden.py h2o            # seconds
    python tests/golden/make_golden.py c10h22         # ~10-15 min
    python tests/golden/make_golden.py h2o64          # ~2 min (pair setup + sampled quartets)
    python tests/golden/make_golden.py grid           # seconds (H2O SCF + evaluation script)
    python tests/golden/make_golden.py br2            # d shells (STO-3G Br2)
    python tests/golden/make_golden.py gc             # general contractions + d (H2O, test basis)
    python tests/golden/make_golden.py gcf            # the same with f (O) and d (H) shells
    python tests/golden/make_golden.py grid_gc        # grid evaluation on the generally contracted H2O
"""
from __future__ import annotations

import argparse
import contextlib
import ctypes
import io
import json
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import build_ref  # noqa: E402
from dft_b200 import geometry  # noqa: E402

REFERENCE = os.environ.get("DFT_REFERENCE", "/root/reference")


# --------------------------------------------------------------------------- fake cupy
class _Kernel:
    def __init__(self, lib, name):
        self.name = name
        self.fn = getattr(lib, "ref_run_" + name)
        self.fn.restype = None

    def __call__(self, grid, block, args):
        n = int(grid[0]) * int(block[0])
        cargs = [ctypes.c_longlong(n)]
        for a in args:
            if isinstance(a, np.ndarray):
                if not a.flags["C_CONTIGUOUS"] or a.dtype not in (np.float64, np.int32):
                    raise TypeError(f"{self.name}: bad array arg {a.dtype} {a.flags}")
                cargs.append(ctypes.c_void_p(a.ctypes.data))
            else:
                cargs.append(ctypes.c_int(int(a)))
        self.fn(*cargs)


class _RawModule:
    expected_source = None
    lib = None

    def __init__(self, code, name_expressions=()):
        if code != _RawModule.expected_source:
            raise RuntimeError("kernel source differs from the one compiled into oracle/_ref")
        self.names = set(name_expressions)

    def get_function(self, name):
        return _Kernel(_RawModule.lib, name)


def install_fake_cupy():
    import scipy.special

    lib_path = build_ref.build(REFERENCE, quiet=True)
    _RawModule.lib = ctypes.CDLL(lib_path)
    _RawModule.expected_source = build_ref.extract_kernel_source(REFERENCE)

    cp = types.ModuleType("cupy")
    for k in dir(np):
        if not k.startswith("__"):
            setattr(cp, k, getattr(np, k))
    cp.asnumpy = np.asarray
    cp.RawModule = _RawModule
    runtime = types.SimpleNamespace(deviceSetLimit=lambda *a: None, cudaLimitStackSize=1,
                                    deviceSynchronize=lambda: None)
    cp.cuda = types.SimpleNamespace(runtime=runtime)
    cp.get_default_memory_pool = lambda: types.SimpleNamespace(free_all_blocks=lambda: None)
    cupyx = types.ModuleType("cupyx")
    cupyx_scipy = types.ModuleType("cupyx.scipy")
    cupyx_scipy.special = scipy.special
    cupyx.scipy = cupyx_scipy
    sys.modules["cupy"] = cp
    sys.modules["cupyx"] = cupyx
    sys.modules["cupyx.scipy"] = cupyx_scipy
    sys.modules["cupyx.scipy.special"] = scipy.special


# --------------------------------------------------------------------------- patching
def _replace_once(text, old, new):
    n = text.count(old)
    if n != 1:
        raise RuntimeError(f"patch anchor found {n} times: {old!r}")
    return text.replace(old, new)


def patched_shelled(etol=None, ptol=None, stop_before_eri=False):
    with open(os.path.join(REFERENCE, "shelled.py")) as fh:
        text = fh.read()
    text = _replace_once(text, 'data = json.load(open("ANO-RCC-MB.json"))',
                         "data = json.load(open(__BASIS_PATH__))")
    text = _replace_once(text, 'atoms = ["64", "9", "9", "9"]', "atoms = __ATOMS__")
    text = _replace_once(
        text, "centers = [[0.0, 0.0, 0.0], [4.0, 0, 0], [-2.0, 3.464, 0], [-2.0, -3.464, 0]]",
        "centers = __CENTERS__")
    text = _replace_once(text, "mult = 8", "mult = __MULT__")
    # NumPy refuses float index arrays; the electron counts are whole numbers.
    text = text.replace("xp.arange(0, N_a)", "xp.arange(0, int(N_a))")
    text = text.replace("xp.arange(0, N_b)", "xp.arange(0, int(N_b))")
    if etol is not None:
        text = _replace_once(text, "if delta_E < 1e-8 and delta_P < 1e-6:",
                             f"if delta_E < {etol!r} and delta_P < {ptol!r}:")
    if stop_before_eri:
        cut = text.index("calc_eri(pair_list, pair_cache, shells)\nprocess_eri()")
        text = text[:cut]
    return text


def run_reference(atoms, centers, mult=1, etol=None, ptol=None, stop_before_eri=False, basis_path=None):
    """Execute the patched reference script; return (namespace, workdir)."""
    text = patched_shelled(etol, ptol, stop_before_eri)
    work = tempfile.mkdtemp(prefix="dft_ref_")
    os.makedirs(os.path.join(work, "compute_eri"))
    os.makedirs(os.path.join(work, "eval_checkpoints"))
    ns = {
        "__name__": "shelled_reference_run",
        "__BASIS_PATH__": basis_path or os.path.join(REFERENCE, "STO-3G.json"),
        "__ATOMS__": list(atoms),
        "__CENTERS__": [[float(x) for x in c] for c in centers],
        "__MULT__": mult,
    }
    cwd = os.getcwd()
    os.chdir(work)
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            exec(compile(text, os.path.join(REFERENCE, "shelled.py") + ":patched", "exec"), ns)
    finally:
        os.chdir(cwd)
    return ns, work


def _load_processed(work):
    d = os.path.join(work, "compute_eri")
    out = {}
    for name in ("processed_eri_values", "processed_eri_indices", "processed_eri_quads",
                 "block_idxs", "chunked_quad_shape", "eri_quads", "eri_indices",
                 "eri_quads_shapes"):
        out[name] = np.load(os.path.join(d, name + ".npy"))
    return out


# --------------------------------------------------------------------------- cases
def case_h2o(out_dir):
    atoms, centers = geometry.water()
    res = {"atoms": np.array(atoms), "centers": centers}
    # reference convergence thresholds (shelled.py:1261)
    ns, work = run_reference(atoms, centers)
    res["energy_refthr"] = float(ns["E_total_new"])
    res["iterations_refthr"] = int(ns["count"])
    # tightened thresholds
    ns, work = run_reference(atoms, centers, etol=1e-12, ptol=1e-9)
    res["energy"] = float(ns["E_total_new"])
    res["iterations"] = int(ns["count"])
    for k in ("overlaps", "T_matrix", "V_matrix", "P_a", "P_b", "J_matrix", "K_a", "K_b"):
        res[k] = np.asarray(ns[k], dtype=np.float64)
    res["E_NN"] = float(ns["E_NN"])
    res.update(_load_processed(work))
    np.savez_compressed(os.path.join(out_dir, "h2o.npz"), **res)
    print("h2o energy", res["energy"], "iters", res["iterations"],
          "eri values", res["processed_eri_values"].shape)


def case_c10h22(out_dir, sample_every=400):
    atoms, centers = geometry.alkane(10)
    ns, work = run_reference(atoms, centers, etol=1e-10, ptol=1e-8)
    res = {"atoms": np.array(atoms), "centers": centers}
    res["energy"] = float(ns["E_total_new"])
    res["iterations"] = int(ns["count"])
    res["E_NN"] = float(ns["E_NN"])
    for k in ("overlaps", "T_matrix", "V_matrix", "P_a", "J_matrix", "K_a"):
        res[k] = np.asarray(ns[k], dtype=np.float64)
    pe = _load_processed(work)
    # every `sample_every`-th quartet of the reference's own (unsorted) order
    quads = pe["eri_quads"].astype(np.int32)
    idx = pe["eri_indices"]
    vals = np.load(os.path.join(work, "compute_eri", "eri_values.npy"), mmap_mode="r")
    pick = np.arange(0, quads.shape[0], sample_every)
    res["sample_quads"] = quads[pick]
    res["sample_offsets"] = np.concatenate([[0], np.cumsum(idx[pick, 1] - idx[pick, 0])])
    res["sample_values"] = np.concatenate([np.asarray(vals[idx[i, 0]:idx[i, 1]]) for i in pick])
    res["n_quartets"] = int(quads.shape[0])
    np.savez_compressed(os.path.join(out_dir, "c10h22.npz"), **res)
    print("c10h22 energy", res["energy"], "iters", res["iterations"], "quartets", quads.shape[0])


def case_h2o64(out_dir, n_subsets=12, subset_pairs=24, seed=1234):
    """Reference pair setup on (H2O)_64, then calc_eri on random pair subsets."""
    atoms, centers = geometry.water_cluster((4, 4, 4))
    ns, work = run_reference(atoms, centers, stop_before_eri=True)
    pair_list, pair_cache, shells = ns["pair_list"], ns["pair_cache"], ns["shells"]
    rng = np.random.default_rng(seed)
    # bias the subsets toward close pairs so the values are not all ~0
    pos = np.array([np.asarray(s["atom_pos"]) for s in shells])
    all_quads, all_vals, offsets = [], [], [0]
    for _ in range(n_subsets):
        centre = pos[rng.integers(len(shells))]
        near = [k for k, (i, j) in enumerate(pair_list)
                if np.linalg.norm(pos[i] - centre) < 9.0 and np.linalg.norm(pos[j] - centre) < 9.0]
        pick = rng.choice(near, size=min(subset_pairs, len(near)), replace=False)
        sub = [pair_list[k] for k in sorted(pick)]
        cwd = os.getcwd()
        os.chdir(work)
        try:
            with contextlib.redirect_stdout(io.StringIO()):
                ns["calc_eri"](sub, pair_cache, shells)
        finally:
            os.chdir(cwd)
        d = os.path.join(work, "compute_eri")
        q = np.load(os.path.join(d, "eri_quads.npy")).astype(np.int32)
        ix = np.load(os.path.join(d, "eri_indices.npy"))
        v = np.load(os.path.join(d, "eri_values.npy"))
        for t in range(q.shape[0]):
            all_quads.append(q[t])
            all_vals.append(v[ix[t, 0]:ix[t, 1]])
            offsets.append(offsets[-1] + ix[t, 1] - ix[t, 0])
    res = {"atoms": np.array(atoms), "centers": centers,
           "sample_quads": np.array(all_quads, dtype=np.int32),
           "sample_offsets": np.array(offsets, dtype=np.int64),
           "sample_values": np.concatenate(all_vals)}
    for k in ("overlaps", "T_matrix", "V_matrix"):
        m = np.asarray(ns[k])
        res[k + "_diag"] = np.diag(m).copy()
        res[k + "_row0"] = m[0].copy()
    np.savez_compressed(os.path.join(out_dir, "h2o64_sample.npz"), **res)
    print("h2o64 sampled quartets", len(all_quads), "values", res["sample_values"].shape)


BR2 = (["35", "35"], np.array([[0.0, 0.0, 0.0], [0.2, -0.3, 4.29]]))


def case_dshell(out_dir):
    """Br2 with the reference's STO-3G (3d shells on both atoms): every
    processed ERI, the spherical-basis S/T/V, the converged densities, J/K
    and the energy at tightened thresholds."""
    atoms, centers = BR2
    ns, work = run_reference(atoms, centers, etol=1e-11, ptol=1e-8)
    res = {"atoms": np.array(atoms), "centers": centers, "energy": float(ns["E_total_new"]),
           "iterations": int(ns["count"]), "E_NN": float(ns["E_NN"])}
    for k in ("overlaps", "T_matrix", "V_matrix", "P_a", "P_b", "J_matrix", "K_a", "K_b", "A"):
        res[k] = np.asarray(ns[k], dtype=np.float64)
    res.update(_load_processed(work))
    np.savez_compressed(os.path.join(out_dir, "br2.npz"), **res)
    print("br2 energy", res["energy"], "iters", res["iterations"], "eri values", res["processed_eri_values"].shape)


def case_gc(out_dir, basis_file="dz_gc_test.json", out_name="h2o_gc.npz"):
    """H2O with the generally contracted, d-polarised test basis
    (tests/golden/dz_gc_test.json; with basis_file dzf_gc_test.json also an f
    shell on O and a d shell on H): spherical-basis S/T/V, densities, J/K and
    the energy at tightened thresholds."""
    atoms, centers = geometry.water()
    ns, work = run_reference(atoms, centers, etol=1e-11, ptol=1e-8,
                             basis_path=os.path.join(HERE, basis_file))
    res = {"atoms": np.array(atoms), "centers": centers, "energy": float(ns["E_total_new"]),
           "iterations": int(ns["count"]), "E_NN": float(ns["E_NN"])}
    for k in ("overlaps", "T_matrix", "V_matrix", "P_a", "P_b", "J_matrix", "K_a", "K_b", "A"):
        res[k] = np.asarray(ns[k], dtype=np.float64)
    np.savez_compressed(os.path.join(out_dir, out_name), **res)
    print(out_name, "energy", res["energy"], "iters", res["iterations"], "n_sph", res["overlaps"].shape)


def patched_eval(spacing=0.15, chunk=500):
    """The reference's evaluation script with the H2O checkpoint the reference
    SCF just wrote, a coarser grid whose x range is widened by 1 bohr each way
    (the script's own x bounds assume a molecule that is not flat in x) and a
    small chunk size, so several chunks, the last one partial, run."""
    with open(os.path.join(REFERENCE, "shelled_eval.py")) as fh:
        text = fh.read()
    text = _replace_once(text, '"eval_checkpoints/cerium_3_fluoride_eval_checkpoint.npz"',
                         '"eval_checkpoints/gadolinium_3_fluoride_eval_checkpoint.npz"')
    text = _replace_once(text, "grid_spacing = 0.008", f"grid_spacing = {spacing!r}")
    text = _replace_once(text, "minx = float(xp.min(centers[:, 0]))", "minx = float(xp.min(centers[:, 0]) - 1.0)")
    text = _replace_once(text, "maxx = float(xp.max(centers[:, 0]) - 1.0)", "maxx = float(xp.max(centers[:, 0]) + 1.0)")
    text = _replace_once(text, "chunk_size = int(1e6)", f"chunk_size = int({chunk})")
    return text


def case_grid(out_dir, basis_file=None, prefix="h2o"):
    """Orbital densities on a grid for H2O: the reference SCF (its own
    thresholds) writes its evaluation checkpoint, then the reference's
    evaluation script runs on it.  Writes the checkpoint file as it is and the
    grid, total and phase densities.  With basis_file (a test basis in
    tests/golden/) the checkpoint carries d shells, general contractions and a
    non-identity spherical transform A."""
    import shutil

    atoms, centers = geometry.water()
    ns, work = run_reference(atoms, centers,
                             basis_path=os.path.join(HERE, basis_file) if basis_file else None)
    ckpt = os.path.join(work, "eval_checkpoints", "gadolinium_3_fluoride_eval_checkpoint.npz")
    os.makedirs(os.path.join(work, "preprocess"))
    cwd = os.getcwd()
    os.chdir(work)
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            exec(compile(patched_eval(), os.path.join(REFERENCE, "shelled_eval.py") + ":patched", "exec"),
                 {"__name__": "shelled_eval_reference_run"})
    finally:
        os.chdir(cwd)
    pre = os.path.join(work, "preprocess")
    res = {"grid": np.load(os.path.join(pre, "grid.npy")),
           "total_density": np.load(os.path.join(pre, "total_density.npy")),
           "phase_density": np.load(os.path.join(pre, "phase_density.npy")),
           "energy": float(ns["E_total_new"])}
    np.savez_compressed(os.path.join(out_dir, f"grid_{prefix}.npz"), **res)
    shutil.copyfile(ckpt, os.path.join(out_dir, f"{prefix}_eval_checkpoint.npz"))
    print("grid", res["grid"].shape, "total", res["total_density"].shape, "energy", res["energy"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["h2o", "c10h22", "h2o64", "grid", "br2", "gc", "gcf", "grid_gc"])
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    install_fake_cupy()
    {"h2o": case_h2o, "c10h22": case_c10h22, "h2o64": case_h2o64, "grid": case_grid, "br2": case_dshell,
     "gc": case_gc, "gcf": lambda out: case_gc(out, "dzf_gc_test.json", "h2o_gcf.npz"),
     "grid_gc": lambda out: case_grid(out, "dz_gc_test.json", "h2o_gc")}[args.case](args.out)


if __name__ == "__main__":
    main()
