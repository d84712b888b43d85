"""Benchmark: integral-direct J/K Fock builds of (H2O)_64 / STO-3G on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dftk|reference]

One step = one full FP64 direct J/K build (every Schwarz-surviving quartet,
tau 1e-12, density cut 1e-14) of (H2O)_64 / STO-3G (448 basis functions,
seeded 4x4x4 lattice, see dft_b200/geometry.py) at its converged RHF
density, inputs resident in HBM.  The L2 (126 MB) is flushed between steps
by writing a 256 MB buffer, outside the timed events.

Reported besides the headline:
  * e2e      the same build through the reference-facing call
             shelled.fill_matrices(shells, P, P_a, P_b, J, K_a, K_b) with host
             NumPy arrays (host->device densities and device->host J/K inside
             the timed region);
  * mixed    the incremental (D - D_prev) Fock builds of a full (H2O)_64 SCF,
             FP64 vs mixed FP32/FP64 (FP32 where Q_ab Q_cd |dD| < 1e-6),
             as builds/s of the incremental builds, against the plain FP64
             build, plus whole-SCF rates and |dE| in uEh;
  * roofline the dominant class kernel's achieved FP64 rate from the fixed
             flop accounting, against an FMA-loop peak measured here;
  * cpu_baseline  the reference's integral kernel (oracle/_ref, host-compiled)
             plus the restated contraction/digestion, timed on a sample of
             screened quartets per class and extrapolated by class counts.

With N > 1 (torchrun) every rank builds its own replica: weak scaling, no
collective on the data path; the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "J/K Fock builds/s, (H2O)_64 STO-3G, mixed vs FP64 at |ΔE|≤1µEh; grad time"
UNIT = "Fock builds/s"
WORKLOAD = "(H2O)_64 STO-3G RHF, 448 basis functions, direct J/K FP64, Schwarz 1e-12"


# ----------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to print its first sample: start the
            # timed region once it has (bounded wait), counting only what follows
            t_end = time.time() + 3.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines.clear()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return {}


def fma_peak_tflops(torch, lib, precision=64):
    """Measured FMA-pipe peak (TFLOP/s) from an 8-chain FMA loop on every SM."""
    from dft_b200 import _lib

    props = torch.cuda.get_device_properties(0)
    blocks, threads, iters = props.multi_processor_count * 8, 256, 4096
    sink = torch.empty(blocks * threads, dtype=torch.float64, device="cuda")
    s = _lib.stream_handle()
    for _ in range(2):
        _lib.call("dftk_fma_burn", precision, blocks, threads, iters, _lib.ptr(sink), s)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.call("dftk_fma_burn", precision, blocks, threads, iters, _lib.ptr(sink), s)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    flops = 2.0 * 8 * iters * blocks * threads
    return flops / best / 1e12


def setup_workload(torch, shape=(4, 4, 4)):
    from dft_b200 import basis, geometry
    from dft_b200.engine import IntegralEngine
    from dft_b200.scf import scf_rhf

    atoms, centers = geometry.water_cluster(shape)
    shells = basis.build_shells(basis.load_basis(), atoms, centers)
    eng = IntegralEngine(shells, tau_schwarz=1e-12)
    S, T, V = eng.one_electron(atoms, centers)
    H = T + V
    enn = geometry.nuclear_repulsion(atoms, centers)
    nocc = basis.n_electrons(atoms) // 2
    return atoms, centers, shells, eng, S, H, enn, nocc


# ------------------------------------------------------- batches, gradients
def gradient_figures(torch, eng, atoms, centers, res):
    """(H2O)_64 analytic gradient at the converged density: wall time of the
    dftk_grad call (device-synchronised) and per-class kernel times."""
    import ctypes

    from dft_b200 import _lib

    n_occ = basis_n_occ(atoms)
    C = res.C_a[:, :n_occ]
    D = 2.0 * (C @ C.T)
    W = 2.0 * ((C * res.eps_a[:n_occ]) @ C.T)
    Dh = (0.5 * D).contiguous()
    eng.gradient(atoms, centers, D, Dh, Dh, W)
    times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.gradient(atoms, centers, D, Dh, Dh, W)
        torch.cuda.synchronize()
        times.append((time.perf_counter() - t0) * 1e3)
    from dft_b200 import autotune
    from dft_b200.engine import QCLASS_NAMES
    from dft_b200.gradient import GRAD_TAU_FP32

    tuned = autotune.tune(eng, lambda: eng.gradient(atoms, centers, D, Dh, Dh, W), autotune.FAMILY_GRAD,
                          repeats=1)
    times = []
    g64 = None
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g64 = eng.gradient(atoms, centers, D, Dh, Dh, W)
        torch.cuda.synchronize()
        times.append((time.perf_counter() - t0) * 1e3)
    _lib.call("dftk_jk_timing", 1)
    eng.gradient(atoms, centers, D, Dh, Dh, W)
    buf = (ctypes.c_float * 13)()
    _lib.call("dftk_jk_timing_read", buf, 13)
    _lib.call("dftk_jk_timing", 0)
    autotune.tune(eng, lambda: eng.gradient(atoms, centers, D, Dh, Dh, W, tau_fp32=GRAD_TAU_FP32),
                  autotune.FAMILY_GRAD, fp32=True, repeats=1)
    mixed_times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gmx = eng.gradient(atoms, centers, D, Dh, Dh, W, tau_fp32=GRAD_TAU_FP32)
        torch.cuda.synchronize()
        mixed_times.append((time.perf_counter() - t0) * 1e3)
    return {"h2o64_grad_ms": float(np.median(times)),
            "class_ms": {QCLASS_NAMES[c]: float(buf[c]) for c in range(6)},
            "one_electron_ms": float(buf[12]),
            "shapes_threads_x_blocks_per_sm": tuned["shapes"],
            "h2o64_grad_mixed_ms": float(np.median(mixed_times)),
            "mixed_tau_fp32": GRAD_TAU_FP32,
            "mixed_max_abs_diff_vs_fp64_Eh_per_bohr": float(np.abs(gmx - g64).max()),
            "note": "analytic RHF gradient (derivative ERIs + S/T/V derivatives), converged (H2O)_64 density"}


def config4_gradients(torch):
    """The gradient workloads named for nuclear gradients: (H2O)_16 (2x2x4
    lattice) and C10H22, each the analytic RHF/STO-3G gradient at its
    converged density in FP64 and in the mixed form (median of 3 timed calls
    after a warm-up, device-synchronised), the mixed-vs-FP64 difference, and
    a central-difference check (h = 1e-4 bohr) of three coordinates."""
    from dft_b200 import basis, geometry
    from dft_b200.engine import IntegralEngine
    from dft_b200.gradient import GRAD_TAU_FP32, rhf_gradient
    from dft_b200.scf import scf_rhf

    def energy(atoms, c):
        sh = basis.build_shells(basis.load_basis(), atoms, c)
        eng = IntegralEngine(sh, tau_schwarz=1e-12)
        S, T, V = eng.one_electron(atoms, c)
        return scf_rhf(eng, T + V, S, basis.n_electrons(atoms) // 2, geometry.nuclear_repulsion(atoms, c),
                       etol=1e-12, dtol=1e-10).energy

    out = {}
    for name, (atoms, c) in (("h2o16", geometry.water_cluster((2, 2, 4))), ("c10h22", geometry.alkane(10))):
        c = np.asarray(c, dtype=np.float64)
        sh = basis.build_shells(basis.load_basis(), atoms, c)
        eng = IntegralEngine(sh, tau_schwarz=1e-12)
        S, T, V = eng.one_electron(atoms, c)
        nocc = basis.n_electrons(atoms) // 2
        res = scf_rhf(eng, T + V, S, nocc, geometry.nuclear_repulsion(atoms, c), etol=1e-12, dtol=1e-10)
        fig = {}
        for form, t32 in (("fp64", 0.0), ("mixed", GRAD_TAU_FP32)):
            rhf_gradient(eng, atoms, c, res, nocc, tau_fp32=t32)
            ts = []
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                g = rhf_gradient(eng, atoms, c, res, nocc, tau_fp32=t32)
                torch.cuda.synchronize()
                ts.append((time.perf_counter() - t0) * 1e3)
            fig[f"{form}_ms"] = float(np.median(ts))
            fig[f"grad_{form}"] = g
        fd = []
        for k in (0, 4, 3 * len(atoms) - 1):
            a, x = divmod(k, 3)
            cp, cm = c.copy(), c.copy()
            cp[a, x] += 1e-4
            cm[a, x] -= 1e-4
            fd.append(abs((energy(atoms, cp) - energy(atoms, cm)) / 2e-4 - fig["grad_fp64"][a, x]))
        out[name] = {"n_atoms": len(atoms), "n_basis": eng.n_ao, "fp64_ms": fig["fp64_ms"],
                     "mixed_ms": fig["mixed_ms"], "mixed_tau_fp32": GRAD_TAU_FP32,
                     "mixed_max_abs_diff_vs_fp64_Eh_per_bohr": float(np.abs(fig["grad_mixed"] - fig["grad_fp64"]).max()),
                     "fd_max_abs_err_Eh_per_bohr": float(max(fd)), "fd_coordinates": 3,
                     "grad_evals_per_s_fp64": 1e3 / fig["fp64_ms"]}
    return out


def error_figures(torch, eng):
    """Errors stated next to the results: ERIs of the (H2O)_64 quartets sampled
    from the reference's own run (tests/golden/h2o64_sample.npz, 3,600
    quartets) in FP64 and through the mixed path's FP32 kernels, and the H2O
    analytic gradient against central differences of the energy (1e-4 bohr)."""
    from dft_b200 import geometry
    from dft_b200.gradient import energy_and_gradient

    out = {}
    path = os.path.join(REPO, "tests", "golden", "h2o64_sample.npz")
    if os.path.exists(path):
        g = np.load(path)
        ref = g["sample_values"]
        for name, fp32 in (("max_abs_eri_err_fp64", False), ("max_abs_eri_err_fp32", True)):
            vals, _ = eng.eri_blocks(g["sample_quads"], fp32=fp32)
            out[name] = float(np.abs(vals.cpu().numpy() - ref).max())
        out["eri_sample"] = "3,600 (H2O)_64 quartets vs the reference's values"
    atoms, c = geometry.water()
    c = c + np.array([[0.02, -0.03, 0.01], [0.0, 0.05, -0.02], [-0.04, 0.0, 0.03]])
    scf = dict(etol=1e-12, dtol=1e-10)
    _, gr = energy_and_gradient(atoms, c, **scf)
    h, err = 1e-4, 0.0
    for a in range(3):
        for x in range(3):
            cp, cm = c.copy(), c.copy()
            cp[a, x] += h
            cm[a, x] -= h
            fd = (energy_and_gradient(atoms, cp, **scf)[0] - energy_and_gradient(atoms, cm, **scf)[0]) / (2 * h)
            err = max(err, abs(fd - gr[a, x]))
    out["max_abs_grad_err_vs_fd_Eh_per_bohr"] = err
    out["grad_check"] = "H2O (distorted), all 9 coordinates, central differences h = 1e-4 bohr"
    return out


def basis_n_occ(atoms):
    from dft_b200 import basis

    return basis.n_electrons(atoms) // 2


def batch_figures(torch, n_mol=512, n_max=24, n_single=64, n_grad=256, n_grad_max=16):
    """Batched SCF of n_mol seeded water clusters (1..n_max monomers) against
    a loop of single-molecule solves on the first n_single of them, and
    batched analytic gradients of n_grad clusters (1..n_grad_max monomers).
    Wall-clock, device-synchronised; setup (shells, pairs, Schwarz, queue,
    one-electron matrices) included on both sides."""
    from dft_b200 import basis, geometry
    from dft_b200.batch import BatchEngine, rhf_gradient_batch, scf_rhf_batch
    from dft_b200.engine import IntegralEngine
    from dft_b200.scf import scf_rhf

    mols = geometry.water_cluster_batch(n_mol, n_max, seed=0)
    # warm-up (library, cuBLAS handles, graph machinery) and launch-shape
    # tuning on a 64-molecule sub-batch; the timed solve reuses the shapes
    scf_rhf_batch(BatchEngine(mols[:64]), autotune=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    eng = BatchEngine(mols)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    res = scf_rhf_batch(eng)
    torch.cuda.synchronize()
    t_total = time.perf_counter() - t0
    it = res.iterations[res.converged]
    # loop of single solves on a sample
    single_t, single_it, dE = [], [], []
    for m, (atoms, c) in enumerate(mols[:n_single]):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        e1 = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c))
        S, T, V = e1.one_electron(atoms, c)
        r = scf_rhf(e1, T + V, S, basis.n_electrons(atoms) // 2, geometry.nuclear_repulsion(atoms, c))
        torch.cuda.synchronize()
        single_t.append(time.perf_counter() - t1)
        single_it.append(r.iterations)
        dE.append(abs(r.energy - res.energy[m]))
    single_rate = 1.0 / float(np.mean(single_t))
    out = {
        "batch_scf": {
            "workload": f"{n_mol} water clusters, 1..{n_max} monomers (seed 0), RHF/STO-3G FP64, one shell set",
            "molecules_per_s": n_mol / t_total, "seconds": t_total, "setup_s": t_setup,
            "solve_s": res.seconds, "fock_graph_replays": res.fock_builds, "fock_s": res.fock_seconds,
            "converged": int(res.converged.sum()),
            "iterations_p50": float(np.percentile(it, 50)), "iterations_p99": float(np.percentile(it, 99)),
            "single_loop": {"sample": n_single, "molecules_per_s": single_rate,
                            "iterations_p50": float(np.percentile(single_it, 50)),
                            "iterations_p99": float(np.percentile(single_it, 99)),
                            "max_abs_dE_vs_batch_Eh": float(np.max(dE))},
            "speedup_vs_single_loop": (n_mol / t_total) / single_rate,
        }
    }
    gm = geometry.water_cluster_batch(n_grad, n_grad_max, seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    geng = BatchEngine(gm)
    gres = scf_rhf_batch(geng, etol=1e-11, dtol=1e-9)
    torch.cuda.synchronize()
    t_scf = time.perf_counter() - t0
    rhf_gradient_batch(geng, gres)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    grads = rhf_gradient_batch(geng, gres)
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t1
    from dft_b200.gradient import GRAD_TAU_FP32

    rhf_gradient_batch(geng, gres, tau_fp32=GRAD_TAU_FP32)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    gmx = rhf_gradient_batch(geng, gres, tau_fp32=GRAD_TAU_FP32)
    torch.cuda.synchronize()
    t_grad_mx = time.perf_counter() - t1
    out["batch_grad"] = {
        "workload": f"{n_grad} water clusters, 1..{n_grad_max} monomers (seed 1), RHF/STO-3G FP64 analytic gradient",
        "gradient_evals_per_s": n_grad / t_grad, "gradient_s": t_grad,
        "mixed_gradient_evals_per_s": n_grad / t_grad_mx,
        "mixed_max_abs_diff_vs_fp64_Eh_per_bohr": float(max(np.abs(a - b).max() for a, b in zip(gmx, grads))),
        "with_scf_evals_per_s": n_grad / (t_scf + t_grad), "scf_s": t_scf,
        "converged": int(gres.converged.sum()),
        "max_abs_translational_sum": float(max(np.abs(g.sum(axis=0)).max() for g in grads)),
    }
    return out


# ------------------------------------------------------------ reference arm
def _pairs_by_class(shells):
    """Shell pairs (i, j), j <= i, in the reference's pair order, per pair class
    (l_a + l_b)."""
    l = np.array([s["angular_momentum"] for s in shells])
    ii, jj = np.tril_indices(len(shells))
    lo, hi = np.minimum(l[ii], l[jj]), np.maximum(l[ii], l[jj])
    pc = lo + hi
    return [np.stack([ii[pc == c], jj[pc == c]], axis=1) for c in range(3)]


def _sample_quartets(rng, pairs, q_by_class, X, Y, n, tau=1e-12):
    """n random Schwarz-kept unique quartets (Q_ab Q_cd >= tau) of the quartet
    class with pair classes (X, Y), as an (n, 4) int32 array of shells."""
    px, py = pairs[X], pairs[Y]
    qx, qy = q_by_class[X], q_by_class[Y]
    out = []
    have = 0
    while have < n:
        r = rng.integers(len(px), size=8 * n)
        k = rng.integers(len(py), size=8 * n)
        if X == Y:
            r, k = np.maximum(r, k), np.minimum(r, k)
        keep = qx[r] * qy[k] >= tau
        r, k = r[keep], k[keep]
        out.append(np.hstack([px[r], py[k]]))
        have += len(r)
    return np.ascontiguousarray(np.vstack(out)[:n], dtype=np.int32)


# Sample sizes (quartets) of the two timed calls per class: the marginal cost
# per quartet is the slope between them, so the fixed cost of one call (shell
# arrays, per-thread accumulators of 3 N^2 doubles, their reduction, thread
# start-up) is not multiplied by the class counts.  About 3 s of work on 16
# host threads for (H2O)_64.
CPU_SAMPLE_SMALL = (4000, 4000, 2000, 2000, 1000, 250)
CPU_SAMPLE_LARGE = (60000, 60000, 24000, 24000, 9000, 2250)


def cpu_reference_rate(eng_totals, shells, q_by_class, seed=0, small=CPU_SAMPLE_SMALL, large=CPU_SAMPLE_LARGE):
    """Fock builds/s of the reference's CPU path from per-class marginal costs.

    For each quartet class, two samples of Schwarz-kept quartets (sizes
    small[c] and large[c]) go through the reference's host-compiled
    eri_kernel (oracle/_ref; the restated one when it is not built) with the
    restated contraction and fill_matrices digestion; the slope between the
    two timings is the class's cost per quartet, the intercept the fixed cost
    of one call.  One build = sum_c slope_c * count_c + one fixed cost.
    Returns a dict: builds_per_s, cores, kind, us_per_quartet (per class),
    fixed_ms, sample_s (wall time of the timed calls), sample (description)."""
    from oracle import oracle as orc
    from dft_b200.engine import QCLASS_NAMES, QCLASS_PAIRS

    rng = np.random.default_rng(seed)
    pairs = _pairs_by_class(shells)
    sa = orc.ShellArrays(shells)
    N = sa.N
    A = rng.normal(size=(N, N))
    P = (A + A.T) * 0.01
    Ph = P / 2
    ref = orc.ref_lib()
    kind = "reference" if ref is not None else "port"

    def run(quads):
        t0 = time.perf_counter()
        if ref is not None:
            orc.direct_jk_reference_kernel(shells, quads, P, Ph, Ph, ref=ref, sa=sa)
        else:
            orc.direct_jk(shells, quads, P, Ph, Ph, sa=sa)
        return time.perf_counter() - t0

    run(_sample_quartets(rng, pairs, q_by_class, 0, 0, 64))  # thread pool and caches warm
    us, fixed, wall = {}, [], 0.0
    build_s = 0.0
    for c, (X, Y) in enumerate(QCLASS_PAIRS):
        if eng_totals[c] == 0:
            continue
        q1 = _sample_quartets(rng, pairs, q_by_class, X, Y, small[c])
        q2 = _sample_quartets(rng, pairs, q_by_class, X, Y, large[c])
        t1, t2 = run(q1), run(q2)
        wall += t1 + t2
        slope = max(t2 - t1, 1e-9) / (large[c] - small[c])
        us[QCLASS_NAMES[c]] = slope * 1e6
        fixed.append(max(t1 - slope * small[c], 0.0))
        build_s += slope * eng_totals[c]
    fixed_s = float(np.median(fixed)) if fixed else 0.0
    build_s += fixed_s
    cores = orc.lib().orc_num_threads()
    sample = (f"per class two timed calls of {'/'.join(map(str, small))} and {'/'.join(map(str, large))} "
              f"Schwarz-kept quartets (ss|ss)..(pp|pp) of (H2O)_64; the slope is the cost per quartet, "
              f"extrapolated by the class counts {list(map(int, eng_totals))} plus one fixed call cost; "
              f"{cores} OpenMP threads")
    return {"builds_per_s": 1.0 / build_s, "cores": cores, "kind": kind, "us_per_quartet": us,
            "fixed_ms": fixed_s * 1e3, "sample_s": wall, "sample": sample}


def cpu_reference_class_rates(shells, q_by_class, small, large, seed=0):
    """Shell quartets/s per class of the reference's CPU path (host-compiled
    eri_kernel + restated contraction and digestion) from the slope between
    two sample sizes of Schwarz-kept quartets (CPU-baseline leg)."""
    from oracle import oracle as orc
    from dft_b200.engine import QCLASS_PAIRS

    rng = np.random.default_rng(seed)
    pairs = _pairs_by_class(shells)
    sa = orc.ShellArrays(shells)
    N = sa.N
    A = rng.normal(size=(N, N))
    P = (A + A.T) * 0.01
    ref = orc.ref_lib()

    def run(quads):
        t0 = time.perf_counter()
        if ref is not None:
            orc.direct_jk_reference_kernel(shells, quads, P, P / 2, P / 2, ref=ref, sa=sa)
        else:
            orc.direct_jk(shells, quads, P, P / 2, P / 2, sa=sa)
        return time.perf_counter() - t0

    run(_sample_quartets(rng, pairs, q_by_class, 0, 0, 64))
    rates = []
    for c, (X, Y) in enumerate(QCLASS_PAIRS):
        t1 = run(_sample_quartets(rng, pairs, q_by_class, X, Y, small[c]))
        t2 = run(_sample_quartets(rng, pairs, q_by_class, X, Y, large[c]))
        rates.append((large[c] - small[c]) / max(t2 - t1, 1e-9))
    return rates, orc.lib().orc_num_threads(), "reference" if ref is not None else "port"


def grid_figures(torch, eng, centers, res, nocc, cpu: bool, n_points=1_000_000):
    """Orbital densities of the converged (H2O)_64 RHF on a grid (the
    evaluation-script workload): 320 occupied orbitals x 448 AOs at 1e6 random
    points in the cluster's box.  Device time per chunk (AO kernel, FP64 MO
    GEMM, density kernel) with CUDA events, the host-to-host rate through
    OrbitalGrid.evaluate, and the oracle on a 2,000-point sample."""
    import ctypes

    import numpy as np

    from dft_b200 import _lib, grid

    C = res.C_a.detach().cpu().numpy()
    n = eng.n_ao
    ck = {"centers": np.asarray(centers), "N_a": np.float64(nocc), "N_b": np.float64(nocc), "C_a": C, "C_b": C,
          "total_ao": np.int64(n), "shells": eng.shells, "A": np.eye(n)}
    og = grid.OrbitalGrid(ck)
    c = np.asarray(centers)
    rng = np.random.default_rng(0)
    host_pts = rng.uniform(c.min(0) - 2.0, c.max(0) + 2.0, size=(n_points, 3)).astype(np.float32)
    pts = torch.as_tensor(host_pts, device=eng.device)
    tot = torch.empty((og.n_mo, n_points), dtype=torch.float32, device=eng.device)
    ph = torch.empty((og.n_a, n_points), dtype=torch.float32, device=eng.device)
    for _ in range(3):
        og.chunk(pts, tot, ph)
    ms = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        og.chunk(pts, tot, ph)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    ao = torch.empty((n, n_points), dtype=torch.float64, device=eng.device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    _lib.call("dftk_grid_ao", ctypes.byref(eng.c_shells), n_points, _lib.ptr(pts), _lib.ptr(ao), n_points,
              _lib.stream_handle())
    ev[1].record()
    psi = og.Ca @ ao
    ev[2].record()
    _lib.call("dftk_grid_density", og.n_mo, og.n_a, og.n_b, n_points, _lib.ptr(psi), _lib.ptr(psi), n_points,
              _lib.ptr(tot), _lib.ptr(ph), n_points, _lib.stream_handle())
    ev[3].record()
    ev[3].synchronize()
    part = [ev[i].elapsed_time(ev[i + 1]) for i in range(3)]
    del ao, psi
    # host to host, steady state: outputs and pinned staging allocated by a
    # first call, the second call timed
    h_tot = np.zeros((og.n_mo, n_points), dtype=np.float32)
    h_ph = np.zeros((og.n_mo, n_points), dtype=np.float32)
    og.evaluate(host_pts, chunk_size=n_points, total=h_tot, phase=h_ph)
    t0 = time.perf_counter()
    og.evaluate(host_pts, chunk_size=n_points, total=h_tot, phase=h_ph)
    e2e_s = time.perf_counter() - t0
    chunk_ms = float(np.median(ms))
    out = {"workload": "(H2O)_64 RHF/STO-3G, 320 occupied orbitals x 448 AOs, 1e6 random points in the box",
           "points_per_s": n_points / (chunk_ms / 1e3), "chunk_ms": chunk_ms,
           "ao_kernel_ms": part[0], "mo_gemm_ms": part[1], "density_kernel_ms": part[2],
           "mo_gemm_tflops": 2.0 * og.n_mo * n * n_points / (part[1] / 1e3) / 1e12,
           "density_kernel_gbs": (og.n_mo * n_points * 8 + 2 * og.n_mo * n_points * 4) / (part[2] / 1e3) / 1e9,
           "e2e_points_per_s": n_points / e2e_s,
           "e2e_note": "host FP32 points in, host FP32 total and phase arrays out (2.56 GB per 1e6 points), "
                       "outputs and pinned staging reused (steady state of a multi-chunk run)"}
    if cpu:
        from oracle import oracle

        sample = host_pts[:2000]
        t0 = time.perf_counter()
        oracle.grid_densities(ck, sample)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": len(sample) / dt, "unit": "points/s", "cores": 1, "kind": "port",
                               "sample": "oracle.grid_densities (NumPy) on 2,000 of the points"}
    return out


def dshell_workload(torch):
    """(H2O)_16 (2x2x4 lattice) with the generally contracted, d-polarised test
    basis and a banded symmetric density: (engine, D, D/2)."""
    from dft_b200 import basis, geometry
    from dft_b200.engine import IntegralEngine

    with open(os.path.join(REPO, "tests", "golden", "dz_gc_test.json")) as fh:
        data = json.load(fh)
    atoms, centers = geometry.water_cluster((2, 2, 4))
    eng = IntegralEngine(basis.build_shells(data, atoms, centers), tau_schwarz=1e-12)
    N = eng.n_ao
    rng = np.random.default_rng(4)
    M = rng.normal(size=(N, N)) * np.exp(-0.2 * np.abs(np.subtract.outer(np.arange(N), np.arange(N))))
    D = torch.as_tensor(0.05 * (M + M.T), device=eng.device)
    return eng, D, (0.5 * D).contiguous()


def dshell_cpu_reference(seed=3, small=5000, large=30000, tau=1e-12):
    """The reference's CPU path on the d-basis workload: uniform samples of
    the Schwarz-kept unique quartets of the reference's own (generally
    contracted) shells at two sizes through the host-compiled reference
    eri_kernel (oracle/_ref; the restatement when it is not built) with the
    restated contraction and digestion; the slope between the two timings
    times the number of kept quartets, plus the intercept, is one build."""
    from dft_b200 import basis, geometry
    from oracle import oracle as orc

    with open(os.path.join(REPO, "tests", "golden", "dz_gc_test.json")) as fh:
        data = json.load(fh)
    atoms, centers = geometry.water_cluster((2, 2, 4))
    shells = basis.build_shells(data, atoms, centers)
    ii, jj = np.tril_indices(len(shells))
    diag = np.stack([ii, jj, ii, jj], axis=1).astype(np.int32)
    vals, off = orc.eri_quartets(shells, diag)
    q = np.sqrt(np.array([np.abs(vals[off[t]:off[t + 1]]).max() for t in range(len(ii))]))
    # kept unique quartets (pair r >= pair k, q_r q_k >= tau): count by sorting
    order = np.argsort(-q)
    qs = q[order]
    cnt = np.searchsorted(-qs, -np.where(qs > 0, tau / np.where(qs > 0, qs, 1.0), np.inf), side="right")
    total = int(np.minimum(cnt, np.arange(1, qs.size + 1)).sum())
    rng = np.random.default_rng(seed)
    sa = orc.ShellArrays(shells)
    N = sa.N
    A = rng.normal(size=(N, N))
    P = (A + A.T) * 0.01
    ref = orc.ref_lib()

    def sample(n):
        out = []
        while len(out) < n:
            r = rng.integers(q.size, size=4 * n)
            k = rng.integers(q.size, size=4 * n)
            r, k = np.maximum(r, k), np.minimum(r, k)
            keep = q[r] * q[k] >= tau
            for x, y in zip(r[keep], k[keep]):
                out.append((ii[x], jj[x], ii[y], jj[y]))
        return np.array(out[:n], dtype=np.int32)

    def run(quads):
        t0 = time.perf_counter()
        if ref is not None:
            orc.direct_jk_reference_kernel(shells, quads, P, P / 2, P / 2, ref=ref, sa=sa)
        else:
            orc.direct_jk(shells, quads, P, P / 2, P / 2, sa=sa)
        return time.perf_counter() - t0

    qs, ql = sample(small), sample(large)
    # median of three timings of the same samples (the host cores are shared)
    fits = []
    for _ in range(3):
        t_small, t_large = run(qs), run(ql)
        slope = max((t_large - t_small) / (large - small), 0.0)
        fits.append((slope * total + max(t_small - slope * small, 0.0), slope, t_small + t_large))
    fits.sort()
    s_build, slope, _ = fits[1]
    return {"kind": "reference" if ref is not None else "port", "cores": os.cpu_count(),
            "kept_unique_quartets": total, "us_per_quartet": slope * 1e6, "s_per_build": s_build,
            "sample": f"{small} and {large} uniformly drawn Schwarz-kept quartets (tau {tau}) of the reference's "
                      "generally contracted shells; slope x kept quartets + intercept; median of 3 timings",
            "s_per_build_3_timings": [f[0] for f in fits], "sample_s": sum(f[2] for f in fits)}


def dshell_scf(torch):
    """RHF/DIIS SCF of the d-basis workload ((H2O)_16, generally contracted
    d-polarised basis, spherical basis as the reference's SCF), FP64 and
    mixed: wall time (device-synchronised, after one warm-up solve),
    iterations, Fock builds and their time, energy and the mixed-vs-FP64
    energy difference."""
    from dft_b200 import basis, geometry
    from dft_b200.engine import IntegralEngine
    from dft_b200.scf import scf_rhf

    with open(os.path.join(REPO, "tests", "golden", "dz_gc_test.json")) as fh:
        data = json.load(fh)
    atoms, centers = geometry.water_cluster((2, 2, 4))
    eng = IntegralEngine(basis.build_shells(data, atoms, centers), tau_schwarz=1e-12)
    S, T, V = eng.one_electron(atoms, centers)
    nocc = basis.n_electrons(atoms) // 2
    enn = geometry.nuclear_repulsion(atoms, centers)
    out = {"workload": "(H2O)_16 2x2x4 lattice, generally contracted d-polarised test basis, RHF/DIIS"}
    scf_rhf(eng, T + V, S, nocc, enn)
    for name, mixed in (("fp64", False), ("mixed", True)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = scf_rhf(eng, T + V, S, nocc, enn, mixed=mixed)
        torch.cuda.synchronize()
        out[name] = {"wall_s": time.perf_counter() - t0, "iterations": r.iterations, "converged": bool(r.converged),
                     "fock_builds": r.fock_builds, "fock_s": r.fock_seconds, "energy": r.energy}
    out["mixed_minus_fp64_uEh"] = (out["mixed"]["energy"] - out["fp64"]["energy"]) * 1e6
    return out


def dshell_figures(torch):
    """The d/f path on a polarised basis: (H2O)_16 (2x2x4 lattice) with the
    generally contracted, d-polarised test basis (tests/golden/dz_gc_test.json;
    384 basis functions): one full FP64 J/K build at a converged-looking
    density, the s/p part (dftk_jk) and the d part (dftk_jk_hl) timed with
    CUDA events, and the quartets with a d shell."""
    import ctypes

    from dft_b200 import _lib

    eng, D, Dh = dshell_workload(torch)
    N = eng.n_ao
    J = torch.empty((N, N), dtype=torch.float64, device=eng.device)
    K = torch.empty_like(J)
    stream = _lib.stream_handle()

    def sp():
        _lib.call("dftk_jk", ctypes.byref(eng.c_shells), eng.c_pairs, ctypes.byref(eng.c_queue), _lib.ptr(D),
                  _lib.ptr(Dh), None, _lib.ptr(J), _lib.ptr(K), None, 0, 1e-14, 1e-14, _lib.ptr(eng.workspace),
                  eng.workspace_bytes, None, stream)

    def hl():
        _lib.call("dftk_jk_hl", ctypes.byref(eng.c_shells), ctypes.byref(eng.c_hl), _lib.ptr(D), _lib.ptr(Dh), None,
                  _lib.ptr(J), _lib.ptr(K), None, 0, 1e-14, _lib.ptr(eng.workspace), eng.workspace_bytes, None,
                  stream)

    def timed(fn, reps=5):
        fn()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    return {"workload": "(H2O)_16 2x2x4 lattice, generally contracted d-polarised test basis, FP64 J/K",
            "n_basis": N, "n_shells_segmented": eng.ns,
            "sp_part_ms": timed(sp), "d_part_ms": timed(hl), "full_build_ms": timed(lambda: eng.jk(D, Dh, tau=1e-14)),
            "d_candidate_quartets": [int(x) for x in eng.hl_totals], "sp_candidate_quartets": int(sum(eng.totals))}


def c10h22_figures(torch, cpu: bool):
    """C10H22 / STO-3G (72 basis functions): per-class ERI throughput of one
    full FP64 build at the converged density (CUDA events per class kernel),
    next to the reference's CPU path per class."""
    import ctypes

    from dft_b200 import _lib, basis, geometry
    from dft_b200.engine import QCLASS_NAMES, IntegralEngine
    from dft_b200.scf import scf_rhf

    atoms, c = geometry.alkane(10)
    shells = basis.build_shells(basis.load_basis(), atoms, c)
    eng = IntegralEngine(shells)
    S, T, V = eng.one_electron(atoms, c)
    r = scf_rhf(eng, T + V, S, basis.n_electrons(atoms) // 2, geometry.nuclear_repulsion(atoms, c))
    D = r.D_a
    Dt = (2 * D).contiguous()
    for _ in range(3):
        eng.jk(Dt, D, tau=1e-14)
    counts = torch.zeros(24, dtype=torch.int64, device="cuda")
    eng.jk(Dt, D, tau=1e-14, counts=counts)
    torch.cuda.synchronize()
    ev = counts[:6].tolist()
    _lib.call("dftk_jk_timing", 1)
    ms = []
    for _ in range(5):
        eng.jk(Dt, D, tau=1e-14)
        buf = (ctypes.c_float * 13)()
        _lib.call("dftk_jk_timing_read", buf, 13)
        ms.append(buf[:6])
    _lib.call("dftk_jk_timing", 0)
    ms = np.median(np.array(ms), axis=0)
    out = {"energy": r.energy, "quartets_per_class": eng.quartet_totals(), "evaluated_per_class": ev,
           "class_ms": {QCLASS_NAMES[k]: float(ms[k]) for k in range(6)},
           "quartets_per_s": {QCLASS_NAMES[k]: (ev[k] / (ms[k] / 1e3) if ms[k] > 0 else None) for k in range(6)}}
    if cpu:
        qs = schwarz_by_reference_order(shells)
        small, large = (2000, 2000, 1000, 1000, 500, 200), (10000, 10000, 5000, 5000, 2500, 1000)
        rates, cores, kind = cpu_reference_class_rates(shells, qs, small, large, seed=3)
        out["cpu_reference_quartets_per_s"] = {QCLASS_NAMES[k]: rates[k] for k in range(6)}
        out["cpu_reference"] = {"cores": cores, "kind": kind,
                                "sample": (f"slope between {'/'.join(map(str, small))} and {'/'.join(map(str, large))} "
                                           "Schwarz-kept quartets per class")}
    return out


def schwarz_by_reference_order(shells):
    """Per pair-class Schwarz factors in the reference pair order (CPU oracle)."""
    from oracle import oracle as orc

    l = np.array([s["angular_momentum"] for s in shells])
    ii, jj = np.tril_indices(len(shells))
    diag = np.stack([ii, jj, ii, jj], axis=1).astype(np.int32)
    vals, off = orc.eri_quartets(shells, diag)
    q = np.sqrt(np.array([np.abs(vals[off[t]:off[t + 1]]).max() for t in range(len(ii))]))
    pc = np.maximum(l[ii], l[jj]) + np.minimum(l[ii], l[jj])
    return [q[pc == c] for c in range(3)]


def run_reference_arm(args, rank, world):
    """The reference's CPU path on the host cores: each step times the
    per-class samples of cpu_reference_rate (a bounded sample of one (H2O)_64
    build) and extrapolates one build from their slopes.  Rank 0 only."""
    if rank != 0:
        return 0
    from dft_b200 import basis, geometry
    from dft_b200.engine import QCLASS_PAIRS, candidate_offsets

    atoms, centers = geometry.water_cluster((4, 4, 4))
    shells = basis.build_shells(basis.load_basis(), atoms, centers)
    qs = schwarz_by_reference_order(shells)
    qsorted = [np.sort(q)[::-1] for q in qs]
    totals = [int(candidate_offsets(qsorted[X], qsorted[Y], X == Y, 1e-12)[-1]) for X, Y in QCLASS_PAIRS]
    small = tuple(max(1, n // 10) for n in CPU_SAMPLE_SMALL)
    large = tuple(max(2, n // 10) for n in CPU_SAMPLE_LARGE)
    for w in range(max(0, args.warmup)):
        cpu_reference_rate(totals, shells, qs, seed=1 + w, small=small, large=large)
    rates, step_s, res = [], [], None
    t0 = time.perf_counter()
    for s in range(args.steps):
        ts = time.perf_counter()
        res = cpu_reference_rate(totals, shells, qs, seed=100 + s)
        step_s.append(time.perf_counter() - ts)
        rates.append(res["builds_per_s"])
    wall = time.perf_counter() - t0
    value = float(np.mean(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        # one step is a timed sample of a build, not a whole build (about 1e4 s)
        "ms_per_step": 1e3 * float(np.mean(step_s)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(len(shells) and shells[-1]["ao_stop"]),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["cores"], "kind": res["kind"],
                         "sample": res["sample"], "us_per_quartet": res["us_per_quartet"],
                         "fixed_ms_per_call": res["fixed_ms"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "extrapolated_s_per_build": 1.0 / value,
        "builds_per_s_per_step": rates,
        "wall_s": wall,
        "quartets_per_class": totals,
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(n_basis):
    """The config object both arms print for the (H2O)_64 J/K workload."""
    return {"workload": WORKLOAD, "molecule": "(H2O)_64 4x4x4 lattice seed 0", "basis": "STO-3G",
            "n_basis": int(n_basis), "tau_schwarz": 1e-12, "tau_density": 1e-14,
            "l2": "flushed between steps (256 MB write)", "parallelism": "replicas x1"}


# ---------------------------------------------------------------- main arm
def run_dftk_arm(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    from dft_b200 import _lib, shelled
    from dft_b200.engine import FLOPS_PER_PRIM_QUARTET, QCLASS_NAMES
    from dft_b200.scf import fp32_threshold, scf_rhf

    atoms, centers, shells, eng, S, H, enn, nocc = setup_workload(torch)
    # converged FP64 SCF (setup, untimed) gives the density of the timed builds
    ref_scf = scf_rhf(eng, H, S, nocc, enn, incremental=True, mixed=False, count_quartets=False)
    D = ref_scf.D_a
    Dt = (2.0 * D).contiguous()
    N = eng.n_ao
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    counts = torch.zeros(24, dtype=torch.int64, device="cuda")
    J = torch.empty((N, N), dtype=torch.float64, device="cuda")
    Ka = torch.empty((N, N), dtype=torch.float64, device="cuda")

    shard = None
    if dist is not None and args.shard:
        from dft_b200.sharding import ShardedFock

        shard = ShardedFock(eng)

    def build():
        if shard is not None:
            shard.jk(Dt, D, tau=1e-14)
        else:
            eng.jk(Dt, D, tau=1e-14, out=(J, Ka, None))

    for _ in range(max(args.warmup, 3)):
        build()
    torch.cuda.synchronize()
    # per-class launch shapes measured on this workload (dft_b200/autotune.py)
    from dft_b200 import autotune

    tuned = autotune.tune_jk(eng, Dt, D)
    tuned32 = autotune.tune_jk_mixed(eng, (1e-3 * D).contiguous())
    for _ in range(2):
        build()
    torch.cuda.synchronize()
    counts.zero_()
    eng.jk(Dt, D, tau=1e-14, counts=counts)
    torch.cuda.synchronize()
    evaluated = counts[:6].tolist()          # shell quartets per class
    prim_evaluated = counts[12:18].tolist()  # primitive quartets per class (after primitive screening)
    # per-class kernel times (events around each class launch inside dftk_jk)
    lib = _lib.load()
    _lib.call("dftk_jk_timing", 1)
    class_ms = np.zeros(12)
    n_timing = 3
    for _ in range(n_timing):
        flush.zero_()
        build()
        buf = (__import__("ctypes").c_float * 12)()
        _lib.call("dftk_jk_timing_read", buf, 12)
        class_ms += np.array(buf[:])
    class_ms /= n_timing
    _lib.call("dftk_jk_timing", 0)

    # timed steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            flush.zero_()
            starts[k].record()
            build()
            stops[k].record()
        torch.cuda.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    tot_ms = float(np.sum(step_ms))
    if dist is not None:
        t = torch.tensor([tot_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
        dist.barrier()
    ms_per_step = tot_ms / args.steps
    plain_rate = args.steps / (tot_ms / 1e3)  # builds/s of one system on this configuration
    # replicas: every rank builds the whole system (N builds per step);
    # sharded: the ranks build one system together (one build per step)
    value = (1 if shard is not None else world) * args.steps / (tot_ms / 1e3)

    # e2e through the reference-facing call with host arrays
    Dh = D.cpu().numpy()
    Ph = (2.0 * Dh).copy()
    Jh, Kah, Kbh = (np.zeros((N, N)) for _ in range(3))
    for _ in range(2):
        shelled.fill_matrices(shells, Ph, Dh, Dh, Jh, Kah, Kbh, tau=1e-14)
    e2e_ms = []
    for _ in range(max(2, min(args.steps, 5))):
        Jh[:] = 0
        Kah[:] = 0
        Kbh[:] = 0
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        shelled.fill_matrices(shells, Ph, Dh, Dh, Jh, Kah, Kbh, tau=1e-14)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_value = world * 1e3 / float(np.mean(e2e_ms))

    line = None
    if rank == 0:
        peaks = measured_peaks()
        fp64_peak = fma_peak_tflops(torch, lib, 64)
        fp32_peak = fma_peak_tflops(torch, lib, 32)
        class_flops = [FLOPS_PER_PRIM_QUARTET[c] * prim_evaluated[c] for c in range(6)]
        dom = int(np.argmax(class_ms[:6]))
        achieved = class_flops[dom] / (class_ms[dom] / 1e3) / 1e12
        total_flops = sum(class_flops)
        # the same accounting with every primitive quartet of the evaluated shell
        # quartets counted (STO-3G: 3 primitives per shell, 81 per quartet), i.e.
        # the rate a build without primitive screening would need to match
        full_prim_flops = sum(FLOPS_PER_PRIM_QUARTET[c] * 81 * evaluated[c] for c in range(6))
        # mixed vs FP64 over a full incremental SCF (setup of the comparison, timed per build)
        r64 = scf_rhf(eng, H, S, nocc, enn, incremental=True, mixed=False, count_quartets=True)
        rmx = scf_rhf(eng, H, S, nocc, enn, incremental=True, mixed=True, count_quartets=True)
        b64 = r64.fock_builds / r64.fock_seconds
        bmx = rmx.fock_builds / rmx.fock_seconds
        i64 = r64.incremental_builds / max(r64.incremental_seconds, 1e-12)
        imx = rmx.incremental_builds / max(rmx.incremental_seconds, 1e-12)
        traffic = None
        tpath = os.path.join(REPO, "profiles", "jk_traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as fh:
                tj = json.load(fh)
            traffic = tj.get("per_launch_bytes", {}).get(QCLASS_NAMES[dom])
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            from dft_b200.engine import QCLASS_PAIRS

            # the reference arm of this script in a child process: the same
            # code and samples as `--impl reference`, on host cores that this
            # process's GPU work and thread pools leave alone (timed in-process
            # after the GPU work, the same samples ran up to a third slower)
            import subprocess

            child = subprocess.run([sys.executable, os.path.abspath(__file__), "--impl", "reference", "--steps", "3",
                                    "--warmup", "3"], capture_output=True, text=True, timeout=600,
                                   env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
            ref_lines = [x for x in child.stdout.splitlines() if x.startswith("{")]
            if child.returncode == 0 and ref_lines:
                rl = json.loads(ref_lines[-1])
                cb = rl.get("cpu_baseline", {})
                cpu = {"value": rl["value"], "unit": UNIT, "cores": cb.get("cores"), "kind": cb.get("kind"),
                       "sample": cb.get("sample"), "us_per_quartet": cb.get("us_per_quartet"),
                       "builds_per_s_per_step": rl.get("builds_per_s_per_step"),
                       "method": "bench.py --impl reference --steps 3 --warmup 3, run as a child process"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if shard is not None else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(N), parallelism=(
                f"candidate space sharded x{world}, NCCL all-reduce of J/K" if shard is not None
                else f"replicas x{world}")),
            "quartets_per_class": eng.quartet_totals(), "evaluated_per_class": evaluated,
            "primitive_quartets_per_class": prim_evaluated, "tau_prim": eng.tau_prim,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * N * N * 8,
                    "d2h_bytes_per_step": 3 * N * N * 8, "call": "shelled.fill_matrices (host NumPy arrays)"},
            # per build: k_dsh, one k_select and one k_jk_list per class with candidates, k_symmetrize
            "gpu_launches": args.steps * (2 + 2 * sum(1 for c in range(6) if eng.quartet_totals()[c] > 0)),
            "roofline": {"bound": "fp64_fma", "kernel": f"k_jk<{dom},double> {QCLASS_NAMES[dom]}",
                         "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                         "peak_source": "measured FP64 FMA loop (dftk_fma_burn) on this GPU",
                         "traffic": traffic,
                         "traffic_source": ("profiles/jk_traffic.json: dram__bytes_read.sum + dram__bytes_write.sum "
                                            "of one launch of this kernel from an earlier ncu capture of this "
                                            "workload, read by the bench (not measured in this run)"),
                         "whole_build_tflops": total_flops / (ms_per_step / 1e3) / 1e12,
                         "whole_build_tflops_81_prims_per_quartet": full_prim_flops / (ms_per_step / 1e3) / 1e12,
                         "class_ms": {QCLASS_NAMES[c]: float(class_ms[c]) for c in range(6)},
                         "fp32_peak_tflops": fp32_peak, "hbm_peak_gbs": peaks.get("hbm_gbs")},
            "mixed": {"speedup_mixed_vs_fp64_incremental": imx / i64,
                      "comparison": "like for like: the incremental (D - D_prev) builds of the same SCF, "
                                    "FP64 against mixed; same screening, only the precision differs",
                      "tau_fp32": fp32_threshold(sum(eng.quartet_totals())),
                      "tau_fp32_rule": "1 uEh budget / (2^-20 sqrt(Schwarz candidates)), clamped to [1e-6, 1e-4]",
                      "plain_fp64_builds_per_s": plain_rate,
                      "fp64_incremental_builds_per_s": i64, "mixed_incremental_builds_per_s": imx,
                      "speedup_mixed_vs_plain_fp64": imx / plain_rate,
                      "incremental_builds": [r64.incremental_builds, rmx.incremental_builds],
                      "scf_builds_per_s_fp64": b64, "scf_builds_per_s_mixed": bmx,
                      "scf_speedup": bmx / b64, "scf_iterations_fp64": r64.iterations,
                      "scf_iterations_mixed": rmx.iterations,
                      "energy_fp64": r64.energy, "energy_mixed_final": rmx.energy,
                      "delta_E_uEh_final": abs(rmx.energy - r64.energy) * 1e6,
                      "delta_E_uEh_last_mixed_build": abs(rmx.energy_last_build - r64.energy) * 1e6,
                      "quartets_fp64_fp32_mixed": rmx.counts},
            "autotune": {"shapes_threads_x_blocks_per_sm": tuned["shapes"], "tiles": tuned.get("tiles"),
                         "default_class_ms": tuned["default_ms"], "tuned_class_ms": tuned["tuned_ms"],
                         "fp32_shapes": tuned32["shapes"], "fp32_tiles": tuned32.get("tiles"),
                         "fp32_default_class_ms": tuned32["default_ms"],
                         "fp32_tuned_class_ms": tuned32["tuned_ms"]},
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        line["eri_quartets_per_s"] = sum(evaluated) / (ms_per_step / 1e3)
        if not args.no_extras:
            line["c10h22"] = c10h22_figures(torch, cpu=world == 1 and not args.no_cpu_baseline)
            line["d_basis"] = dshell_figures(torch)
            if world == 1 and not args.no_cpu_baseline:
                ref = dshell_cpu_reference()
                ref["gpu_speedup"] = ref["s_per_build"] / (line["d_basis"]["full_build_ms"] / 1e3)
                line["d_basis"]["cpu_reference"] = ref
            line["d_basis"]["scf"] = dshell_scf(torch)
            line["grad"] = gradient_figures(torch, eng, atoms, centers, r64)
            line["grad"]["config4"] = config4_gradients(torch)
            line["grid"] = grid_figures(torch, eng, centers, r64, nocc, cpu=world == 1 and not args.no_cpu_baseline)
            line["errors"] = error_figures(torch, eng)
            line.update(batch_figures(torch))
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_profile(args):
    """A few builds of the benchmark workload for ncu captures: two full FP64
    builds, then one mixed build of a scaled-down density (kernel launch order
    per build: k_dsh, k_select x6, k_jk_list<0..5,double>, [k_jk_list<0..5,float>],
    k_symmetrize), then one gradient (and with --profile-grid two grid chunks)."""
    import torch

    if args.profile_dshell:
        # two full FP64 J/K builds of the d-basis workload: k_dsh, the s/p
        # class kernels, k_symmetrize, then k_dsh, k_hlc<C, S> per class and
        # component chunk, k_hl_jk<2>,
        # k_symmetrize_add per build
        deng, D, Dh = dshell_workload(torch)
        for _ in range(2):
            deng.jk(D, Dh, tau=1e-14)
        torch.cuda.synchronize()
        print("profile workload done")
        return 0
    atoms, centers, shells, eng, S, H, enn, nocc = setup_workload(torch)
    X = torch.linalg.inv(torch.linalg.cholesky(S)).T
    _, C = torch.linalg.eigh(X.T @ H @ X)
    C = X @ C
    D = C[:, :nocc] @ C[:, :nocc].T
    for _ in range(2):
        eng.jk(2 * D, D, tau=1e-14)
    dD = D * 1e-3
    eng.jk(2 * dD, dD, mixed=True, tau=1e-12, tau_fp32=1e-6)
    # one analytic gradient at this (core-guess) density: launch order k_dsh,
    # k_grad_overlap_kinetic/k_grad_nuclear x3, k_select x6, k_grad_eri<0..5>
    Dt = (2 * D).contiguous()
    eng.gradient(atoms, centers, Dt, D, D, Dt)
    torch.cuda.synchronize()
    if args.profile_grid:
        # two 200,000-point grid chunks with the core-guess orbitals: launch
        # order k_grid_ao, (DGEMM), k_grid_density, twice
        from dft_b200 import grid

        n = eng.n_ao
        Ch = C.detach().cpu().numpy()
        ck = {"centers": np.asarray(centers), "N_a": np.float64(nocc), "N_b": np.float64(nocc), "C_a": Ch,
              "C_b": Ch, "total_ao": np.int64(n), "shells": eng.shells, "A": np.eye(n)}
        og = grid.OrbitalGrid(ck)
        c = np.asarray(centers)
        m = 200_000
        pts = torch.as_tensor(np.random.default_rng(0).uniform(c.min(0) - 2, c.max(0) + 2, size=(m, 3))
                              .astype(np.float32), device=eng.device)
        tot = torch.empty((og.n_mo, m), dtype=torch.float32, device=eng.device)
        ph = torch.empty((og.n_a, m), dtype=torch.float32, device=eng.device)
        for _ in range(2):
            og.chunk(pts, tot, ph)
        torch.cuda.synchronize()
    print("profile workload done")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dftk", choices=["dftk", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the gradient and batch figures")
    ap.add_argument("--shard", action="store_true",
                    help="with N > 1: the ranks build one (H2O)_64 Fock matrix together (strong scaling)")
    ap.add_argument("--profile", action="store_true", help="only run a few builds (for ncu captures)")
    ap.add_argument("--profile-grid", action="store_true", help="with --profile: also two grid-evaluation chunks")
    ap.add_argument("--profile-dshell", action="store_true",
                    help="with --profile: only two J/K builds of the d-basis (H2O)_16 workload")
    args = ap.parse_args()
    if args.profile:
        return run_profile(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    return run_dftk_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
