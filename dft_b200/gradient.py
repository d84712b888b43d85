"""Analytic RHF nuclear gradients and a torch.autograd.Function from
coordinates to energy.

The electronic part comes from ``dftk_grad`` (derivative integrals at L + 1
with exponent-shifted Hermite coefficients, contracted on the GPU with the
densities); the nuclear repulsion part is analytic on the host.
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np
import torch

from . import basis as _basis, geometry as _geometry
from .engine import IntegralEngine
from .scf import SCFResult, scf_rhf


# mixed form: quartets whose gradient bound Q_ab Q_cd max|D|^2 is below this
# are differentiated in FP32 (sums in FP64); the J/K build's FP32 threshold.
# Measured on (H2O)_64: 3e-10 Eh/bohr from the FP64 gradient, 1.5x faster
GRAD_TAU_FP32 = 1e-6


def rhf_gradient(engine: IntegralEngine, atoms: Sequence[str], centers, res: SCFResult, n_occ: int,
                 tau: float = 1e-14, tau_fp32: float = 0.0) -> np.ndarray:
    """dE/dR (n_atoms, 3) of a converged RHF solution: D = 2 C_occ C_occ^T,
    W = 2 C_occ diag(eps_occ) C_occ^T (tau_fp32 > tau: the mixed form)."""
    C = res.C_a[:, :n_occ]
    eps = res.eps_a[:n_occ]
    D = 2.0 * (C @ C.T)
    W = 2.0 * ((C * eps) @ C.T)
    Dh = (0.5 * D).contiguous()
    g = engine.gradient(atoms, centers, D, Dh, Dh, W, tau=tau, tau_fp32=tau_fp32)
    return g + _geometry.nuclear_repulsion_gradient(atoms, np.asarray(centers, dtype=np.float64))


def energy_and_gradient(atoms: Sequence[str], centers, basis_data: Optional[dict] = None, charge: int = 0,
                        mixed: bool = False, tau_schwarz: float = 1e-12, **scf_kw) -> Tuple[float, np.ndarray]:
    """RHF energy and analytic gradient at one geometry (bohr).  mixed=True:
    mixed FP32/FP64 incremental SCF and the mixed gradient (GRAD_TAU_FP32)."""
    centers = np.asarray(centers, dtype=np.float64)
    shells = _basis.build_shells(basis_data if basis_data is not None else _basis.load_basis(), atoms, centers)
    eng = IntegralEngine(shells, tau_schwarz=tau_schwarz)
    S, T, V = eng.one_electron(atoms, centers)
    n = _basis.n_electrons(atoms, charge)
    if n % 2:
        raise ValueError("RHF gradient needs an even electron count")
    res = scf_rhf(eng, T + V, S, n // 2, _geometry.nuclear_repulsion(atoms, centers), mixed=mixed, **scf_kw)
    if not res.converged:
        raise RuntimeError("SCF did not converge")
    return res.energy, rhf_gradient(eng, atoms, centers, res, n // 2, tau_fp32=GRAD_TAU_FP32 if mixed else 0.0)


class RHFEnergy(torch.autograd.Function):
    """E(coords) with dE/dcoords from the analytic gradient.

    forward(coords (n_atoms, 3) float64 tensor, atoms tuple, options dict) -> scalar energy."""

    @staticmethod
    def forward(ctx, coords: torch.Tensor, atoms, options):
        E, g = energy_and_gradient(list(atoms), coords.detach().cpu().numpy(), **(options or {}))
        ctx.save_for_backward(torch.as_tensor(g, dtype=coords.dtype, device=coords.device))
        return torch.tensor(E, dtype=coords.dtype, device=coords.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None


def rhf_energy(coords: torch.Tensor, atoms: Sequence[str], **options) -> torch.Tensor:
    """Differentiable RHF/STO-3G energy of a geometry (bohr)."""
    return RHFEnergy.apply(coords, tuple(atoms), options)
