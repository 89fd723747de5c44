"""Differentiable real-DOF layer (drop-in for jht's ``diff`` module, src/jht/diff.py:55-138).

``synthesis_real = S o T^-1`` and ``analysis_real = T o analysis`` are plain
R^n -> R^m maps; their torch gradients come from the hand-written backward of
S (built from S^T) and of S^T (built from S) in :mod:`jht_b200.healpix`.
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np
import torch

from ._analysis import analysis
from .healpix import alm_metric_weight, synthesis
from .masked import alm_to_real, n_dof, real_to_alm
from .offgrid import adjoint_synthesis_general, synthesis_general

__all__ = ["synthesis_real", "analysis_real", "synthesis_general_real", "adjoint_synthesis_general_real", "bandpower",
           "alm_to_real", "real_to_alm", "n_dof"]


def synthesis_real(x, nside: int, lmax: int, spin: int = 0, *, precision: str = "fp64") -> torch.Tensor:
    """``S o T^-1``: real DOF vector (length ``n_dof(lmax, spin)``) -> map (diff.py:55-61)."""
    return synthesis(real_to_alm(x, lmax, spin), nside, lmax, spin, precision=precision)


def analysis_real(maps, nside: int, lmax: int, spin: int = 0, niter: int = 3, use_weights: bool = True, *,
                  precision: str = "fp64") -> torch.Tensor:
    """``T o analysis``: map -> real DOF vector (diff.py:64-72)."""
    a = analysis(maps, nside, lmax, spin=spin, niter=niter, use_weights=use_weights, precision=precision)
    return alm_to_real(a, lmax, spin)


def synthesis_general_real(x, loc, *, spin: int = 0, lmax: int, epsilon: float = 1e-10) -> torch.Tensor:
    """``S_g o T^-1``: real DOF vector -> field at the points ``loc`` (diff.py:79-92); a plain
    real-linear map, differentiable in ``x`` and ``loc``."""
    return synthesis_general(real_to_alm(x, lmax, spin), loc, spin=spin, lmax=lmax, epsilon=epsilon)


def adjoint_synthesis_general_real(field, loc, *, spin: int = 0, lmax: int, epsilon: float = 1e-10) -> torch.Tensor:
    """``T o S_g^T``: field at ``loc`` -> real DOF vector, the Euclidean transpose of
    :func:`synthesis_general_real` (diff.py:95-107)."""
    return alm_to_real(adjoint_synthesis_general(field, loc, spin=spin, lmax=lmax, epsilon=epsilon), lmax, spin)


@lru_cache(maxsize=None)
def _ell_of_idx(lmax: int) -> np.ndarray:
    return np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])


def bandpower(alm, lmax: int, spin: int = 0) -> torch.Tensor:
    """``C_l = (2l+1)^-1 sum_m (2 - delta_m0) |a_lm|^2`` (diff.py:119-138)."""
    a = alm if isinstance(alm, torch.Tensor) else torch.as_tensor(np.asarray(alm))
    dev = a.device
    ells = torch.as_tensor(_ell_of_idx(lmax), device=dev)
    wgt = torch.as_tensor(np.array(alm_metric_weight(lmax)), device=dev)
    norm = 1.0 / (2.0 * torch.arange(lmax + 1, device=dev, dtype=torch.float64) + 1.0)

    def one(v):
        p = wgt * v.abs() ** 2
        return torch.zeros(lmax + 1, dtype=torch.float64, device=dev).index_add(0, ells, p) * norm

    return one(a) if spin == 0 else torch.stack([one(a[0]), one(a[1])])
