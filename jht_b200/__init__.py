"""jht_b200 -- B200-native (sm_100a) on-grid HEALPix spherical-harmonic transforms.

A drop-in for the on-grid path of jht (src/jht/__init__.py): the same names,
signatures and conventions, running hand-written CUDA kernels through the
``jhtb`` C ABI (include/jhtb.h) with torch tensors at the boundary.

    import jht_b200 as jht
    m = jht.synthesis(alm, nside, lmax, spin=0)        # a_lm -> map
    a = jht.analysis(m, nside, lmax, spin=0, niter=3)  # map -> a_lm

Out of scope here (not provided): the off-grid NUFFT transforms.
"""

from __future__ import annotations

from ._analysis import analysis, bare_analysis, map2alm
from ._azimuth import enable_looped_fft, get_azimuth_fft_mode, set_azimuth_fft_mode
from ._cache import enable_compilation_cache
from .diff import adjoint_synthesis_general_real, analysis_real, bandpower, synthesis_general_real, synthesis_real
from .healpix import (
    adjoint_synthesis,
    adjoint_synthesis_batch,
    alm_metric_weight,
    alm_size,
    synthesis,
    synthesis_batch,
)
from .masked import (
    alm_to_real,
    constrained_realization,
    deconvolve,
    deconvolve_batch,
    n_dof,
    pseudo_alm,
    real_to_alm,
    wiener,
    wiener_batch,
)
from .offgrid import adjoint_synthesis_general, synthesis_general
from .weights import pixel_weights, ring_weights

__version__ = "0.1.0"

__all__ = [
    "__version__",
    "synthesis",
    "adjoint_synthesis",
    "analysis",
    "map2alm",
    "bare_analysis",
    "ring_weights",
    "pixel_weights",
    "pseudo_alm",
    "deconvolve",
    "wiener",
    "constrained_realization",
    "synthesis_general",
    "adjoint_synthesis_general",
    "synthesis_real",
    "analysis_real",
    "synthesis_general_real",
    "adjoint_synthesis_general_real",
    "bandpower",
    "alm_to_real",
    "real_to_alm",
    "n_dof",
    "alm_size",
    "alm_metric_weight",
    "enable_compilation_cache",
    "set_azimuth_fft_mode",
    "get_azimuth_fft_mode",
    "enable_looped_fft",
    # extensions beyond jht's surface
    "synthesis_batch",
    "adjoint_synthesis_batch",
    "deconvolve_batch",
    "wiener_batch",
]
