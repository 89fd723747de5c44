"""The public surface: every name jht exports (jht tests/test_api.py:21-40) is present and
callable here, and the re-exports are the implementing objects (no CPU or GPU work)."""

from __future__ import annotations

import jht_b200 as jhtb
from jht_b200 import _analysis, diff, healpix, masked, offgrid, weights

JHT_SURFACE = {
    "synthesis", "adjoint_synthesis", "analysis", "map2alm", "bare_analysis",
    "synthesis_general", "adjoint_synthesis_general",
    "ring_weights", "pixel_weights", "pseudo_alm", "deconvolve",
    "wiener", "constrained_realization",
    "synthesis_real", "analysis_real",
    "synthesis_general_real", "adjoint_synthesis_general_real",
    "bandpower",
    "alm_to_real", "real_to_alm", "n_dof", "alm_size", "alm_metric_weight",
    "enable_compilation_cache",
    "set_azimuth_fft_mode", "get_azimuth_fft_mode", "enable_looped_fft",
}


def test_every_jht_name_is_exported_and_callable():
    advertised = set(jhtb.__all__) - {"__version__"}
    assert JHT_SURFACE <= advertised
    for name in advertised:
        assert callable(getattr(jhtb, name)), name


def test_reexports_are_the_implementations():
    assert jhtb.synthesis is healpix.synthesis
    assert jhtb.adjoint_synthesis is healpix.adjoint_synthesis
    assert jhtb.synthesis_general is offgrid.synthesis_general
    assert jhtb.adjoint_synthesis_general is offgrid.adjoint_synthesis_general
    assert jhtb.analysis is _analysis.analysis
    assert jhtb.map2alm is jhtb.analysis
    assert jhtb.bare_analysis is _analysis.bare_analysis
    assert jhtb.ring_weights is weights.ring_weights
    assert jhtb.pixel_weights is weights.pixel_weights
    assert jhtb.deconvolve is masked.deconvolve
    assert jhtb.synthesis_real is diff.synthesis_real
    assert jhtb.synthesis_general_real is diff.synthesis_general_real
    assert jhtb.alm_to_real is masked.alm_to_real
