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


_REQ = object()  # no default

# jht v0.2.0's signatures: name -> (positional parameters with defaults, keyword-only parameters
# with defaults); the source line of each def is given beside it.
JHT_SIGNATURES = {
    "synthesis": ({"alm": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0}, {}),  # healpix.py:363
    "adjoint_synthesis": ({"m": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0}, {}),  # healpix.py:390
    "synthesis_general": ({"alm": _REQ, "loc": _REQ}, {"spin": 0, "lmax": _REQ, "epsilon": 1e-10}),  # offgrid.py:172
    "adjoint_synthesis_general": ({"field": _REQ, "loc": _REQ},
                                  {"spin": 0, "lmax": _REQ, "epsilon": 1e-10}),  # offgrid.py:215
    "analysis": ({"maps": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0, "niter": 3, "use_weights": True},
                 {}),  # _analysis.py:55
    "bare_analysis": ({"maps": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0, "use_weights": True},
                      {}),  # _analysis.py:49
    "ring_weights": ({"nside": _REQ}, {}),  # weights.py:61
    "pixel_weights": ({"nside": _REQ, "use_weights": True}, {}),  # weights.py:87
    "pseudo_alm": ({"maps": _REQ, "mask": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0, "niter": 3,
                    "use_weights": True}, {}),  # masked.py:99
    "deconvolve": ({"maps": _REQ, "mask": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0},
                   {"max_iter": 200, "tol": 1e-8, "reg": 0.0, "use_weights": True, "x0": None}),  # masked.py:278
    "wiener": ({"maps": _REQ, "signal_cl": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0},
               {"inv_noise": None, "mask": None, "max_iter": 200, "tol": 1e-8, "use_weights": True,
                "x0": None}),  # masked.py:320
    "constrained_realization": ({"maps": _REQ, "signal_cl": _REQ, "nside": _REQ, "lmax": _REQ, "key": _REQ,
                                 "spin": 0},
                                {"inv_noise": None, "mask": None, "max_iter": 200, "tol": 1e-8,
                                 "use_weights": True, "x0": None}),  # masked.py:374
    "synthesis_real": ({"x": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0}, {}),  # diff.py:55
    "analysis_real": ({"maps": _REQ, "nside": _REQ, "lmax": _REQ, "spin": 0, "niter": 3, "use_weights": True},
                      {}),  # diff.py:64
    "synthesis_general_real": ({"x": _REQ, "loc": _REQ}, {"spin": 0, "lmax": _REQ, "epsilon": 1e-10}),  # diff.py:79
    "adjoint_synthesis_general_real": ({"field": _REQ, "loc": _REQ},
                                       {"spin": 0, "lmax": _REQ, "epsilon": 1e-10}),  # diff.py:95
    "bandpower": ({"alm": _REQ, "lmax": _REQ, "spin": 0}, {}),  # diff.py:119
    "alm_to_real": ({"alm": _REQ, "lmax": _REQ, "spin": 0}, {}),  # masked.py:160
    "real_to_alm": ({"x": _REQ, "lmax": _REQ, "spin": 0}, {}),  # masked.py:169
    "n_dof": ({"lmax": _REQ, "spin": 0}, {}),  # masked.py:140
    "alm_size": ({"lmax": _REQ}, {}),  # healpix.py:49
    "alm_metric_weight": ({"lmax": _REQ}, {}),  # healpix.py:59
    "enable_compilation_cache": ({"directory": _REQ}, {"min_compile_time_secs": 1.0}),  # _cache.py:25
    "set_azimuth_fft_mode": ({"mode": _REQ}, {}),  # _azimuth.py:60
    "get_azimuth_fft_mode": ({}, {}),  # _azimuth.py:82
    "enable_looped_fft": ({}, {}),  # _azimuth.py:87
}


def test_signatures_match_jht():
    """Every jht call still binds: the same positional parameters in the same order with the
    same defaults, the same keyword-only parameters with the same defaults.  Additions are
    allowed only as keyword-only parameters with a default (``precision``)."""
    import inspect

    sigs = dict(JHT_SIGNATURES, map2alm=JHT_SIGNATURES["analysis"])  # an alias of analysis in jht (_analysis.py:67)
    assert set(sigs) == JHT_SURFACE
    for name, (pos, kw) in sigs.items():
        params = inspect.signature(getattr(jhtb, name)).parameters.values()
        got_pos = {p.name: (_REQ if p.default is p.empty else p.default) for p in params
                   if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)}
        got_kw = {p.name: (_REQ if p.default is p.empty else p.default) for p in params
                  if p.kind == p.KEYWORD_ONLY}
        assert list(got_pos) == list(pos), name
        for k, d in pos.items():
            assert got_pos[k] is d if d is _REQ else got_pos[k] == d, (name, k)
        for k, d in kw.items():
            assert k in got_kw, (name, k)
            assert got_kw[k] is d if d is _REQ else got_kw[k] == d, (name, k)
        for k in set(got_kw) - set(kw):
            assert got_kw[k] is not _REQ, (name, k)


def test_input_validation_before_device_work():
    """Wrong-size inputs raise jht's errors (tests/test_healpix.py:138-149 and
    tests/test_diff_offgrid.py:138-151 of jht) before any device work, so they read the
    same on a host without a GPU."""
    import numpy as np
    import pytest

    nside, lmax = 16, 24
    K = jhtb.alm_size(lmax)
    with pytest.raises(ValueError, match="alm shape"):
        jhtb.synthesis(np.zeros(K - 1, dtype=np.complex128), nside, lmax, spin=0)
    with pytest.raises(ValueError, match="alm shape"):
        jhtb.synthesis(np.zeros(K, dtype=np.complex128), nside, lmax, spin=2)  # missing (2, K)
    with pytest.raises(ValueError, match="map shape"):
        jhtb.adjoint_synthesis(np.zeros(12 * nside**2 - 1), nside, lmax, spin=0)
    with pytest.raises(ValueError, match="map shape"):
        jhtb.adjoint_synthesis(np.zeros(12 * nside**2), nside, lmax, spin=2)  # missing (2, npix)

    L = 8
    rng = np.random.default_rng(700)
    loc = np.stack([rng.uniform(0, np.pi, 10), rng.uniform(0, 2 * np.pi, 10)], axis=1)
    alm = np.zeros(jhtb.alm_size(L), dtype=np.complex128)
    with pytest.raises(ValueError, match="alm shape"):
        jhtb.synthesis_general(np.zeros(3, dtype=complex), loc, spin=0, lmax=L)
    with pytest.raises(ValueError, match="loc must"):
        jhtb.synthesis_general(alm, loc[:, :1], spin=0, lmax=L)
    with pytest.raises(ValueError, match="field shape"):
        jhtb.adjoint_synthesis_general(np.zeros(9), loc, spin=0, lmax=L)
    with pytest.raises(ValueError, match="field shape"):
        jhtb.adjoint_synthesis_general(np.zeros(10), loc, spin=2, lmax=L)  # missing (2, npts)
    with pytest.raises(TypeError, match="real"):
        jhtb.adjoint_synthesis_general(np.zeros(10, dtype=complex), loc, spin=0, lmax=L)


def test_band_ceiling_warning_before_device_work():
    """lmax > 1.5 nside warns once per geometry (jht tests/test_healpix.py:152-160); on a host
    without a GPU the call then fails loudly instead of falling back to the CPU."""
    import contextlib

    import numpy as np
    import pytest
    import torch

    a = np.zeros(jhtb.alm_size(8), dtype=np.complex128)  # 8 > 1.5 * 5; a geometry no other test uses
    no_gpu = not torch.cuda.is_available()
    with pytest.warns(UserWarning, match="ceiling"):
        with pytest.raises(RuntimeError, match="CUDA") if no_gpu else contextlib.nullcontext():
            jhtb.synthesis(a, 5, 8, spin=0)


def test_azimuth_mode_toggle_validation():
    """jht tests/test_azimuth_fft.py:224-228: a bad mode raises and leaves the mode unchanged;
    the shortcut selects "looped".  (Both modes run the same ring kernels here.)"""
    import pytest

    assert jhtb.get_azimuth_fft_mode() == "unrolled"
    with pytest.raises(ValueError, match="unknown azimuth FFT mode"):
        jhtb.set_azimuth_fft_mode("bogus")
    assert jhtb.get_azimuth_fft_mode() == "unrolled"
    try:
        jhtb.enable_looped_fft()
        assert jhtb.get_azimuth_fft_mode() == "looped"
    finally:
        jhtb.set_azimuth_fft_mode("unrolled")
