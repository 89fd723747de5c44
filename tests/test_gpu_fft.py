"""The library's FFT kernel (jhtb_fft_c2c, used by the off-grid transforms) against NumPy.

Batched complex FP64 transforms of 2,3,5-smooth lengths along either axis of a 2-D array,
both signs, with scaling; lengths above the shared-memory limit run as two batched calls
(four-step, which also exercises the kernel's strides and twiddle).  The tolerance is
the FFT's own FP64 rounding (max |error| / max |value| <= 1e-13).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU hosts
    pytest.skip("no CUDA device", allow_module_level=True)

from jht_b200 import _fft  # noqa: E402

TOL = 1e-13


def _ref(x, dim, sign, scale):
    n = x.shape[dim]
    y = np.fft.fft(x, axis=dim) if sign < 0 else np.fft.ifft(x, axis=dim) * n
    return y * scale


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 9, 25, 60, 243, 625, 1000, 2160, 4320, 8640, 10240])
@pytest.mark.parametrize("dim", [0, 1])
def test_fft_matches_numpy(n, dim):
    rng = np.random.default_rng(n + 7 * dim)
    other = 5 if n > 1000 else 17
    shape = (n, other) if dim == 0 else (other, n)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    xt = torch.as_tensor(x, device="cuda")
    for sign, scale in ((-1, 1.0), (1, 1.0 / max(n, 1)), (-1, 0.5)):
        got = _fft.fft(xt, dim, sign, scale).cpu().numpy()
        ref = _ref(x, dim, sign, scale)
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err <= TOL, (n, dim, sign, err)


@pytest.mark.parametrize("n", [12288, 17280, 30000])
@pytest.mark.parametrize("dim", [0, 1])
def test_four_step_matches_numpy(n, dim):
    """Lengths above the shared-memory limit (two batched calls with the four-step twiddle)."""
    rng = np.random.default_rng(n + dim)
    shape = (n, 3) if dim == 0 else (3, n)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    xt = torch.as_tensor(x, device="cuda")
    for sign in (-1, 1):
        got = _fft.fft(xt, dim, sign).cpu().numpy()
        ref = _ref(x, dim, sign, 1.0)
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= TOL, (n, dim, sign)


@pytest.mark.parametrize("n", [60, 8640, 17280])
def test_fft_without_a_roots_table(n, monkeypatch):
    """A NULL roots table: each butterfly computes its root (one sincospi)."""

    class _Null:
        def data_ptr(self):
            return 0

    monkeypatch.setattr(_fft, "_roots", lambda n, device: _Null())
    rng = np.random.default_rng(n)
    x = rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))
    got = _fft.fft(torch.as_tensor(x, device="cuda"), 1, -1).cpu().numpy()
    ref = _ref(x, 1, -1, 1.0)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= TOL


def test_fft_rejects_unsupported_lengths():
    x = torch.zeros((7, 3), dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError, match="smooth"):
        _fft.fft(x, 0, -1)
