"""Synthesis and adjoint at nside 4096 (small lmax) against the C oracle on sampled rings.

At nside 4096 the azimuthal stage takes its longest paths: the belt rings (16384 points) run
as four power-of-two pieces and the long polar-cap rings (chirp-z lengths above 16384) as
Bluestein transforms split through the ring scratch rows.  The oracle's Legendre sums are
evaluated only at the sampled rings and assembled with NumPy FFTs per ring.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import jht_b200 as jhtb  # noqa: E402
from oracle import _cref  # noqa: E402
from oracle import jht_oracle as O  # noqa: E402

NSIDE, LMAX = 4096, 96
T = 2 * NSIDE
TOL = 1e-12


def _half_rings():
    # poles, short and long caps (chirp-z in one CTA / in pieces / through scratch rows), belt
    t = np.concatenate([np.arange(4), [100, 1000, 2047, 2048, 2300, 3000, 4094, 4095, 4096, 6000, T - 2, T - 1]])
    return np.unique(t)


def _full_rings(half):
    out = []
    for t in half:
        out.append(int(t))
        if t < T - 1:
            out.append(4 * NSIDE - 2 - int(t))
    return sorted(out)


def _alm(spin, seed):
    rng = np.random.default_rng(seed)
    ell, _ = O.lm_of_index(LMAX)
    out = []
    for _ in range(2 if spin == 2 else 1):
        a = (rng.standard_normal(ell.size) + 1j * rng.standard_normal(ell.size)) / (ell + 10.0)
        a[: LMAX + 1] = a[: LMAX + 1].real
        if spin == 2:
            a[ell < 2] = 0.0
        out.append(a)
    return np.stack(out)


def _ring_samples(parts, col, geo, r, spin):
    m = np.arange(LMAX + 1)
    north = r < T
    c = col[r if north else 4 * NSIDE - 2 - r]
    sgn = 1.0 if north else (-1.0) ** m
    ph = np.exp(1j * m * geo.phi0[r])
    Gp = sgn * (parts[0][:, c] if north else parts[1][:, c]) * ph
    Gm = Gp if spin == 0 else sgn * (parts[2][:, c] if north else parts[3][:, c]) * ph
    N = int(geo.nring[r])
    D = np.zeros(N, np.complex128)
    np.add.at(D, m % N, Gp)
    np.add.at(D, (-m[1:]) % N, np.conj(Gm[1:]))
    y = np.fft.ifft(D) * N
    return y.real[None, :] if spin == 0 else np.stack([y.real, y.imag])


@pytest.mark.parametrize("spin", [2, 0])
def test_synthesis_at_nside4096_on_sampled_rings(spin):
    geo = O.Rings(NSIDE)
    half = _half_rings()
    col = {int(t): k for k, t in enumerate(half)}
    a = _alm(spin, 40 + spin)
    parts = _cref.load().synth(spin, LMAX, geo.z[half], a)
    m = jhtb.synthesis(a[0] if spin == 0 else a, NSIDE, LMAX, spin).reshape(-1, geo.npix)
    got, ref = [], []
    for r in _full_rings(half):
        s, N = int(geo.start[r]), int(geo.nring[r])
        got.append(m[:, s : s + N].cpu().numpy())
        ref.append(_ring_samples(parts, col, geo, r, spin))
    got, ref = np.concatenate(got, 1), np.concatenate(ref, 1)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= TOL


@pytest.mark.parametrize("spin", [2, 0])
def test_adjoint_at_nside4096_on_sampled_rings(spin):
    """S^T of a map that is non-zero on the sampled rings only."""
    geo = O.Rings(NSIDE)
    half = _half_rings()
    col = {int(t): k for k, t in enumerate(half)}
    rings = _full_rings(half)
    rng = np.random.default_rng(50 + spin)
    nc = 1 if spin == 0 else 2
    d = torch.zeros((nc, geo.npix), dtype=torch.float64, device="cuda")
    M = LMAX + 1
    mm = np.arange(M)
    V = [np.zeros((M, len(half)), np.complex128) for _ in range(2 if spin == 0 else 4)]
    for r in rings:
        s, N = int(geo.start[r]), int(geo.nring[r])
        v = rng.standard_normal((nc, N))
        d[:, s : s + N] = torch.as_tensor(v, device="cuda")
        z = v[0] if spin == 0 else v[0] + 1j * v[1]
        W = np.fft.fft(z.astype(np.complex128))
        ph = np.exp(-1j * mm * geo.phi0[r])
        wp, wm = W[mm % N] * ph, np.conj(W[(-mm) % N]) * ph
        if r < T:
            V[0][:, col[r]] = wp
            if spin == 2:
                V[2][:, col[r]] = wm
        else:
            c, sg = col[4 * NSIDE - 2 - r], (-1.0) ** mm
            V[1][:, c] = sg * wp
            if spin == 2:
                V[3][:, c] = sg * wm
    parts = _cref.load().adjoint(spin, LMAX, geo.z[half], V)
    ref = parts[0][None, :] if spin == 0 else np.stack([0.5 * (-parts[0] - parts[1]), 0.5 * (1j * parts[0] - 1j * parts[1])])
    got = jhtb.adjoint_synthesis(d[0] if spin == 0 else d, NSIDE, LMAX, spin).cpu().numpy().reshape(ref.shape)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= TOL
