"""Parity at the full benchmark size (nside 2048, lmax 4096) on a B200, against an
extended-precision arbiter.

Two FP64 evaluations of the degree-4096 recursion -- jht's own log-renormalised form
(the oracle) and the kernels' scaled normalised form -- both round, and near the poles
each lands about 1e-12 of the map's maximum away from the exact transform.  Which side
carries a difference is decided by the arbiter: the oracle's algorithm carried out in
80-bit long double (``oracle/legendre_ref.c``, ``extended=True``), 2048 times finer than
FP64.  Every check below measures the CUDA path's error against the arbiter and the
oracle's error against the arbiter on the same entries, and requires the CUDA path to
be within 1e-12 of the arbiter or within twice the error of jht's own FP64 algorithm.

* full-band synthesis: the seeded benchmark input (all l, m) on 46 sampled rings
  (both poles, caps, belt, equator), the Legendre stage evaluated by the arbiter at
  those rings only;
* full-band adjoint: a map that is non-zero on the same sampled rings, all a_lm;
* m-subset adjoint of a full random map (every ring contributes) on m columns at the
  low, middle and high end;
* the inner-product identity <S a, v> = <a, S^T v>_G on the whole band, and the VJP
  against central differences on 64 real-DOF directions.
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

NSIDE, LMAX = 2048, 4096
T = 2 * NSIDE
M_RANGES = [(0, 4), (1501, 1505), (4090, 4097)]
# Accept the CUDA path if it is within ABS_TOL of the arbiter, or within SLACK times the
# FP64 oracle's distance to it: two FP64 evaluations of different algorithms round
# independently, and on B200 runs the CUDA/oracle ratio over these five checks ranged
# 0.47 .. 1.8 (the CUDA path the more accurate in three of them); both stay below
# MAX_ERR, a few 1e-11 of the largest value, at this degree.
ABS_TOL = 1e-12
SLACK = 2.0
MAX_ERR = 3e-11


def _half_rings():
    """Sampled half-grid rings: the polar ones, a geometric spread, the equator region."""
    t = np.concatenate([np.arange(8), np.geomspace(8, T - 1, 12).astype(int), [NSIDE - 1, NSIDE, T - 2, T - 1]])
    return np.unique(t)


def _full_rings(half):
    out = []
    for t in half:
        out.append(int(t))
        if t < T - 1:
            out.append(4 * NSIDE - 2 - int(t))
    return sorted(out)


def _config_alm(spin):
    """The benchmark's seeded input: E with C_l = 1/(l+10)^2, B 0.1/(l+10)^2, l < 2 zero."""
    rng = np.random.default_rng(1234)
    ell, _ = O.lm_of_index(LMAX)
    out = []
    for amp in (1.0, 0.1):
        cl = amp / (ell + 10.0) ** 2
        g1, g2 = rng.standard_normal(ell.size), rng.standard_normal(ell.size)
        a = np.sqrt(cl / 2.0) * (g1 + 1j * g2)
        a[: LMAX + 1] = np.sqrt(cl[: LMAX + 1]) * g1[: LMAX + 1]
        if spin == 2:
            a[ell < 2] = 0.0
        out.append(a)
    return np.stack(out) if spin == 2 else out[0][None, :]


def _ring_samples(parts, col, geo, r, spin):
    """RING samples of ring r from half-grid Legendre sums (oracle layout) at column col[t]."""
    m = np.arange(LMAX + 1)
    north = r < T
    c = col[r if north else 4 * NSIDE - 2 - r]
    sgn = 1.0 if north else (-1.0) ** m
    ph = np.exp(1j * m * geo.phi0[r])
    if spin == 0:
        Gp = Gm = sgn * (parts[0][:, c] if north else parts[1][:, c]) * ph
    else:
        Gp = sgn * (parts[0][:, c] if north else parts[1][:, c]) * ph
        Gm = sgn * (parts[2][:, c] if north else parts[3][:, c]) * ph
    N = int(geo.nring[r])
    D = np.zeros(N, np.complex128)
    np.add.at(D, m % N, Gp)
    np.add.at(D, (-m[1:]) % N, np.conj(Gm[1:]))
    y = np.fft.ifft(D) * N
    return y.real[None, :] if spin == 0 else np.stack([y.real, y.imag])


def _errors(got, fp64, arb):
    den = max(float(np.max(np.abs(arb))), 1e-300)
    return float(np.max(np.abs(got - arb))) / den, float(np.max(np.abs(fp64 - arb))) / den


def _check(name, e_gpu, e_orc):
    print(f"{name}: CUDA vs arbiter {e_gpu:.3e}, jht FP64 algorithm vs arbiter {e_orc:.3e}")
    assert e_gpu <= max(ABS_TOL, SLACK * e_orc), (name, e_gpu, e_orc)
    assert e_gpu <= MAX_ERR and e_orc <= MAX_ERR, (name, e_gpu, e_orc)


@pytest.mark.parametrize("spin", [2, 0])
def test_full_band_synthesis_vs_arbiter(spin):
    geo = O.Rings(NSIDE)
    half = _half_rings()
    col = {int(t): k for k, t in enumerate(half)}
    x = geo.z[half]
    a = _config_alm(spin)
    ref = _cref.load()
    arb = ref.synth(spin, LMAX, x, a, extended=True)
    f64 = ref.synth(spin, LMAX, x, a)
    got = jhtb.synthesis(a[0] if spin == 0 else a, NSIDE, LMAX, spin).cpu().numpy().reshape(-1, geo.npix)
    G, E, F = [], [], []
    for r in _full_rings(half):
        s, N = int(geo.start[r]), int(geo.nring[r])
        G.append(got[:, s : s + N])
        E.append(_ring_samples(arb, col, geo, r, spin))
        F.append(_ring_samples(f64, col, geo, r, spin))
    e_gpu, e_orc = _errors(np.concatenate(G, 1), np.concatenate(F, 1), np.concatenate(E, 1))
    _check(f"synthesis spin {spin}", e_gpu, e_orc)


def _ring_inputs(d, geo, rings, col, ncol, spin):
    """Half-grid adjoint inputs (oracle layout) of the rings' forward DFTs."""
    M = LMAX + 1
    m = np.arange(M)
    z = d[0] if spin == 0 else d[0] + 1j * d[1]
    V = [np.zeros((M, ncol), np.complex128) for _ in range(2 if spin == 0 else 4)]
    for r in rings:
        N, s = int(geo.nring[r]), int(geo.start[r])
        W = np.fft.fft(z[s : s + N].astype(np.complex128))
        ph = np.exp(-1j * m * geo.phi0[r])
        wp = W[m % N] * ph
        wm = np.conj(W[(-m) % N]) * ph
        if r < T:
            c = col[r]
            V[0][:, c] = wp
            if spin == 2:
                V[2][:, c] = wm
        else:
            c = col[4 * NSIDE - 2 - r]
            sg = (-1.0) ** m
            V[1][:, c] = sg * wp
            if spin == 2:
                V[3][:, c] = sg * wm
    return V


def _alm_from_parts(parts, spin):
    if spin == 0:
        return parts[0][None, :]
    p2, m2 = parts
    return np.stack([0.5 * (-p2 - m2), 0.5 * (1j * p2 - 1j * m2)])


@pytest.mark.parametrize("spin", [2, 0])
def test_full_band_adjoint_vs_arbiter(spin):
    """S^T of a map that is non-zero on the sampled rings only: every (l, m) is exercised."""
    geo = O.Rings(NSIDE)
    half = _half_rings()
    col = {int(t): k for k, t in enumerate(half)}
    rings = _full_rings(half)
    rng = np.random.default_rng(77 + spin)
    d = np.zeros((1 if spin == 0 else 2, geo.npix))
    for r in rings:
        s, N = int(geo.start[r]), int(geo.nring[r])
        d[:, s : s + N] = rng.standard_normal((d.shape[0], N))
    V = _ring_inputs(d, geo, rings, col, len(half), spin)
    ref = _cref.load()
    x = geo.z[half]
    arb = _alm_from_parts(ref.adjoint(spin, LMAX, x, V, extended=True), spin)
    f64 = _alm_from_parts(ref.adjoint(spin, LMAX, x, V), spin)
    got = jhtb.adjoint_synthesis(d[0] if spin == 0 else d, NSIDE, LMAX, spin).cpu().numpy().reshape(arb.shape)
    e_gpu, e_orc = _errors(got, f64, arb)
    _check(f"adjoint spin {spin}", e_gpu, e_orc)


def test_m_subset_adjoint_vs_arbiter():
    """S^T of a full random map on the m columns of M_RANGES: all 4096 rings contribute."""
    spin = 2
    rng = np.random.default_rng(7)
    geo = O.Rings(NSIDE)
    d = rng.standard_normal((2, geo.npix))
    got = jhtb.adjoint_synthesis(d, NSIDE, LMAX, spin).cpu().numpy()
    ms = np.concatenate([np.arange(lo, hi) for lo, hi in M_RANGES])
    M = LMAX + 1
    V = [np.zeros((M, T), np.complex128) for _ in range(4)]
    z = d[0] + 1j * d[1]
    sign = (-1.0) ** ms
    for N in np.unique(geo.nring):
        rows = np.flatnonzero(geo.nring == N)
        pix = geo.start[rows][:, None] + np.arange(N)[None, :]
        W = np.fft.fft(z[pix], axis=1)
        ph = np.exp(-1j * ms[None, :] * geo.phi0[rows][:, None])
        wp, wm = W[:, ms % N] * ph, np.conj(W[:, (-ms) % N]) * ph
        for k, r in enumerate(rows):
            if r < T:
                V[0][ms, r], V[2][ms, r] = wp[k], wm[k]
            else:
                t = 4 * NSIDE - 2 - r
                V[1][ms, t], V[3][ms, t] = sign * wp[k], sign * wm[k]
    ref = _cref.load()
    x = geo.z[:T]
    K = O.alm_size(LMAX)
    arb = np.zeros((2, K), np.complex128)
    f64 = np.zeros((2, K), np.complex128)
    for lo, hi in M_RANGES:
        arb += _alm_from_parts(ref.adjoint(2, LMAX, x, V, lo, hi, extended=True), 2)
        f64 += _alm_from_parts(ref.adjoint(2, LMAX, x, V, lo, hi), 2)
    idx = np.concatenate([O.alm_base(m, LMAX) + np.arange(LMAX + 1 - m) for m in ms])
    e_gpu, e_orc = _errors(got[:, idx], f64[:, idx], arb[:, idx])
    _check("adjoint m-subset, all rings", e_gpu, e_orc)


def test_inner_product_identity_full_size():
    spin = 2
    gen = torch.Generator("cuda").manual_seed(5)
    K = jhtb.alm_size(LMAX)
    ell = torch.as_tensor(np.concatenate([np.arange(m, LMAX + 1) for m in range(LMAX + 1)]), device="cuda")
    a = torch.complex(torch.randn((2, K), dtype=torch.float64, device="cuda", generator=gen),
                      torch.randn((2, K), dtype=torch.float64, device="cuda", generator=gen)) / (ell + 10.0)
    a[:, : LMAX + 1] = a[:, : LMAX + 1].real.to(torch.complex128)
    a[:, ell < 2] = 0
    v = torch.randn((2, 12 * NSIDE * NSIDE), dtype=torch.float64, device="cuda", generator=gen)
    lhs = float(torch.sum(jhtb.synthesis(a, NSIDE, LMAX, spin) * v))
    b = jhtb.adjoint_synthesis(v, NSIDE, LMAX, spin)
    G = torch.as_tensor(jhtb.alm_metric_weight(LMAX).copy(), device="cuda")
    rhs = float(torch.sum(G * torch.real(torch.conj(a) * b)))
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_vjp_matches_fd_on_64_real_dof_directions_full_size():
    """Loss 0.5 |S a - d|^2 at nside 2048, lmax 4096, spin 2: the torch VJP against central
    differences along 64 seeded real-DOF directions (the loss is quadratic, so the
    central difference is exact up to rounding; tolerance 1e-6 as jht's FD gates)."""
    spin = 2
    gen = torch.Generator("cuda").manual_seed(64)
    K = jhtb.alm_size(LMAX)
    ell = torch.as_tensor(np.concatenate([np.arange(m, LMAX + 1) for m in range(LMAX + 1)]), device="cuda")
    amp = torch.stack([1.0 / (ell + 10.0), 0.3162 / (ell + 10.0)])
    a = torch.complex(torch.randn((2, K), dtype=torch.float64, device="cuda", generator=gen),
                      torch.randn((2, K), dtype=torch.float64, device="cuda", generator=gen)) * amp
    a[:, : LMAX + 1] = a[:, : LMAX + 1].real.to(torch.complex128)
    a[:, ell < 2] = 0
    d = torch.randn((2, 12 * NSIDE * NSIDE), dtype=torch.float64, device="cuda", generator=gen)

    def loss(x):
        return 0.5 * torch.sum((jhtb.synthesis(x, NSIDE, LMAX, spin) - d) ** 2)

    ar = a.clone().requires_grad_(True)
    loss(ar).backward()
    grad = ar.grad.detach()
    m0 = torch.zeros(K, dtype=torch.bool, device="cuda")
    m0[: LMAX + 1] = True
    live = (ell >= 2)
    worst = 0.0
    for k in range(64):
        # a real-DOF direction: real parts on m = 0, both parts elsewhere, nothing below l = 2
        u = torch.complex(torch.randn((2, K), dtype=torch.float64, device="cuda", generator=gen),
                          torch.randn((2, K), dtype=torch.float64, device="cuda", generator=gen))
        u = torch.where(m0, torch.complex(u.real, torch.zeros_like(u.real)), u) * live
        u = u / torch.sqrt(torch.sum(torch.abs(u) ** 2))
        h = 1.0
        fd = (float(loss(a + h * u)) - float(loss(a - h * u))) / (2 * h)
        an = float(torch.sum(grad.real * u.real + grad.imag * u.imag))
        worst = max(worst, abs(fd - an) / max(1.0, abs(an)))
    assert worst <= 1e-6, worst
