"""CPU-only checks of the boundary and the host-side logic (no GPU needed).

* the C-ABI library loads and exports every function ``include/jhtb.h`` declares;
* argument validation answers with a status code before any device work;
* the host seed tables, ring geometry, packing, metric, quadrature weights and the
  real-DOF isometry of the product package agree with the oracle and the golden
  vectors produced by the reference's own code;
* without a CUDA device the transforms raise instead of falling back to the CPU.
"""

from __future__ import annotations

import ctypes
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import ROOT, relerr

import jht_b200 as jhtb  # noqa: E402
from jht_b200 import _lib, healpix, masked, weights  # noqa: E402
from oracle import jht_oracle as O  # noqa: E402

HEADER = ROOT / "include" / "jhtb.h"


@pytest.fixture(scope="module")
def lib():
    if not _lib.LIB_PATH.exists():
        # incremental in-tree build (nvcc cross-compiles without a GPU)
        subprocess.run([sys.executable, "-m", "jht_b200.build"], cwd=ROOT, check=True)
    return _lib.load_library()


def _declared_functions() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return set(re.findall(r"\b(jhtb_[a-z0-9_]+)\s*\(", text))


def test_header_declares_exactly_the_binding_exports():
    assert _declared_functions() == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    raw = ctypes.CDLL(str(_lib.LIB_PATH))
    for name in sorted(_declared_functions()):
        assert hasattr(raw, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True, check=True)
    dyn = {ln.split()[-1] for ln in out.stdout.splitlines() if ln.strip()}
    assert _declared_functions() <= dyn
    # nothing else named jhtb_* leaks out of the shared object
    assert {s for s in dyn if s.startswith("jhtb_")} == _declared_functions()


def test_version_and_last_error(lib):
    assert lib.jhtb_version() == 100
    assert lib.jhtb_last_error(None, 0) == _lib.JHTB_ERR_INVALID


@pytest.mark.parametrize(
    "args,status,needle",
    [
        ((16, 24, 1, 0, 1), _lib.JHTB_ERR_UNSUPPORTED, "spin"),
        ((0, 24, 0, 0, 1), _lib.JHTB_ERR_INVALID, "nside"),
        ((8192, 24, 0, 0, 1), _lib.JHTB_ERR_INVALID, "nside"),
        ((16, -1, 0, 0, 1), _lib.JHTB_ERR_INVALID, "lmax"),
        ((16, 24, 0, 1, 1), _lib.JHTB_ERR_UNSUPPORTED, "FP32"),
        ((16, 24, 0, 7, 1), _lib.JHTB_ERR_INVALID, "precision"),
        ((16, 24, 0, 0, 0), _lib.JHTB_ERR_INVALID, "max_batch"),
    ],
)
def test_plan_create_validates_before_device_work(lib, args, status, needle):
    h = ctypes.c_void_p()
    assert lib.jhtb_plan_create(*args, None, ctypes.byref(h)) == status
    assert h.value is None
    assert needle in _lib.last_error()


def test_null_pointers_are_rejected(lib):
    assert lib.jhtb_plan_create(16, 24, 0, 0, 1, None, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_synthesis(None, None, None, 1, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_adjoint_synthesis(None, None, None, 1, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_plan_destroy(None) == _lib.JHTB_OK
    assert lib.jhtb_plan_set_watchdog(None, 10**9) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_plan_inject_fault(None, 1) == _lib.JHTB_ERR_INVALID
    i64, i32, dbl = ctypes.c_int64(), ctypes.c_int(), ctypes.c_double()
    ms, counts = (ctypes.c_double * 16)(), (ctypes.c_int64 * 16)()
    buf = ctypes.c_void_p(16)
    calls = {
        "jhtb_plan_bytes": lambda: lib.jhtb_plan_bytes(None, ctypes.byref(i64)),
        "jhtb_plan_status": lambda: lib.jhtb_plan_status(None, ctypes.byref(i32)),
        "jhtb_plan_timings": lambda: lib.jhtb_plan_timings(None, ms, counts, 0),
        "jhtb_plan_set_timing": lambda: lib.jhtb_plan_set_timing(None, 1),
        "jhtb_plan_set_tuning": lambda: lib.jhtb_plan_set_tuning(None, 0, 0),
        "jhtb_plan_ring_costs": lambda: lib.jhtb_plan_ring_costs(None, 4, ctypes.byref(i64), 1),
        "jhtb_plan_set_ring_range": lambda: lib.jhtb_plan_set_ring_range(None, 0, 4),
        "jhtb_weighted_residual": lambda: lib.jhtb_weighted_residual(None, buf, None, None, buf, 1, None),
        "jhtb_dot": lambda: lib.jhtb_dot(None, 4, buf, buf, buf, None),
        "jhtb_axpy": lambda: lib.jhtb_axpy(-1, 1.0, buf, buf, None),
        "jhtb_probe_fp64_fma": lambda: lib.jhtb_probe_fp64_fma(0, 1, buf, ctypes.byref(dbl), ctypes.byref(dbl), None),
    }
    for name, call in calls.items():
        assert call() == _lib.JHTB_ERR_INVALID, name
        assert name in _lib.last_error(), name
    assert lib.jhtb_axpy(4, 1.0, None, buf, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_axpy(0, 1.0, None, None, None) == _lib.JHTB_OK  # empty: nothing launched


@pytest.mark.parametrize("nside", [1, 4, 13, 64])
def test_geometry_matches_oracle(nside):
    g = healpix.RingInfo(nside)
    r = O.Rings(nside)
    np.testing.assert_array_equal(g.npix_ring, r.nring)
    np.testing.assert_array_equal(g.startpix, r.start)
    np.testing.assert_allclose(g.z, r.z, rtol=0, atol=0)
    np.testing.assert_allclose(g.phi0, r.phi0, rtol=0, atol=0)
    np.testing.assert_array_equal(_lib._half_grid_z(nside), r.z[: 2 * nside])


@pytest.mark.parametrize("lmax", [0, 1, 7, 100])
def test_packing_and_metric(lmax):
    assert jhtb.alm_size(lmax) == O.alm_size(lmax)
    for m in range(lmax + 1):
        assert healpix.alm_column_base(m, lmax) == O.alm_base(m, lmax)
    np.testing.assert_array_equal(jhtb.alm_metric_weight(lmax), O.metric_weight(lmax))


@pytest.mark.parametrize("nside,lmax", [(8, 12), (16, 40), (64, 128)])
def test_host_seed_tables_match_oracle(nside, lmax):
    t0 = _lib.host_tables(nside, lmax, 0)
    for m in range(lmax + 1):
        assert abs(t0["seed_logc"][m] - O.sectoral_log_const(m)) <= 1e-13 * max(1.0, abs(O.sectoral_log_const(m)))
    t2 = _lib.host_tables(nside, lmax, 2)
    for h, s in enumerate((2, -2)):
        for m in range(lmax + 1):
            lmin = max(m, 2)
            # at x = 0 both half-angle factors are sqrt(1/2) and their powers sum to 2 lmin
            _, logd = O.wigner_seed(np.zeros(1), -m, s, lmin)
            logc = float(logd[0]) + lmin * np.log(2.0)
            assert abs(t2["seed_logc"][h, m] - logc) <= 1e-12 * max(1.0, abs(logc)), (s, m)


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 12, 16, 32, 64])
def test_ring_weights_match_golden(golden, nside):
    np.testing.assert_allclose(weights.ring_weights(nside), golden[f"weights/ring_n{nside}"], rtol=0, atol=1e-12)


def test_pixel_weights_match_golden(golden):
    np.testing.assert_allclose(weights.pixel_weights(8), golden["weights/pix_n8"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(weights.pixel_weights(8, False), np.full(768, 4 * np.pi / 768), rtol=1e-15)


def test_real_dof_matches_golden_on_cpu(golden):
    x0 = masked.alm_to_real(torch.as_tensor(golden["real/a0"]), 12, 0)
    x2 = masked.alm_to_real(torch.as_tensor(golden["real/a2"]), 12, 2)
    np.testing.assert_array_equal(x0.numpy(), golden["real/x0"])
    np.testing.assert_array_equal(x2.numpy(), golden["real/x2"])
    np.testing.assert_allclose(masked.real_to_alm(x0, 12, 0).numpy(), golden["real/a0"], atol=1e-15)
    np.testing.assert_allclose(masked.real_to_alm(x2, 12, 2).numpy(), golden["real/a2"], atol=1e-15)
    assert jhtb.n_dof(12, 0) == golden["real/x0"].size
    assert jhtb.n_dof(12, 2) == golden["real/x2"].size


@pytest.mark.parametrize("lmax,spin", [(0, 0), (5, 0), (30, 0), (5, 2), (30, 2)])
def test_real_dof_is_an_isometry(lmax, spin):
    rng = np.random.default_rng(lmax + spin)
    n = jhtb.n_dof(lmax, spin)
    x = torch.as_tensor(rng.standard_normal(n))
    a = masked.real_to_alm(x, lmax, spin)
    back = masked.alm_to_real(a, lmax, spin)
    np.testing.assert_allclose(back.numpy(), x.numpy(), rtol=0, atol=1e-15)
    G = torch.as_tensor(np.array(jhtb.alm_metric_weight(lmax)))
    na = float(torch.sum(G * a.abs() ** 2))
    assert abs(na - float(torch.sum(x * x))) <= 1e-12 * max(1.0, na)
    # batch helpers used by the CG agree with the single-vector form
    xb = torch.stack([x, 2 * x])
    ab = masked._alm_batch(xb, lmax, spin)
    np.testing.assert_allclose(ab[0].reshape(a.shape).numpy(), a.numpy(), atol=0)
    np.testing.assert_allclose(masked._real_batch(ab, lmax, spin).numpy(), xb.numpy(), atol=1e-15)


def test_bandpower_matches_oracle():
    rng = np.random.default_rng(3)
    lmax = 20
    K = jhtb.alm_size(lmax)
    a = rng.standard_normal((2, K)) + 1j * rng.standard_normal((2, K))
    got = jhtb.bandpower(torch.as_tensor(a), lmax, 2).numpy()
    assert relerr(got, O.bandpower(a, lmax, 2)) <= 1e-14


def test_workspace_budget_caps_batch():
    per = _lib.workspace_bytes_per_map(2048, 4096, 2)
    assert per > 1 << 30
    assert _lib.workspace_bytes_per_map(64, 128, 0) < _lib.workspace_bytes_per_map(64, 128, 2)


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour on a host without CUDA")
def test_no_cpu_fallback():
    a = np.zeros(jhtb.alm_size(8), dtype=np.complex128)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        jhtb.synthesis(a, 8, 8, 0)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        jhtb.adjoint_synthesis(np.zeros(768), 8, 8, 0)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        jhtb.analysis(np.zeros(768), 8, 8, 0)


def test_ring_set_plan_validates_before_device_work(lib):
    x = np.array([1.0, 0.7, 0.2, 0.0])
    ht = _lib.HostTables(x.ctypes.data, None, None, None, None)
    h = ctypes.c_void_p()
    # even ring count, bad spin, missing x, increasing x
    assert lib.jhtb_plan_create_rings(8, 16, 0, 0, 1, ctypes.byref(ht), ctypes.byref(h)) == _lib.JHTB_ERR_INVALID
    assert "odd" in _lib.last_error()
    assert lib.jhtb_plan_create_rings(7, 16, 1, 0, 1, ctypes.byref(ht), ctypes.byref(h)) == _lib.JHTB_ERR_UNSUPPORTED
    assert lib.jhtb_plan_create_rings(7, 16, 0, 0, 1, None, ctypes.byref(h)) == _lib.JHTB_ERR_INVALID
    bad = np.array([0.2, 0.7, 1.0, 0.0])
    ht_bad = _lib.HostTables(bad.ctypes.data, None, None, None, None)
    assert lib.jhtb_plan_create_rings(7, 16, 0, 0, 1, ctypes.byref(ht_bad), ctypes.byref(h)) == _lib.JHTB_ERR_INVALID
    assert "non-increasing" in _lib.last_error()
    assert h.value is None


def test_nufft_calls_validate_before_device_work(lib):
    one = ctypes.c_void_p(16)  # never dereferenced: every call below fails its argument checks
    d = ctypes.c_double(1.0)
    assert lib.jhtb_nufft_interp(None, 8, 8, 14, d, None, None, 4, None, None, None, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_nufft_interp(one, 8, 8, 7, d, one, one, 4, one, None, None, None) == _lib.JHTB_ERR_UNSUPPORTED
    assert lib.jhtb_nufft_interp(one, 8, 8, 14, d, one, one, 4, one, one, None, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_nufft_spread(one, one, one, -1, 8, 8, 14, d, one, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_nufft_spread(one, one, one, 4, 0, 8, 14, d, one, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_nufft_spread_tiles(one, one, one, 4, 2, None, None, None, 4, 8, 8, 14, d, one, None) == \
        _lib.JHTB_ERR_INVALID
    assert lib.jhtb_nufft_spread_tiles(one, one, one, 4, -1, one, one, one, 4, 8, 8, 14, d, one, None) == \
        _lib.JHTB_ERR_INVALID
    assert lib.jhtb_legendre_synthesis(None, None, None, 1, None) == _lib.JHTB_ERR_INVALID
    assert lib.jhtb_legendre_adjoint(None, None, None, 1, None) == _lib.JHTB_ERR_INVALID


@pytest.mark.parametrize("nside", [2, 16, 128, 256, 512])
def test_product_ring_weights_make_m0_quadrature_exact(nside):
    """jht's weight gates (tests/test_weights.py:40-99): with the product's ring weights the
    m = 0 quadrature integrates every Legendre polynomial up to degree 2 nside to within
    1e-9 * 4 pi, the weights sum to 4 pi, and southern rings carry their north partner's
    weight."""
    from numpy.polynomial.legendre import legvander

    geo = healpix.RingInfo(nside)
    pw = weights.pixel_weights(nside)
    ring_w = np.add.reduceat(pw, geo.startpix)
    q = ring_w @ legvander(geo.z, 2 * nside)
    assert abs(q[0] - 4 * np.pi) < 1e-9 * 4 * np.pi
    assert np.max(np.abs(q[1:])) < 1e-9 * 4 * np.pi
    assert abs(pw.sum() - 4 * np.pi) < 1e-10
    per_ring = ring_w / geo.npix_ring
    np.testing.assert_array_equal(per_ring[: 2 * nside - 1], per_ring[::-1][: 2 * nside - 1])


def test_tuning_table_lookup(tmp_path):
    """The autotuner's table: exact entries, the largest tuned batch not above the
    requested one, no entry for other precisions or geometries, unknown knobs refused."""
    import json

    from jht_b200 import autotune as A

    t = {A.key(2048, 4096, 2, 16, "bf16x3"): {"knobs": {"tc_fold": 512, "tc_group": 16}},
         A.key(2048, 4096, 2, 4, "bf16x3"): {"knobs": {"tc_group": 8}},
         A.key(512, 1024, 0, 64, "fp64"): {"knobs": {"leg_ctas": 2}}}
    assert A.lookup(2048, 4096, 2, 16, "bf16x3", t) == {"tc_fold": 512, "tc_group": 16}
    assert A.lookup(2048, 4096, 2, 40, "bf16x3", t) == {"tc_fold": 512, "tc_group": 16}
    assert A.lookup(2048, 4096, 2, 8, "bf16x3", t) == {"tc_group": 8}
    assert A.lookup(2048, 4096, 2, 2, "bf16x3", t) == {}
    assert A.lookup(2048, 4096, 2, 16, "fp64", t) == {}
    assert A.lookup(512, 1024, 0, 64, "fp64", t) == {"leg_ctas": 2}
    p = tmp_path / "t.json"
    p.write_text(json.dumps(t))
    assert A.load_table(p) == t
    p.write_text(json.dumps({A.key(8, 12, 0, 1, "fp64"): {"knobs": {"warp_size": 3}}}))
    with pytest.raises(ValueError):
        A.load_table(p)
    # the committed table only holds known knobs, and every candidate is a valid setting
    A.load_table()
    for prec in ("fp64", "bf16x3"):
        for c in A.candidates(prec, 2):
            assert set(c) <= set(A.KNOBS)


def test_tuning_knobs_reject_null_plan(lib):
    assert lib.jhtb_plan_set_tuning(None, 1, 256) == _lib.JHTB_ERR_INVALID


def test_debug_library_exports_the_same_symbols():
    """The bounds-checked build (make debug) exports exactly the release library's entry points."""
    if not _lib.DEBUG_LIB_PATH.exists():
        pytest.skip("debug library not built")
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.DEBUG_LIB_PATH)], capture_output=True, text=True,
                         check=True)
    dyn = {ln.split()[-1] for ln in out.stdout.splitlines() if ln.strip()}
    assert {s for s in dyn if s.startswith("jhtb_")} == _declared_functions()


def test_release_debug_bounds_is_unsupported(lib):
    cnt, site, idx, ext = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
    rc = lib.jhtb_debug_bounds(ctypes.byref(cnt), ctypes.byref(site), ctypes.byref(idx), ctypes.byref(ext))
    assert rc == _lib.JHTB_ERR_UNSUPPORTED
    assert "debug library" in _lib.last_error()
    assert lib.jhtb_debug_bounds(None, None, None, None) == _lib.JHTB_ERR_INVALID


def test_fft_split_and_argument_checks(lib):
    """The four-step split of the off-grid FFT lengths, and the C entry point's argument
    checks (made before any device work)."""
    from jht_b200 import _fft

    for n in (12288, 17280, 30000, 34560, 102400):
        n1, n2 = _fft._split(n)
        assert n1 * n2 == n and n1 <= _fft.SM_MAX and n2 <= _fft.SM_MAX
        assert _fft._smooth(n1) and _fft._smooth(n2)
    buf = ctypes.c_void_p(16)
    args = (1, 1, 1, 1, 0, 1, 1, 0, -1, 1.0, 0, None, None)
    assert lib.jhtb_fft_c2c(buf, buf, 7, *args) == _lib.JHTB_ERR_INVALID      # not 2,3,5-smooth
    assert "smooth" in _lib.last_error()
    assert lib.jhtb_fft_c2c(buf, buf, 20480, *args) == _lib.JHTB_ERR_INVALID  # above the shared-memory limit
    assert lib.jhtb_fft_c2c(buf, buf, 8, 1, 1, 1, 1, 0, 1, 1, 0, 2, 1.0, 0, None, None) == _lib.JHTB_ERR_INVALID  # sign
    assert lib.jhtb_fft_c2c(None, buf, 8, *args) == _lib.JHTB_ERR_INVALID


def test_fft_four_step_composition_on_a_model_of_the_kernel(monkeypatch):
    """The host's four-step composition (strides, batch split, twiddle) run against a NumPy
    model of jhtb_fft_c2c's contract, for lengths above the shared-memory limit."""
    from jht_b200 import _fft

    mem = {}

    def model(x, out, n, howmany, inner, in_stride, in_do, in_di, out_stride, out_do, out_di, sign, scale, tw):
        src, dst = mem[x.data_ptr()], mem[out.data_ptr()]
        i = np.arange(n)
        for b in range(howmany):
            o, t = divmod(b, inner)
            v = src[o * in_do + t * in_di + i * in_stride]
            y = (np.fft.fft(v) if sign < 0 else np.fft.ifft(v) * n) * scale
            if tw:
                y = y * np.exp(sign * 2j * np.pi * ((t * i) % tw) / tw)
            dst[o * out_do + t * out_di + i * out_stride] = y

    class Buf:
        def __init__(self, arr):
            self.arr = arr.reshape(-1)
            mem[id(self)] = self.arr

        def data_ptr(self):
            return id(self)

    class T:  # a stand-in for a 2-D complex128 CUDA tensor
        def __init__(self, a):
            self.a = np.ascontiguousarray(a)
            self.buf = Buf(self.a)
            self.shape = a.shape
            self.dtype, self.is_cuda = torch.complex128, True

        def dim(self):
            return 2

        def contiguous(self):
            return self

        def numel(self):
            return self.a.size

        def data_ptr(self):
            return self.buf.data_ptr()

    monkeypatch.setattr(_fft, "_call", model)
    monkeypatch.setattr(_fft.torch, "empty_like", lambda x: T(np.zeros_like(x.a)))
    rng = np.random.default_rng(3)
    for n, other, dim in ((12288, 2, 0), (12288, 3, 1), (17280, 2, 1)):
        shape = (n, other) if dim == 0 else (other, n)
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        for sign in (-1, 1):
            got = _fft.fft(T(x), dim, sign, 0.5).a
            ref = (np.fft.fft(x, axis=dim) if sign < 0 else np.fft.ifft(x, axis=dim) * n) * 0.5
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12, (n, dim, sign)


def test_fft_roots_table_against_a_40_digit_reference():
    """The FFT kernel's table of roots of unity: exact symmetries, and each sampled entry
    within one FP64 ulp of e^{-2 pi i k / n} taken at 40 digits."""
    mpmath = pytest.importorskip("mpmath")
    from jht_b200 import _fft

    mpmath.mp.dps = 40
    for n in (1, 2, 3, 243, 625, 8640, 10240):
        z = _fft._roots_host(n)
        assert z.shape == (n,) and z.dtype == np.complex128 and z[0] == 1.0
        k = np.arange(1, n)
        assert np.array_equal(z[n - k], np.conj(z[k]))
        if n % 2 == 0:
            assert z[n // 2] == -1.0
        if n % 4 == 0:
            assert z[n // 4] == -1j and z[3 * n // 4] == 1j
        ks = np.unique(np.r_[np.arange(0, n, max(1, n // 499)), n - 1])
        ref = np.array([complex(mpmath.cos(2 * mpmath.pi * int(j) / n), -mpmath.sin(2 * mpmath.pi * int(j) / n))
                        for j in ks])
        assert np.max(np.abs(z[ks] - ref)) <= 1.2e-16, n


def _quadrature_moments(nside):
    """Q_l = sum over pixels of W_pix P_l(z_pix), l <= 2 nside, summed ring by ring (every
    pixel of a ring has the same z)."""
    from numpy.polynomial.legendre import legvander

    from jht_b200.healpix import RingInfo

    geo = RingInfo(nside)
    ring_w = np.add.reduceat(weights.pixel_weights(nside), geo.startpix)
    return ring_w @ legvander(geo.z, 2 * nside)


@pytest.mark.parametrize("nside", [2, 4, 8, 16, 32, 64, 128, 256, 512, 2048])
def test_ring_weight_properties(nside):
    """jht tests/test_weights.py:40-68: the ring weights are small corrections to 1, and with
    them the m = 0 quadrature integrates P_l exactly for even l <= 2 nside (Q_0 = 4 pi, the
    higher even moments vanish); up to the benchmark's nside 2048."""
    w = weights.ring_weights(nside)
    assert w.shape == (2 * nside,) and np.all(np.isfinite(w)) and np.max(np.abs(w)) < 0.5
    q = _quadrature_moments(nside)
    assert abs(q[0] - 4 * np.pi) < 1e-12 * 4 * np.pi
    assert np.max(np.abs(q[2::2])) < 1e-12 * 4 * np.pi


def test_pixel_weight_properties():
    """jht tests/test_weights.py:70-89: the pixel weights sum to 4 pi (with and without the
    ring weights), and a southern ring's pixels carry its northern partner's weight."""
    from jht_b200.healpix import RingInfo

    for nside in (4, 16, 64, 256):
        assert abs(weights.pixel_weights(nside).sum() - 4 * np.pi) < 1e-11
        w0 = weights.pixel_weights(nside, use_weights=False)
        assert np.allclose(w0, 4 * np.pi / (12 * nside**2)) and abs(w0.sum() - 4 * np.pi) < 1e-12
    nside = 32
    geo, wv = RingInfo(nside), weights.pixel_weights(nside)
    for r in (0, 5, 2 * nside - 2):
        assert abs(wv[geo.startpix[r]] - wv[geo.startpix[4 * nside - 2 - r]]) < 1e-15


def _rand_alm_host(lmax, spin, seed):
    rng = np.random.default_rng(seed)
    ell, _ = O.lm_of_index(lmax)
    out = []
    for _ in range(2 if spin == 2 else 1):
        a = rng.standard_normal(ell.size) + 1j * rng.standard_normal(ell.size)
        a[: lmax + 1] = a[: lmax + 1].real
        if spin == 2:
            a[ell < 2] = 0.0
        out.append(a)
    return out[0] if spin == 0 else np.stack(out)


@pytest.mark.parametrize("spin", [0, 2])
def test_real_dof_isometry(spin):
    """jht tests/test_masked.py:125-145: T^-1 T = I on packed a_lm, and ||T a||^2 equals the
    (2 - delta_m0)-weighted norm of a; n_dof is the length of T a."""
    lmax = 10
    a = _rand_alm_host(lmax, spin, 1 + spin)
    x = masked.alm_to_real(torch.as_tensor(a), lmax, spin)
    assert x.shape == (jhtb.n_dof(lmax, spin),)
    back = masked.real_to_alm(x, lmax, spin).numpy()
    assert np.max(np.abs(back - a)) <= 1e-14
    w = jhtb.alm_metric_weight(lmax)
    wnorm2 = float(np.sum(w * np.abs(np.atleast_2d(a)) ** 2))
    assert abs(float(torch.sum(x * x)) - wnorm2) <= 1e-13 * wnorm2


def test_bandpower_on_host_tensors_matches_oracle():
    """bandpower is plain tensor arithmetic: on host tensors it equals the oracle's C_l."""
    lmax = 12
    a = _rand_alm_host(lmax, 0, 9)
    got = jhtb.bandpower(torch.as_tensor(a), lmax).numpy()
    ref = O.bandpower(a, lmax)
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))


def _fft_kernel_model(x, sign):
    """The index arithmetic of fft_smooth_kernel (fft.cu) in NumPy: radix counts (4, 2, 3, 5
    in that order), the mixed-radix digit-reversed load, in-place DIT stages whose butterfly
    (g, j) twiddles element q by roots[j n / L]^q (sign applied to the table's e^{-2 pi i k/n})
    before an R-point DFT.  Used to sweep every smooth length; the kernel runs on the GPU."""
    from jht_b200 import _fft

    n = x.size
    counts, r = [], n
    for R in (4, 2, 3, 5):
        c = 0
        while r % R == 0:
            c, r = c + 1, r // R
        counts.append(c)
    assert r == 1
    radices = [R for R, c in zip((4, 2, 3, 5), counts) for _ in range(c)]
    i = np.arange(n)
    pos, span, rem = np.zeros(n, dtype=np.int64), n, i.copy()
    for R in reversed(radices):  # the last stage's radix is the least significant digit
        span //= R
        pos += (rem % R) * span
        rem //= R
    buf = np.empty(n, dtype=np.complex128)
    buf[pos] = x
    roots = _fft._roots_host(n)
    m = 1
    for R in radices:
        L = m * R
        bi = np.arange(n // R)
        gq, j = bi // m, bi % m
        base = gq * L + j
        v = np.stack([buf[base + q * m] for q in range(R)])
        w = roots[j * (n // L)]
        if sign > 0:
            w = np.conj(w)
        v = v * w[None, :] ** np.arange(R)[:, None]
        dft = np.exp(sign * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
        v = dft @ v
        for q in range(R):
            buf[base + q * m] = v[q]
        m = L
    return buf


def test_fft_kernel_index_model_for_every_smooth_length():
    """Every 2,3,5-smooth length up to the shared-memory limit, both signs: the kernel's
    digit-reversed load and stage indexing compose to the DFT (NumPy's fft)."""
    from jht_b200 import _fft

    rng = np.random.default_rng(11)
    lengths = [n for n in range(1, _fft.SM_MAX + 1) if _fft._smooth(n)]
    assert len(lengths) == 177
    for n in lengths:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        for sign in (-1, 1):
            got = _fft_kernel_model(x, sign)
            ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
            assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref))), (n, sign)


@pytest.mark.parametrize("N,Q", [(8192, 2), (16384, 4), (4 * 3000, 4), (4 * 1537, 4)])
@pytest.mark.parametrize("shifted", [False, True])
def test_ring_piece_decomposition(N, Q, shifted):
    """The decimation in frequency of the piece kernels (ringfft.cu): piece s of a ring of
    N = Q Lq points computes the outputs Q j + s from a_s[k1] = sum_k2 D[k1 + Lq k2]
    e^{i pi c (k1 + Lq k2) / N}, c = shifted + 2 s (the ring phase e^{i pi k / N} when
    phi0 = pi / N, and the piece twiddle), followed by a length-Lq transform; the adjoint
    gathers b_s[j1] = sum_j2 v[j1 + Lq j2] e^{-2 pi i s (j1 + Lq j2) / N}.  For Q = 2 the
    k2 = 1 factor is e^{i pi c / 2}, exactly +-1 or +-i."""
    rng = np.random.default_rng(N + Q)
    Lq = N // Q
    D = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    ph = np.exp(1j * np.pi * np.arange(N) / N) if shifted else np.ones(N)
    ref = np.fft.ifft(D * ph) * N
    v = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    W = np.fft.fft(v)
    k1, k2 = np.arange(Lq)[:, None], np.arange(Q)[None, :]
    idx = k1 + Lq * k2
    for s in range(Q):
        c = (1 if shifted else 0) + 2 * s
        a = np.sum(D[idx] * np.exp(1j * np.pi * c * (idx % (2 * N)) / N), axis=1)
        out = np.fft.ifft(a) * Lq
        assert np.max(np.abs(out - ref[s::Q])) <= 1e-10 * np.max(np.abs(ref))
        if Q == 2:
            assert np.isclose(np.exp(1j * np.pi * c * Lq / N), 1j ** (c % 4), atol=1e-15)
        b = np.sum(v[idx] * np.exp(-2j * np.pi * s * idx / N), axis=1)
        assert np.max(np.abs(np.fft.fft(b) - W[s::Q])) <= 1e-10 * np.max(np.abs(W))
