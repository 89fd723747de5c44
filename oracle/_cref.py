"""ctypes loader for the C part of the oracle (``legendre_ref.c``).

TEST INFRASTRUCTURE ONLY.  The shared library is built by ``oracle/Makefile``
into ``oracle/_ref_build/liblegendre_ref.so`` (``__graft_entry__.build()`` runs
the same recipe); if it is missing and ``make`` + ``gcc`` are available it is
built on first use.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref_build" / "liblegendre_ref.so"


def build() -> Path:
    subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


class _Ref:
    def __init__(self, lib):
        self.lib = lib
        argt = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        for name in ("oracle_synth", "oracle_adjoint", "oracle_synth_ld", "oracle_adjoint_ld"):
            getattr(lib, name).argtypes = argt
            getattr(lib, name).restype = None

    def synth(self, spin, lmax, x, alm, m_lo=0, m_hi=None, extended=False):
        """Half-grid synthesis contraction; alm is (ncomp, K). Returns 2 (spin 0) or 4 (M, T) arrays.

        ``extended=True`` runs the same algorithm in 80-bit long double (the arbiter)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        T = x.size
        M = lmax + 1
        m_hi = M if m_hi is None else m_hi
        alm = np.ascontiguousarray(alm, dtype=np.complex128)
        nout = 2 if spin == 0 else 4
        out = np.zeros((nout, M, T), np.complex128)
        f = self.lib.oracle_synth_ld if extended else self.lib.oracle_synth
        f(spin, lmax, T, x.ctypes.data, alm.ctypes.data, out.ctypes.data, m_lo, m_hi)
        return tuple(out)

    def adjoint(self, spin, lmax, x, V, m_lo=0, m_hi=None, extended=False):
        """Half-grid adjoint contraction; V is a list of (M, T). Returns packed (K,) arrays.

        ``extended=True`` runs the same algorithm in 80-bit long double (the arbiter)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        T = x.size
        M = lmax + 1
        K = M * (M + 1) // 2
        m_hi = M if m_hi is None else m_hi
        Vin = np.ascontiguousarray(np.stack(V), dtype=np.complex128)
        nout = 1 if spin == 0 else 2
        out = np.zeros((nout, K), np.complex128)
        f = self.lib.oracle_adjoint_ld if extended else self.lib.oracle_adjoint
        f(spin, lmax, T, x.ctypes.data, Vin.ctypes.data, out.ctypes.data, m_lo, m_hi)
        return tuple(out)


_INSTANCE = None


def load() -> _Ref:
    global _INSTANCE
    if _INSTANCE is None:
        if not LIB.exists():
            build()
        _INSTANCE = _Ref(ctypes.CDLL(str(LIB), mode=os.RTLD_LOCAL))
    return _INSTANCE
