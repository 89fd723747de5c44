"""ctypes binding of the jhtb C ABI (include/jhtb.h) and the per-geometry plan cache.

The CUDA library is built in-tree (``python -m jht_b200.build``) into
``jht_b200/_lib/libjhtb.so``.  There is no CPU fallback: if the library or a
CUDA device is missing, every transform raises.
"""

from __future__ import annotations

import ctypes
import math
import os
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libjhtb.so"

JHTB_OK = 0
JHTB_ERR_INVALID = -1
JHTB_ERR_UNSUPPORTED = -2
JHTB_ERR_CUDA = -3
JHTB_ERR_NOMEM = -4

PRECISIONS = {"fp64": 0, "fp32": 1, "bf16x3": 2}
TUNE_KEYS = {"tc_fold": 1, "tca_fold": 2, "tc_group": 3, "leg_ctas": 4}
TC_MAPS = 16  # maps per tensor-core GEMM group (kTcMaps in the CUDA sources)

# every exported symbol of include/jhtb.h (checked by the CPU test suite)
EXPORTS = (
    "jhtb_version",
    "jhtb_last_error",
    "jhtb_plan_create",
    "jhtb_plan_destroy",
    "jhtb_plan_bytes",
    "jhtb_synthesis",
    "jhtb_adjoint_synthesis",
    "jhtb_weighted_residual",
    "jhtb_axpy",
    "jhtb_dot",
    "jhtb_plan_set_timing",
    "jhtb_plan_timings",
    "jhtb_probe_fp64_fma",
    "jhtb_synthesis_noalloc",
    "jhtb_plan_status",
    "jhtb_plan_set_watchdog",
    "jhtb_plan_inject_fault",
    "jhtb_plan_set_tuning",
    "jhtb_plan_ring_costs",
    "jhtb_plan_set_ring_range",
    "jhtb_plan_create_rings",
    "jhtb_legendre_synthesis",
    "jhtb_legendre_adjoint",
    "jhtb_nufft_interp",
    "jhtb_nufft_spread",
    "jhtb_nufft_spread_tiles",
    "jhtb_debug_bounds",
    "jhtb_fft_c2c",
)


class HostTables(ctypes.Structure):
    _fields_ = [
        ("x", ctypes.c_void_p),
        ("logsin", ctypes.c_void_p),
        ("logcos_half", ctypes.c_void_p),
        ("logsin_half", ctypes.c_void_p),
        ("seed_logc", ctypes.c_void_p),
    ]


class JhtbError(RuntimeError):
    """A jhtb C-ABI call returned a non-zero status."""


_lib = None
_lib_lock = threading.Lock()


def load_library(path: str | os.PathLike | None = None):
    """Load libjhtb.so (once) and declare the C signatures."""
    global _lib
    with _lib_lock:
        if _lib is not None and path is None:
            return _lib
        env = os.environ.get("JHTB_LIBRARY")
        p = Path(path) if path else (Path(env) if env else LIB_PATH)
        if not p.exists():
            raise ImportError(
                f"jht_b200 CUDA library not found at {p}; build it with `python -m jht_b200.build` "
                "(there is no CPU fallback)"
            )
        lib = ctypes.CDLL(str(p), mode=os.RTLD_LOCAL)
        vp, i32, i64, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p
        sig = {
            "jhtb_version": (i32, []),
            "jhtb_last_error": (i32, [ctypes.c_char_p, ctypes.c_size_t]),
            "jhtb_plan_create": (i32, [i32, i32, i32, i32, i32, ctypes.POINTER(HostTables), ctypes.POINTER(vp)]),
            "jhtb_plan_destroy": (i32, [vp]),
            "jhtb_plan_bytes": (i32, [vp, ctypes.POINTER(i64)]),
            "jhtb_synthesis": (i32, [vp, vp, vp, i32, vp]),
            "jhtb_adjoint_synthesis": (i32, [vp, vp, vp, i32, vp]),
            "jhtb_weighted_residual": (i32, [vp, dp, dp, dp, dp, i32, vp]),
            "jhtb_axpy": (i32, [i64, ctypes.c_double, dp, dp, vp]),
            "jhtb_dot": (i32, [vp, i64, dp, dp, dp, vp]),
            "jhtb_plan_set_timing": (i32, [vp, i32]),
            "jhtb_plan_timings": (i32, [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(i64), i32]),
            "jhtb_probe_fp64_fma": (i32, [i32, i32, dp, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double), vp]),
            "jhtb_synthesis_noalloc": (i32, [i32, i32, vp, vp, vp]),
            "jhtb_plan_status": (i32, [vp, ctypes.POINTER(i32)]),
            "jhtb_plan_set_watchdog": (i32, [vp, i64]),
            "jhtb_plan_inject_fault": (i32, [vp, i32]),
            "jhtb_plan_set_tuning": (i32, [vp, i32, i32]),
            "jhtb_plan_ring_costs": (i32, [vp, i32, ctypes.POINTER(i64), i32]),
            "jhtb_plan_set_ring_range": (i32, [vp, i32, i32]),
            "jhtb_plan_create_rings": (i32, [i32, i32, i32, i32, i32, ctypes.POINTER(HostTables),
                                             ctypes.POINTER(vp)]),
            "jhtb_legendre_synthesis": (i32, [vp, vp, vp, i32, vp]),
            "jhtb_legendre_adjoint": (i32, [vp, vp, vp, i32, vp]),
            "jhtb_nufft_interp": (i32, [vp, i32, i32, i32, ctypes.c_double, dp, dp, i64, vp, vp, vp, vp]),
            "jhtb_nufft_spread": (i32, [vp, dp, dp, i64, i32, i32, i32, ctypes.c_double, vp, vp]),
            "jhtb_nufft_spread_tiles": (i32, [vp, dp, dp, i64, i64, vp, vp, vp, i32, i32, i32, i32, ctypes.c_double,
                                              vp, vp]),
            "jhtb_debug_bounds": (i32, [ctypes.POINTER(i64), ctypes.POINTER(i32), ctypes.POINTER(i64),
                                        ctypes.POINTER(i64)]),
            "jhtb_fft_c2c": (i32, [vp, vp, i32, i64, i64, i64, i64, i64, i64, i64, i64, i32, ctypes.c_double, i64,
                                   vp, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        if path is None:
            _lib = lib
        return lib


DEBUG_LIB_PATH = LIB_PATH.parent.parent / "_lib_debug" / "libjhtb.so"


def debug_bounds(lib=None) -> dict:
    """The bounds-check record of a debug library (``make debug``): failed accesses since
    the last call, with the first one's site code, index and extent (clears the record).
    Raises NotImplementedError (status JHTB_ERR_UNSUPPORTED) on the release library."""
    lib = lib or load_library()
    cnt, site, idx, ext = ctypes.c_int64(), ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
    check(lib.jhtb_debug_bounds(ctypes.byref(cnt), ctypes.byref(site), ctypes.byref(idx), ctypes.byref(ext)),
          "jhtb_debug_bounds")
    return {"count": cnt.value, "site": site.value, "index": idx.value, "extent": ext.value}


def last_error() -> str:
    lib = load_library()
    buf = ctypes.create_string_buffer(1024)
    lib.jhtb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str) -> None:
    if status == JHTB_OK:
        return
    msg = f"{what} failed ({status}): {last_error()}"
    if status == JHTB_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if status == JHTB_ERR_INVALID:
        raise ValueError(msg)
    if status == JHTB_ERR_NOMEM:
        raise MemoryError(msg)
    raise JhtbError(msg)


# ---------------------------------------------------------------------------------------
# host seed tables, computed exactly as jht's NumPy plan computes them
# (_recursion.py:305-333): same geometry, same np.log / np.sum / math.lgamma calls.
# ---------------------------------------------------------------------------------------
def _half_grid_z(nside: int) -> np.ndarray:
    i = np.arange(1, 2 * nside + 1, dtype=np.int64)
    z = np.where(
        i < nside,
        1.0 - i**2 / (3.0 * nside**2),
        4.0 / 3.0 - 2.0 * i / (3.0 * nside),
    )
    return z.astype(np.float64)


def host_tables(nside: int, lmax: int, spin: int) -> dict[str, np.ndarray]:
    return host_tables_x(_half_grid_z(nside), lmax, spin)


def host_tables_x(x: np.ndarray, lmax: int, spin: int) -> dict[str, np.ndarray]:
    """Seed tables for the northern rings at cos theta = x (poles give log 0 = -inf)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    with np.errstate(divide="ignore"):
        logsin = np.log(np.sqrt(np.clip(1.0 - x * x, 0.0, 1.0)))
        logch = np.log(np.sqrt(np.clip((1.0 + x) / 2.0, 0.0, 1.0)))
        logsh = np.log(np.sqrt(np.clip((1.0 - x) / 2.0, 0.0, 1.0)))
    M = lmax + 1
    if spin == 0:
        seed = np.empty(M)
        for m in range(M):
            k = np.arange(1, m + 1, dtype=np.float64)
            seed[m] = float(-0.5 * np.log(4.0 * np.pi) + 0.5 * np.sum(np.log((2.0 * k + 1.0) / (2.0 * k))))
    else:
        lg = math.lgamma
        seed = np.empty((2, M))
        for h, s in enumerate((2, -2)):
            for m in range(M):
                Mm, lmin = -m, max(m, 2)
                k0 = max(0, Mm - s)
                seed[h, m] = 0.5 * (lg(lmin + Mm + 1) + lg(lmin - Mm + 1) + lg(lmin + s + 1) + lg(lmin - s + 1)) - (
                    lg(k0 + 1) + lg(lmin + Mm - k0 + 1) + lg(lmin - s - k0 + 1) + lg(k0 - Mm + s + 1)
                )
    return {"x": x, "logsin": logsin, "logcos_half": logch, "logsin_half": logsh, "seed_logc": np.ascontiguousarray(seed)}


class Plan:
    """Owns one jhtb plan handle for (nside, lmax, spin, precision) on one device."""

    def __init__(self, nside: int, lmax: int, spin: int, precision: str = "fp64", max_batch: int = 1,
                 device: int | None = None, rings: tuple[int, np.ndarray] | None = None):
        """``rings = (nrings, x_north)`` makes a ring-set plan (Legendre stage only) instead
        of a HEALPix plan; ``nside`` is then ignored."""
        import torch

        if precision not in PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}; expected one of {tuple(PRECISIONS)}")
        self.lib = load_library()
        self.nside, self.lmax, self.spin, self.precision = nside, lmax, spin, precision
        self.max_batch = max_batch
        self.device = torch.cuda.current_device() if device is None else device
        self.ncomp = 1 if spin == 0 else 2
        self.K = (lmax + 1) * (lmax + 2) // 2
        self.npix = 12 * nside * nside if rings is None else 0
        self.nrings = 4 * nside - 1 if rings is None else int(rings[0])
        if rings is None:
            tabs = host_tables(nside, lmax, spin) if spin in (0, 2) else None
        else:
            tabs = host_tables_x(rings[1], lmax, spin) if spin in (0, 2) else {"x": np.ascontiguousarray(rings[1])}
        self._keep = tabs
        ht = None
        if tabs is not None:
            ht = HostTables(*(tabs[k].ctypes.data if k in tabs else None
                              for k in ("x", "logsin", "logcos_half", "logsin_half", "seed_logc")))
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            if rings is None:
                st = self.lib.jhtb_plan_create(nside, lmax, spin, PRECISIONS[precision], max_batch,
                                               ctypes.byref(ht) if ht is not None else None, ctypes.byref(handle))
            else:
                st = self.lib.jhtb_plan_create_rings(self.nrings, lmax, spin, PRECISIONS[precision], max_batch,
                                                     ctypes.byref(ht), ctypes.byref(handle))
        check(st, "jhtb_plan_create" if rings is None else "jhtb_plan_create_rings")
        self.handle = handle
        self._keep = None

    def bytes(self) -> int:
        b = ctypes.c_int64()
        check(self.lib.jhtb_plan_bytes(self.handle, ctypes.byref(b)), "jhtb_plan_bytes")
        return int(b.value)

    def status(self) -> int:
        """Device error flag of the plan's kernels (synchronises); 0 = ok."""
        e = ctypes.c_int()
        check(self.lib.jhtb_plan_status(self.handle, ctypes.byref(e)), "jhtb_plan_status")
        return int(e.value)

    def set_watchdog(self, timeout_ns: int) -> None:
        """Time limit (ns) of the tensor-core kernels' bounded waits (default 2 s)."""
        check(self.lib.jhtb_plan_set_watchdog(self.handle, int(timeout_ns)), "jhtb_plan_set_watchdog")

    def set_tuning(self, **knobs: int) -> None:
        """Apply tuning knobs (tc_fold, tca_fold, tc_group, leg_ctas); see jhtb.h."""
        for k, v in knobs.items():
            if k not in TUNE_KEYS:
                raise ValueError(f"unknown tuning knob {k!r}; expected one of {tuple(TUNE_KEYS)}")
            check(self.lib.jhtb_plan_set_tuning(self.handle, TUNE_KEYS[k], int(v)), "jhtb_plan_set_tuning")
        self.tuning = dict(getattr(self, "tuning", {}), **knobs)

    def inject_fault(self, kind: int) -> None:
        """Test hook: 1 makes the tensor-core kernels' waits run out (see jhtb.h); 0 turns it off."""
        check(self.lib.jhtb_plan_inject_fault(self.handle, int(kind)), "jhtb_plan_inject_fault")

    def ring_costs(self, granule: int = 256) -> np.ndarray:
        """Legendre work (ring-recursion steps) of each group of `granule` half-grid rings."""
        n = (2 * self.nside + granule - 1) // granule
        out = (ctypes.c_int64 * n)()
        check(self.lib.jhtb_plan_ring_costs(self.handle, granule, out, n), "jhtb_plan_ring_costs")
        return np.array(out[:], dtype=np.int64)

    def set_ring_range(self, t0: int, t1: int) -> None:
        """Restrict the plan to half-grid rings [t0, t1) and their southern mirrors."""
        check(self.lib.jhtb_plan_set_ring_range(self.handle, int(t0), int(t1)), "jhtb_plan_set_ring_range")

    def set_timing(self, enable: bool) -> None:
        check(self.lib.jhtb_plan_set_timing(self.handle, int(enable)), "jhtb_plan_set_timing")

    def timings(self, reset: bool = True) -> dict[str, tuple[float, int]]:
        """Per-stage (total ms, launches) since the last reset."""
        ms = (ctypes.c_double * 4)()
        cnt = (ctypes.c_int64 * 4)()
        check(self.lib.jhtb_plan_timings(self.handle, ms, cnt, int(reset)), "jhtb_plan_timings")
        names = ("legendre_synth", "ring_synth", "ring_adjoint", "legendre_adjoint")
        return {n: (float(ms[i]), int(cnt[i])) for i, n in enumerate(names)}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.jhtb_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_plans: dict[tuple, Plan] = {}
_plans_lock = threading.Lock()


def workspace_bytes_per_map(nside: int, lmax: int, spin: int) -> int:
    ncomp = 1 if spin == 0 else 2
    K = (lmax + 1) * (lmax + 2) // 2
    return 16 * (ncomp * (4 * nside - 1) * (lmax + 1) + 2 * 12 * nside * nside + 4 * ncomp * K)


def get_plan(nside: int, lmax: int, spin: int, precision: str = "fp64", batch: int = 1) -> Plan:
    """Cached plan; the workspace holds up to min(batch, budget) maps per pass."""
    import torch

    dev = torch.cuda.current_device()
    per = workspace_bytes_per_map(nside, lmax, spin)
    if precision == "bf16x3":
        # the tensor-core path shares one recursion among the maps of a pass: hold whole
        # groups of TC_MAPS maps when device memory allows
        cached = _plans.get((dev, nside, lmax, spin, precision))
        if cached is None or cached.max_batch < min(batch, 64):
            torch.cuda.empty_cache()  # a new plan: return torch's idle cached blocks first
        free, _ = torch.cuda.mem_get_info(dev)
        budget = min(64 << 30, max(free // 2, free - (24 << 30)))
        cap = max(1, min(64, budget // per))
        for g in (TC_MAPS, 8):
            if cap >= g:
                cap -= cap % g
                break
    else:
        cap = max(1, min(64, (4 << 30) // per))
    want = max(1, min(batch, cap))
    key = (dev, nside, lmax, spin, precision)
    with _plans_lock:
        plan = _plans.get(key)
        if plan is None or plan.max_batch < want:
            if plan is not None:
                plan.close()
            plan = Plan(nside, lmax, spin, precision, max_batch=want, device=dev)
            from .autotune import lookup  # the tuned knobs of this configuration, if any

            knobs = lookup(nside, lmax, spin, batch, precision)
            if knobs:
                plan.set_tuning(**knobs)
            _plans[key] = plan
        return plan


def clear_plans() -> None:
    with _plans_lock:
        for p in _plans.values():
            p.close()
        _plans.clear()


def stream_ptr():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
