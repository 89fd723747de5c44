"""Per-configuration tuning of the plan knobs, timed on the device.

The CUDA library exposes a few knobs that change speed but not the transform
(``jhtb_plan_set_tuning``, ``include/jhtb.h``): the FP32 accumulation block of the
tensor-core synthesis (``tc_fold``, degrees) and adjoint (``tca_fold``, rings), the maps
per tensor-core synthesis group (``tc_group``) and the CTAs per SM of the FP64 Legendre
kernels (``leg_ctas``).  For one configuration (nside, lmax, spin, batch, precision)
:func:`tune` times the pair S and S^T for every candidate setting, replayed from a
captured CUDA graph (CUDA events around the replays), keeps only candidates whose
result stays within ``tol`` of the FP64 transforms (mixed precision; FP64 candidates are
bit-identical by construction; the gate is half the tested 1e-6 bound, to keep a margin
for inputs the tuner has not seen), and returns the fastest.  The winners live in
``tuning.json`` next to this module, keyed ``"nside,lmax,spin,batch,precision"``;
:func:`jht_b200._lib.get_plan` applies the entry for its configuration (the largest
tuned batch not above the requested one) to every plan it creates.

jht's counterpart is its best-of-N stage timing (scripts/bench_transforms.py:47-57); it
has no knobs to choose.

    python -m jht_b200.autotune --config 2048,4096,2,16,bf16x3 --out tuning.json
"""

from __future__ import annotations

import argparse
import itertools
import json
import threading
from pathlib import Path

import numpy as np

TABLE = Path(__file__).resolve().parent / "tuning.json"
KNOBS = ("tc_fold", "tca_fold", "tc_group", "leg_ctas")
MIXED_TOL = 1e-6
# a candidate must stay within half the tested bound on the tuning inputs, so that the
# choice keeps a margin for inputs it was not tuned on
GATE = 0.5 * MIXED_TOL

_table_cache: dict | None = None
_table_lock = threading.Lock()


def key(nside: int, lmax: int, spin: int, batch: int, precision: str) -> str:
    return f"{int(nside)},{int(lmax)},{int(spin)},{int(batch)},{precision}"


def load_table(path: str | Path | None = None) -> dict:
    """The tuning table ({key: {"knobs": {...}, "ms": ...}}); empty if there is none."""
    global _table_cache
    with _table_lock:
        if path is None and _table_cache is not None:
            return _table_cache
        p = Path(path) if path is not None else TABLE
        try:
            table = json.loads(p.read_text())
        except (OSError, ValueError):
            table = {}
        for k, v in table.items():
            bad = set(v.get("knobs", {})) - set(KNOBS)
            if bad:
                raise ValueError(f"tuning table entry {k!r} has unknown knobs {sorted(bad)}")
        if path is None:
            _table_cache = table
        return table


def lookup(nside: int, lmax: int, spin: int, batch: int, precision: str, table: dict | None = None) -> dict:
    """Knobs for a configuration: the exact entry, else the one with the largest tuned batch
    not above ``batch`` for the same (nside, lmax, spin, precision); {} when none applies."""
    table = load_table() if table is None else table
    best, best_b = None, -1
    for k, v in table.items():
        n, l, s, b, prec = k.split(",")
        if (int(n), int(l), int(s), prec) != (nside, lmax, spin, precision):
            continue
        b = int(b)
        if b <= batch and b > best_b:
            best, best_b = v, b
    return dict(best["knobs"]) if best else {}


def candidates(precision: str, spin: int) -> list[dict]:
    """Knob settings tried for a precision (every one is a valid, accuracy-tested setting)."""
    if precision == "fp64":
        return [{"leg_ctas": c} for c in (0, 1, 2, 3)]
    out = []
    for tf, af, grp in itertools.product((256, 512), (256, 512), (16, 8)):
        out.append({"tc_fold": tf, "tca_fold": af, "tc_group": grp})
    return out


def _inputs(nside: int, lmax: int, spin: int, batch: int, seed: int = 7):
    import torch

    rng = np.random.default_rng(seed)
    K = (lmax + 1) * (lmax + 2) // 2
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    nc = 1 if spin == 0 else 2
    a = (rng.standard_normal((batch, nc, K)) + 1j * rng.standard_normal((batch, nc, K))) / (ell + 10.0)
    a[..., : lmax + 1] = a[..., : lmax + 1].real
    if spin == 2:
        a[..., ell < 2] = 0
    v = rng.standard_normal((batch, nc, 12 * nside * nside))
    return torch.as_tensor(a, device="cuda"), torch.as_tensor(v, device="cuda")


def _pair(plan, a, v, m_out, b_out):
    from . import _lib

    B = a.shape[0]
    s = _lib.stream_ptr()
    _lib.check(plan.lib.jhtb_synthesis(plan.handle, a.data_ptr(), m_out.data_ptr(), B, s), "jhtb_synthesis")
    _lib.check(plan.lib.jhtb_adjoint_synthesis(plan.handle, v.data_ptr(), b_out.data_ptr(), B, s),
               "jhtb_adjoint_synthesis")


def _time(plan, a, v, m_out, b_out, reps: int) -> tuple[float, bool]:
    """Device ms per S + S^T pair: replays of a captured CUDA graph when capture works."""
    import torch

    _pair(plan, a, v, m_out, b_out)  # eager warm-up (also finishes lazy set-up outside capture)
    torch.cuda.synchronize()
    graph = None
    try:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            _pair(plan, a, v, m_out, b_out)
        graph = g
    except Exception:  # noqa: BLE001 - capture is an optimisation of the timing only
        torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    run = graph.replay if graph is not None else (lambda: _pair(plan, a, v, m_out, b_out))
    run()
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    graphed = graph is not None
    del graph
    return ms, graphed


def tune(nside: int, lmax: int, spin: int, batch: int, precision: str, reps: int = 3,
         tol: float = GATE, verbose: bool = False) -> dict:
    """Time every candidate setting and return {"knobs", "ms", "default_ms", "err", "trials"}."""
    import torch

    from . import _lib

    a, v = _inputs(nside, lmax, spin, batch)
    nc = 1 if spin == 0 else 2
    K = (lmax + 1) * (lmax + 2) // 2
    npix = 12 * nside * nside
    m_out = torch.empty((batch, nc, npix), dtype=torch.float64, device="cuda")
    b_out = torch.empty((batch, nc, K), dtype=torch.complex128, device="cuda")
    ref_m = ref_b = None
    if precision != "fp64":
        ref = _lib.Plan(nside, lmax, spin, "fp64", max_batch=batch)
        _pair(ref, a, v, m_out, b_out)
        ref_m, ref_b = m_out.clone(), b_out.clone()
        ref.close()
    plan = _lib.Plan(nside, lmax, spin, precision, max_batch=batch)
    trials = []
    try:
        for knobs in candidates(precision, spin):
            plan.set_tuning(**knobs)
            ms, graphed = _time(plan, a, v, m_out, b_out, reps)
            err = 0.0
            if ref_m is not None:
                em = torch.amax(torch.abs(m_out - ref_m).reshape(batch, -1), 1) / torch.amax(torch.abs(ref_m).reshape(batch, -1), 1)
                eb = torch.amax(torch.abs(b_out - ref_b).reshape(batch, -1), 1) / torch.amax(torch.abs(ref_b).reshape(batch, -1), 1)
                err = float(torch.maximum(em, eb).max())
            if plan.status() != 0:
                err = float("inf")
            trials.append({"knobs": dict(knobs), "ms": ms, "err": err, "graph": graphed})
            if verbose:
                print(f"  {knobs}: {ms:.3f} ms, err {err:.2e}, graph {graphed}", flush=True)
    finally:
        plan.close()
    ok = [t for t in trials if t["err"] <= tol]
    if not ok:
        raise RuntimeError(f"no candidate met the error bound {tol} for {key(nside, lmax, spin, batch, precision)}")
    best = min(ok, key=lambda t: t["ms"])
    return {"knobs": best["knobs"], "ms": best["ms"], "default_ms": trials[0]["ms"], "err": best["err"],
            "trials": trials}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--config", action="append", required=True, help="nside,lmax,spin,batch,precision")
    ap.add_argument("--out", default=str(TABLE))
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)
    out = Path(args.out)
    table = load_table(out) if out.exists() else {}
    for c in args.config:
        n, l, s, b, prec = c.split(",")
        print(f"tuning {c}", flush=True)
        res = tune(int(n), int(l), int(s), int(b), prec, reps=args.reps, verbose=True)
        table[key(int(n), int(l), int(s), int(b), prec)] = {
            "knobs": res["knobs"], "ms": round(res["ms"], 4), "default_ms": round(res["default_ms"], 4),
            "err": res["err"]}
        out.write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")
        print(f"  -> {res['knobs']} {res['ms']:.3f} ms (default {res['default_ms']:.3f} ms)", flush=True)


if __name__ == "__main__":
    main()
