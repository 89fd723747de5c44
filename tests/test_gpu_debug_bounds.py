"""The bounds-checked debug library (jht_b200/_lib_debug/libjhtb.so, ``make debug``).

Every checked gather and scatter index of its kernels is tested against the extent of
its buffer; an access out of range is skipped and counted (jhtb_debug_bounds).  A child
process loads the debug library (JHTB_LIBRARY), runs the transforms over geometries that
reach every code path of the azimuthal stage (whole rings, power-of-two pieces of the
belt, chirp-z pieces of the polar caps, chirp-z rings split through the scratch rows at
nside 4096, aliasing short rings) and of the Legendre kernels
(FP64 and tensor-core, spin 0 and 2, full and partial map groups), and must record no
failed access; its outputs must equal the release library's on the same inputs.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU hosts
    pytest.skip("no CUDA device", allow_module_level=True)

import jht_b200 as jhtb  # noqa: E402
from jht_b200 import _lib  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]

# (nside, lmax, spin, batch, precision)
CASES = [
    (1, 4, 0, 1, "fp64"), (2, 5, 2, 1, "fp64"), (12, 20, 2, 1, "fp64"), (16, 40, 0, 1, "fp64"),
    (64, 128, 0, 1, "fp64"), (512, 1024, 2, 1, "fp64"), (1024, 2048, 0, 1, "fp64"),
    (2048, 4096, 2, 1, "fp64"), (4096, 96, 2, 1, "fp64"), (4096, 96, 0, 1, "fp64"), (64, 128, 2, 3, "bf16x3"),
    (256, 512, 0, 17, "bf16x3"),
]

CHILD = textwrap.dedent("""
    import json, sys
    import numpy as np, torch
    sys.path.insert(0, {root!r})
    import jht_b200 as jhtb
    from jht_b200 import _lib
    out = {{}}
    for nside, lmax, spin, nb, prec in {cases!r}:
        a = torch.as_tensor(np.load({tmp!r} + f"/a_{{nside}}_{{lmax}}_{{spin}}_{{nb}}.npy"), device="cuda")
        m = jhtb.synthesis_batch(a, nside, lmax, spin, precision=prec)
        b = jhtb.adjoint_synthesis_batch(m, nside, lmax, spin, precision=prec)
        np.save({tmp!r} + f"/m_{{nside}}_{{lmax}}_{{spin}}_{{nb}}.npy", m.cpu().numpy())
        np.save({tmp!r} + f"/b_{{nside}}_{{lmax}}_{{spin}}_{{nb}}.npy", b.cpu().numpy())
        out[f"{{nside}}_{{lmax}}_{{spin}}_{{nb}}"] = _lib.debug_bounds()
    print("RECORD " + json.dumps(out))
""")


def _alm(rng, nb, lmax, spin):
    K = jhtb.alm_size(lmax)
    shape = (nb, 2, K) if spin else (nb, K)
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / 100
    a[..., : lmax + 1] = a[..., : lmax + 1].real
    if spin:
        ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
        a[..., ell < 2] = 0
    return a


@pytest.fixture(scope="module")
def debug_lib():
    if not _lib.DEBUG_LIB_PATH.exists():
        pytest.fail(f"debug library missing at {_lib.DEBUG_LIB_PATH}: build it with `python -m jht_b200.build --debug`")
    return _lib.DEBUG_LIB_PATH


def test_release_library_has_no_checks():
    with pytest.raises(NotImplementedError, match="debug library"):
        _lib.debug_bounds()


def test_debug_library_records_no_failed_access_and_matches_release(debug_lib, tmp_path):
    rng = np.random.default_rng(77)
    inputs = {}
    for nside, lmax, spin, nb, _ in CASES:
        a = _alm(rng, nb, lmax, spin)
        inputs[(nside, lmax, spin, nb)] = a
        np.save(tmp_path / f"a_{nside}_{lmax}_{spin}_{nb}.npy", a)
    code = CHILD.format(root=str(ROOT), cases=CASES, tmp=str(tmp_path))
    env = dict(os.environ, JHTB_LIBRARY=str(debug_lib))
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stderr[-3000:]
    line = [ln for ln in res.stdout.splitlines() if ln.startswith("RECORD ")][-1]
    record = json.loads(line[len("RECORD "):])
    for key, rec in record.items():
        assert rec["count"] == 0, (key, rec)
    for nside, lmax, spin, nb, prec in CASES:
        a = torch.as_tensor(inputs[(nside, lmax, spin, nb)], device="cuda")
        m = jhtb.synthesis_batch(a, nside, lmax, spin, precision=prec)
        b = jhtb.adjoint_synthesis_batch(m, nside, lmax, spin, precision=prec)
        md = np.load(tmp_path / f"m_{nside}_{lmax}_{spin}_{nb}.npy")
        bd = np.load(tmp_path / f"b_{nside}_{lmax}_{spin}_{nb}.npy")
        em = float(np.max(np.abs(m.cpu().numpy() - md)) / np.max(np.abs(md)))
        eb = float(np.max(np.abs(b.cpu().numpy() - bd)) / np.max(np.abs(bd)))
        assert em <= 1e-14 and eb <= 1e-14, (nside, lmax, spin, nb, prec, em, eb)
