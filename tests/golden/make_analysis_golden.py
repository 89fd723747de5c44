"""Golden vectors for spin-0 analysis at nside 1024, lmax 2048 (niter 3), from jht itself.

Workload: seeded a_lm with C_l = 1/(l+10)^2 (a_l0 = sqrt(C_l) g, a_lm = sqrt(C_l/2)(g1 + i g2),
rng seed 11), synthesised by the FP64 C oracle (``oracle/legendre_ref.c`` + NumPy ring FFTs,
deterministic); the ``noise`` variant adds white noise of sigma 1e-3 per pixel (rng seed 12).
The reference's own ``analysis(maps, nside, lmax, spin=0, niter=3, use_weights=True)``
(src/jht/_analysis.py:55-63) then runs on that map through the NumPy stand-in for JAX
(``jaxshim``), and a fixed sample of the output a_lm is stored: 12288 seeded random
entries, the whole m = 0 column, the l = m diagonal and the l = lmax row.

The GPU test rebuilds the same input map with the same oracle calls and compares its own
analysis at those entries.  One variant takes about 45 minutes on one core::

    python tests/golden/make_analysis_golden.py /path/to/jht/checkout clean
    python tests/golden/make_analysis_golden.py /path/to/jht/checkout noise
"""

from __future__ import annotations

import sys
import warnings
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))

NSIDE, LMAX, NITER, SIGMA = 1024, 2048, 3, 1e-3


def alm_size(lmax: int) -> int:
    return (lmax + 1) * (lmax + 2) // 2


def input_alm() -> np.ndarray:
    ell = np.concatenate([np.arange(m, LMAX + 1) for m in range(LMAX + 1)])
    cl = 1.0 / (ell + 10.0) ** 2
    rng = np.random.default_rng(11)
    K = alm_size(LMAX)
    g1 = rng.standard_normal(K)
    g2 = rng.standard_normal(K)
    a = np.sqrt(cl / 2.0) * (g1 + 1j * g2)
    a[: LMAX + 1] = np.sqrt(cl[: LMAX + 1]) * g1[: LMAX + 1]
    return a.astype(np.complex128)


def input_map(variant: str) -> np.ndarray:
    """FP64 oracle synthesis of input_alm() (+ the seeded noise for ``noise``)."""
    from oracle import jht_oracle as O

    m = O.synthesis(input_alm(), NSIDE, LMAX, 0, use_c=True)
    if variant == "noise":
        m = m + SIGMA * np.random.default_rng(12).standard_normal(m.size)
    return m


def sample_index() -> np.ndarray:
    K = alm_size(LMAX)
    rng = np.random.default_rng(13)
    ms = np.arange(LMAX + 1)
    base = ms * (2 * LMAX + 1 - ms) // 2
    idx = np.concatenate([rng.choice(K, 12288, replace=False), np.arange(LMAX + 1), base + ms, base + LMAX])
    return np.unique(idx).astype(np.int64)


def main(ref_root: str, variant: str) -> None:
    import jaxshim

    if variant not in ("clean", "noise"):
        raise SystemExit("variant must be 'clean' or 'noise'")
    jht = jaxshim.import_reference(str(Path(ref_root) / "src"))
    warnings.simplefilter("ignore")
    maps = input_map(variant)
    out = np.asarray(jht._analysis.analysis(maps, NSIDE, LMAX, spin=0, niter=NITER, use_weights=True))
    idx = sample_index()
    np.savez_compressed(HERE / f"jht_golden_analysis_{variant}.npz", idx=idx, alm=out[idx],
                        meta=np.array([NSIDE, LMAX, NITER]), sigma=np.array(SIGMA if variant == "noise" else 0.0))


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    main(sys.argv[1], sys.argv[2])
