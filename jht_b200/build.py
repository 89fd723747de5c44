"""Build libjhtb.so (sm_100a) in-tree: ``python -m jht_b200.build``.

Cross-compiles with nvcc; no GPU needed.  The library lands in
``jht_b200/_lib/libjhtb.so`` next to the package so it travels with the tree.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent / "csrc"


def build(jobs: int = 4, verbose: bool = False, debug: bool = False) -> Path:
    """Build the release library; with ``debug`` the bounds-checked one instead
    (``jht_b200/_lib_debug/libjhtb.so``, every checked index reported by jhtb_debug_bounds)."""
    cmd = ["make", "-C", str(CSRC), f"-j{jobs}"]
    if debug:
        cmd.append("debug")
    if not verbose:
        cmd.append("-s")
    subprocess.run(cmd, check=True, env=dict(os.environ))
    lib = CSRC.parent / ("_lib_debug" if debug else "_lib") / "libjhtb.so"
    if not lib.exists():
        raise RuntimeError(f"build finished but {lib} is missing")
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, debug="--debug" in sys.argv))
