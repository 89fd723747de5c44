"""``enable_compilation_cache`` kept for API compatibility with jht (src/jht/_cache.py:25-40).

jht opts in to XLA's persistent compile cache.  The kernels here are compiled
ahead of time into libjhtb.so, so there is nothing to cache; the call records the
directory and returns.
"""

from __future__ import annotations

__all__ = ["enable_compilation_cache"]

_settings: dict[str, object] = {}


def enable_compilation_cache(directory: str, *, min_compile_time_secs: float = 1.0) -> None:
    _settings["directory"] = directory
    _settings["min_compile_time_secs"] = float(min_compile_time_secs)
