"""Azimuth-FFT mode switch, kept for API compatibility with jht (src/jht/_azimuth.py:56-89).

In jht the mode trades XLA compile size against run time.  Here every ring
length is handled by the same compiled ring-FFT kernel (power-of-two or
Bluestein per ring), so both modes run the same code and give the same result;
the setting is validated and remembered but changes nothing.
"""

from __future__ import annotations

__all__ = ["set_azimuth_fft_mode", "get_azimuth_fft_mode", "enable_looped_fft"]

_LEGAL = ("unrolled", "looped")
_MODE = "unrolled"


def set_azimuth_fft_mode(mode: str) -> None:
    if mode not in _LEGAL:
        raise ValueError(f"unknown azimuth FFT mode {mode!r}; expected one of {_LEGAL}")
    global _MODE
    _MODE = mode


def get_azimuth_fft_mode() -> str:
    return _MODE


def enable_looped_fft() -> None:
    set_azimuth_fft_mode("looped")
