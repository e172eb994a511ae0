"""Source wavelets (cuwave signals.py:5-71)."""

from __future__ import annotations

import numpy as np


def ricker(t, amplitude: float, frequency: float, delay: float | None = None) -> np.ndarray:
    """Ricker wavelet A (1 - 2 pi^2 f^2 (t - d)^2) exp(-pi^2 f^2 (t - d)^2), d = 1/f by default."""
    if delay is None:
        delay = 1.0 / frequency
    arg = (np.pi * frequency * (np.asarray(t) - delay)) ** 2
    return amplitude * (1.0 - 2.0 * arg) * np.exp(-arg)


def sineburst(t, amplitude: float, frequency: float, cycles: int) -> np.ndarray:
    """Hann-windowed sine burst of `cycles` periods, zero outside its support."""
    t = np.asarray(t)
    mask = (t > 0) & (t <= cycles / frequency)
    return (
        amplitude * mask * np.sin(2 * np.pi * frequency * t)
        * np.sin(np.pi * frequency * t / cycles) ** 2
    )
