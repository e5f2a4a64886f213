"""Time-series analysis of force histories (src/signal.rs), on the host through the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _arr(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def fft(re, im):
    """In-place radix-2 FFT (src/signal.rs:6-43); returns new arrays."""
    re, im = _arr(re).copy(), _arr(im).copy()
    check(lib.vl_fft(_dp(re), _dp(im), len(re)))
    return re, im


def mean(x) -> float:
    x = _arr(x)
    return lib.vl_mean(_dp(x), len(x))


def rms(x) -> float:
    x = _arr(x)
    return lib.vl_rms(_dp(x), len(x))


def dominant_frequency(x, dt):
    """(frequency, amplitude) of the strongest line (src/signal.rs:92-107)."""
    x = _arr(x)
    f, a = C.c_double(), C.c_double()
    check(lib.vl_dominant_frequency(_dp(x), len(x), dt, C.byref(f), C.byref(a)))
    return f.value, a.value


def peaks(x):
    """Parabola-refined local maxima above the mean (src/signal.rs:111-123)."""
    x = _arr(x)
    cap = max(len(x), 1)
    pos, val = np.zeros(cap), np.zeros(cap)
    k = lib.vl_peaks(_dp(x), len(x), _dp(pos), _dp(val), cap)
    return list(zip(pos[:k].tolist(), val[:k].tolist()))


def crossing_frequency(x, dt):
    """Frequency from upward mean crossings, or None (src/signal.rs:127-140)."""
    x = _arr(x)
    out = C.c_double()
    return out.value if check(lib.vl_crossing_frequency(_dp(x), len(x), dt, C.byref(out))) else None


def sample_at(x, pos) -> float:
    x = _arr(x)
    return lib.vl_sample_at(_dp(x), len(x), pos)
