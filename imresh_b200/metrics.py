"""Host-side comparison of reconstructions (numpy; no device work).

Phase retrieval recovers an object only up to the ambiguities of its Fourier
modulus: a circular translation and the twin (the point reflection
x -> -x, conjugated; for the real part of a reconstruction, the reflected
image).  ``aligned_rel_l2`` compares two reconstructions after removing
both: it tries the candidate and its twin, moves each onto the reference by
the integer circular shift that maximises their cross-correlation, and
returns the smaller relative L2 distance.
"""
from __future__ import annotations

import numpy as np


def twin(a: np.ndarray) -> np.ndarray:
    """a(-x) on the periodic grid: index k -> (-k) mod n along both axes."""
    return np.roll(np.flip(a, axis=(0, 1)), 1, axis=(0, 1))


def best_shift(a: np.ndarray, b: np.ndarray):
    """Integer circular shift (dy, dx) that maximises sum(roll(a, d) * b)."""
    xc = np.fft.ifft2(np.conj(np.fft.fft2(a)) * np.fft.fft2(b)).real
    return np.unravel_index(int(np.argmax(xc)), xc.shape)


def aligned_rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||align(a) - b|| / ||b|| with align = best of {a, twin(a)} shifted onto b."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    best = np.inf
    for cand in (a, twin(a)):
        s = np.roll(cand, best_shift(cand, b), axis=(0, 1))
        best = min(best, float(np.linalg.norm(s - b) / nb))
    return best


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / ||b|| in double precision (complex128 when either is complex)."""
    a, b = np.asarray(a), np.asarray(b)
    dt = np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64
    a, b = a.astype(dt), b.astype(dt)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
