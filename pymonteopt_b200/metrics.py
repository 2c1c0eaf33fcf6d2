"""Host post-processing of exit photons with the reference's semantics.

These operate on the ``get_result()`` dict (encoded exit positions, directions
and weights), exactly as ``pymopt.metrics`` does
(pymopt/metrics/_scoring.py:16-51), but with ``np.histogram``-free binning by
index instead of one ``np.where`` pass per bin.  The on-device R(r)/T(r)
tallies of :mod:`pymonteopt_b200.voxel` give the same profiles without
exporting photons.
"""
from __future__ import annotations

import numpy as np


def _bin_index(r: np.ndarray, nn: int, dr: float) -> np.ndarray:
    """Index i with i*dr < r <= (i+1)*dr, or -1 (pymopt/metrics/_scoring.py:22)."""
    alpha = np.array([i * dr for i in range(nn + 1)])
    idx = np.searchsorted(alpha, r, side="left") - 1
    idx[(r <= 0) | (idx < 0) | (idx >= nn)] = -1
    return idx


def _weighted_bins(x: np.ndarray, w: np.ndarray, nn: int, dr: float) -> np.ndarray:
    idx = _bin_index(np.asarray(x, np.float64), nn, dr)
    keep = idx >= 0
    return np.bincount(idx[keep], weights=np.asarray(w, np.float64)[keep], minlength=nn)[:nn]


def radialDistance(p, w, nn, dr, nPh):
    """R(r): weight per annulus (i*dr, (i+1)*dr] / (2*pi*(i+1/2)*dr^2 * nPh)
    (pymopt/metrics/_scoring.py:16-25)."""
    alpha = np.array([i * dr for i in range(nn + 1)])
    da = np.array([2 * np.pi * (i + 0.5) * dr ** 2 for i in range(nn)])
    r = np.sqrt(np.asarray(p[0], np.float64) ** 2 + np.asarray(p[1], np.float64) ** 2)
    return alpha[:-1], _weighted_bins(r, w, nn, dr) / (da * nPh)


def angularyResolved(v, w, nn, nPh):
    """R(alpha) over exit angle bins of pi/(2 nn) per solid angle
    (pymopt/metrics/_scoring.py:27-38)."""
    da = np.pi / (2 * nn)
    alpha = np.array([(i + 0.5) * da for i in range(nn + 1)])
    do = 4 * np.pi * np.sin(alpha) * np.sin(da / 2)
    at = np.arccos(np.sign(v[2]) * (v[2]))
    return alpha[:-1], _weighted_bins(at, w, nn, da) / (do[:-1] * nPh)


def lineDistance(p, w, nn, dr, nPh, y_range=5):
    """Profile along z of exits with |y| < y_range (pymopt/metrics/_scoring.py:40-51)."""
    alpha = np.array([i * dr for i in range(nn + 1)])
    da = np.ones(nn) * dr * y_range * 2
    ind = np.where(np.abs(p[1]) < y_range)[0]
    return alpha[:-1], _weighted_bins(np.asarray(p)[2, ind], np.asarray(w)[ind], nn, dr) / (da * nPh)
