"""Shared helpers of the test-suite: golden fixtures and statistics."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str) -> dict:
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def mean_se(samples):
    a = np.asarray(samples, np.float64)
    return a.mean(axis=0), a.std(axis=0, ddof=1) / np.sqrt(a.shape[0])


def annulus_area(nr: int, dr: float) -> np.ndarray:
    """2*pi*(i + 1/2)*dr^2 (pymopt/metrics/_scoring.py:18)."""
    return np.array([2 * np.pi * (i + 0.5) * dr ** 2 for i in range(nr)])


def z_score(m1, s1, m2, s2):
    den = np.sqrt(np.asarray(s1) ** 2 + np.asarray(s2) ** 2)
    return np.where(den > 0, (np.asarray(m1) - np.asarray(m2)) / np.where(den > 0, den, 1), 0.0)


def profile_agreement(mine, mine_se, ref_samples, min_nonzero: int = 5):
    """Per-bin z-scores of a radial profile against per-seed reference
    profiles, over the bins that most reference seeds populate.  Returns
    (z, chi2, dof)."""
    ref = np.asarray(ref_samples, np.float64)
    rm, rs = mean_se(ref)
    keep = (np.count_nonzero(ref, axis=0) >= min_nonzero) & (rs > 0)
    z = z_score(np.asarray(mine)[keep], np.asarray(mine_se)[keep], rm[keep], rs[keep])
    return z, float(np.sum(z ** 2)), int(keep.sum())
