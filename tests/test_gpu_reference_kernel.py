"""The FP32 product against the reference's own GPU kernel.

``oracle/_ref/libcuvmc_ref.so`` is the reference's ``cuVMC``
(pymopt/voxel_gpu/_cukernel.py:27-227), compiled unchanged by
``oracle/ref_gpu_build.py``.  It runs here on the same volumes with the
reference's launch and read-back (``oracle/ref_gpu.py``).  Its RNG (cuRAND
XORWOW seeded per thread) differs from this kernel's Philox streams, so the
comparison is statistical: Rd and Tt within 3 sigma of the seed-to-seed
standard error (40 seeds a side), and R(r)/T(r) by a chi-square test over
the populated bins.
"""
import os
import sys

import numpy as np
import pytest
import torch
from scipy import stats

from helpers import annulus_area, mean_se, profile_agreement, z_score
from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import engine as E
from pymonteopt_b200 import volumes as V

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import ref_gpu  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(),
                                 reason="reference cuVMC library not built")]


def _ours(prob, seeds, n_per, nr, dr, cuda):
    dp = E.DeviceProblem(prob, cuda)
    area = annulus_area(nr, dr)
    out = {"Rd": [], "Tt": [], "Rr": [], "Tr": []}
    for s in seeds:
        t = E.run_plain(dp, n_per, s, spec=E.TallySpec(nr=nr, dr=dr))
        torch.cuda.synchronize()
        t.check()
        L = t.ledger.cpu().numpy()
        rr = t.rr.cpu().numpy().astype(np.float64)
        out["Rd"].append(L[A.PMO_L_RD] / n_per)
        out["Tt"].append(L[A.PMO_L_TT] / n_per)
        out["Rr"].append((rr[A.PMO_RR_TOP] + rr[A.PMO_RR_LAT_NEG]) / (area * n_per))
        out["Tr"].append((rr[A.PMO_RR_BOTTOM] + rr[A.PMO_RR_LAT_POS]) / (area * n_per))
    return out


def _theirs(prob, seeds, n_per, nr, dr, cuda):
    rv = ref_gpu.RefVolume(prob, cuda)
    out = {"Rd": [], "Tt": [], "Rr": [], "Tr": []}
    for s in seeds:
        r = rv.run(n_per, s, nr=nr, dr=dr)
        torch.cuda.synchronize()
        for k in out:
            out[k].append(r[k])
    return out


CASES = {
    # name: (problem factory, photons per seed, R(r) bins, bin width)
    "c1_slab": (V.c1_slab, 100000, 100, 0.1),
    "c2_pencil": (lambda: V.c2_skin(gaussian=False), 50000, 100, 0.1),
    "c3_ct_like": (lambda: V.c3_ct_like(0), 50000, 100, 0.2),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_statistics_match_reference_gpu_kernel(cuda, case):
    make, n_per, nr, dr = CASES[case]
    prob = make()
    # 40 seeds a side: with few seeds the per-bin z-scores follow a t
    # distribution and the chi-square over 100 bins is exceeded too easily
    mine = _ours(prob, range(300, 340), n_per, nr, dr, cuda)
    ref = _theirs(prob, range(1, 41), n_per, nr, dr, cuda)
    for q in ("Rd", "Tt"):
        m, s = mean_se(mine[q])
        rm, rs = mean_se(ref[q])
        if rm == 0 and rs == 0:
            assert m == 0
            continue
        assert abs(z_score(m, s, rm, rs)) < 3, (case, q, m, s, rm, rs)
    for q in ("Rr", "Tr"):
        m, s = mean_se(mine[q])
        z, chi2, dof = profile_agreement(m, s, ref[q])
        if dof == 0:
            continue
        assert stats.chi2.sf(chi2, dof) > 1e-3, (case, q, chi2, dof, np.round(z, 2))
        assert np.max(np.abs(z)) < 4.5, (case, q, np.round(z, 2))


def test_reference_kernel_conserves_launch_contract(cuda):
    """The launcher reproduces start(): every photon ends exited (|v| = 1,
    w > 0, its voxel index moved into the end-label shell before the exit
    test, pymopt/voxel_gpu/_cukernel.py:122-128) or killed by roulette
    (v = 0, w = 0)."""
    prob = V.c3_ct_like(0)
    rv = ref_gpu.RefVolume(prob, cuda)
    add, p, v, w = rv.initial_state(20000)
    rv.launch(add, p, v, w, seed=3)
    torch.cuda.synchronize()
    a, vv, ww = add.cpu().numpy(), v.cpu().numpy(), w.cpu().numpy()
    norm = np.sqrt((vv.astype(np.float64) ** 2).sum(0))
    killed = ww == 0
    assert np.all(norm[killed] == 0)
    assert np.all(np.abs(norm[~killed] - 1) < 1e-4)
    lab = prob.labels[a[0][~killed], a[1][~killed], a[2][~killed]]
    assert np.all(lab == prob.end_label)
