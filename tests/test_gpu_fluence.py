"""The 3D absorbed-weight grid and the fluence built from it.

The grid holds 64-bit fixed point (2^-32 weight units), so each voxel's sum
is exact and does not depend on the order in which atomics land.

* FP64 device build against the FP64 oracle on identical Philox streams:
  the grids agree voxel by voxel to the 2^-32 rounding of each deposit, up to
  the photons whose histories diverge on a last-ulp branch (each carries at
  most weight 1).  The check runs with voxel-by-voxel stepping and with
  uniform boxes, where the deposit voxel is recovered from the offset inside
  the box.
* The shared-memory window (``PMO_FLU_SHARED``) gives exactly the grid of the
  global atomics on the same photons, and so does a second run.
* ``normalize_fluence``: phi = absorbed / (nPh * l^3 * mu_a) in FP64 over the
  interior, and sum(phi * mu_a) * l^3 equals the absorbed fraction A.
"""
import numpy as np
import pytest
import torch

import oracle
from pymonteopt_b200 import VoxelPlateModel
from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import engine as E
from pymonteopt_b200 import volumes as V
from pymonteopt_b200.problem import pencil_problem

pytestmark = pytest.mark.gpu


def _plate(thickness, n, ma, ms, g, l=0.1, xy=3.0):
    vol, end = V.plate_volume(xy, xy, l, list(thickness))
    return pencil_problem(vol, l, end, list(ma), list(ms), list(g), list(n) + [1.0])


def _diverged(t, ref, cols=(0, 1, 2)):
    """Photons whose event counts (interactions, crossings, Fresnel) or exit
    state differ from the oracle's."""
    counts = t.ph.cpu().numpy().T.astype(np.uint32)
    cols = list(cols)
    same = np.all(counts[:, cols] == ref["ph_counts"][:, cols], axis=1)
    add = t.exit_add.cpu().numpy().T.astype(np.float64)
    p = t.exit_p.cpu().numpy().T.astype(np.float64)
    v = t.exit_v.cpu().numpy().T.astype(np.float64)
    w = t.exit_w.cpu().numpy().astype(np.float64)
    st = np.concatenate([p, v, w[:, None], add], axis=1)
    close = np.all(np.abs(st - ref["ph_state"]) <= 1e-6 * (1 + np.abs(ref["ph_state"])), axis=1)
    return int(np.count_nonzero(~(same & close)))


@pytest.mark.parametrize("skip", [False, True])
def test_absorbed_grid_matches_oracle_fp64(cuda, skip):
    prob = _plate((0.5, 0.5), (1.4, 1.5), (0.5, 0.2), (10.0, 20.0), (0.8, 0.9))
    n, seed = 4000, 21
    dp = E.DeviceProblem(prob, cuda, skip=skip)
    spec = E.TallySpec(nr=30, dr=0.1, fluence=A.PMO_FLU_GLOBAL, export_exits=True,
                       photon_stats=True)
    t = E.run_plain(dp, n, seed, spec=spec, precision=A.PMO_FP64)
    torch.cuda.synchronize()
    t.check()
    ref = oracle.run(prob, n, seed, precision=A.PMO_FP64, nr=30, dr=0.1, fluence=True,
                     per_photon=True)
    a = E.absorbed_weight(t).cpu().numpy()
    b = ref["absorbed"]
    assert a.shape == b.shape
    # box stepping counts box crossings, the oracle voxel crossings
    bad = _diverged(t, ref, cols=(0, 2) if skip else (0, 1, 2))
    assert bad <= 0.005 * n
    # deposits are rounded to 2^-32 each (one per interaction); a diverged
    # photon moves at most weight 1 between voxels
    rounding = float(t.host_counters()[A.PMO_C_INTERACT]) * 2.0 ** -33
    l1 = np.abs(a - b).sum()
    assert l1 <= 2.0 * bad + rounding, (l1, bad, rounding)
    if bad == 0:
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-6)
    # the shell receives nothing; the grid sums to the FP64 ledger
    assert a[0].sum() == 0 and a[-1].sum() == 0 and a[:, :, 0].sum() == 0
    L = t.ledger.cpu().numpy()
    assert abs(a.sum() - L[A.PMO_L_ABS]) <= 1e-9 * L[A.PMO_L_ABS]


def test_shared_window_matches_global_atomics(cuda):
    prob = V.c1_slab()
    cx, cy = prob.center
    lo, dim = (cx - 8, cy - 8, 1), (17, 17, 24)
    dp = E.DeviceProblem(prob, cuda)
    n, seed = 200000, 5
    grids = []
    for flu, win in ((A.PMO_FLU_GLOBAL, None), (A.PMO_FLU_SHARED, (lo, dim)),
                     (A.PMO_FLU_GLOBAL, None)):
        t = E.run_plain(dp, n, seed, spec=E.TallySpec(nr=100, dr=0.1, fluence=flu, window=win))
        torch.cuda.synchronize()
        t.check()
        grids.append(t.absorbed.clone())
    # same photons, same fixed-point deposits: integer sums are exact, so the
    # grids are equal whatever the order of the atomics
    assert torch.equal(grids[1], grids[0])
    assert torch.equal(grids[2], grids[0])
    g0 = grids[0].double().cpu().numpy()
    inside = g0[lo[0]:lo[0] + dim[0], lo[1]:lo[1] + dim[1], lo[2]:lo[2] + dim[2]].sum()
    assert inside > 0.2 * g0.sum()   # the window path carried a good share


def test_normalized_fluence(cuda):
    prob = _plate((1.0, 1.0), (1.37, 1.4), (0.3, 0.05), (10.0, 15.0), (0.9, 0.8), l=0.1)
    n = 100000
    dp = E.DeviceProblem(prob, cuda)
    t = E.run_plain(dp, n, 3, spec=E.TallySpec(nr=30, dr=0.1, fluence=A.PMO_FLU_GLOBAL))
    phi = E.normalize_fluence(dp, t).cpu().numpy()
    torch.cuda.synchronize()
    absorbed = E.absorbed_weight(t).cpu().numpy()[1:-1, 1:-1, 1:-1]
    lab = prob.labels[1:-1, 1:-1, 1:-1]
    ma = np.where(lab == prob.end_label, 0.0, prob.ma.astype(np.float64)[np.minimum(lab, len(prob.ma) - 1)])
    l = float(np.float32(prob.voxel_space))
    want = np.where(ma > 0, absorbed / (n * l ** 3 * np.where(ma > 0, ma, 1.0)), 0.0)
    np.testing.assert_allclose(phi, want, rtol=1e-12, atol=0)
    L = t.ledger.cpu().numpy()
    assert abs((phi * ma).sum() * l ** 3 - L[A.PMO_L_ABS] / n) < 1e-7 * L[A.PMO_L_ABS] / n


def test_model_fluence_getter(cuda):
    m = VoxelPlateModel(nPh=50000, fluence=True, verbose=False)
    m.build(x_size=2.0, y_size=2.0, voxel_space=0.1, thickness=[0.5, 0.5], n=[1.4, 1.45],
            n_air=1.0, ma=[0.2, 0.1], ms=[10, 20], g=[0.9, 0.8])
    m.start(rand_seed=4)
    phi = m.get_fluence()
    shape = m._tallies.absorbed.shape
    assert phi.shape == (shape[0] - 2, shape[1] - 2, shape[2] - 2)
    assert np.all(phi >= 0) and phi.max() > 0
    res = m.getRdTtValues()
    # the fluence integrates to the absorbed fraction
    lab = m.transport_problem().labels[1:-1, 1:-1, 1:-1]
    ma = np.array([0.2, 0.1, 0.0])[np.minimum(lab, 2)]
    a = (phi * ma).sum() * np.float32(0.1) ** 3
    assert abs(a - res["A"]) < 1e-4, (a, res["A"])
