"""Batched layered slabs (pmo_run_stack_batch / StackBatch).

* A stack of one layer draws the Philox streams and does the arithmetic of
  the single-layer slab kernel: same seed, same photons, same sums (FP64 and
  FP32), same derivatives and R(r).
* The reference's own three-layer PlateModel runs (tests/golden/
  ref_three_layer.json; 10 mm wide, 0.4 mm thick, so lateral escape is
  negligible) against the stack form: Rd, Tt within 3 sigma, R(r), T(r) by
  chi-square.
* A stack with index steps between layers against the CPU oracle on a wide
  voxel plate of the same layers.
* Per-layer derivatives against pathwise central differences (the stack
  kernel itself re-run at mu * (1 +- h) on common random numbers).
* Energy ledger, completion, CUDA-graph replay, malformed stacks.
"""
import numpy as np
import pytest
import torch
from scipy import stats

import oracle
from helpers import annulus_area, golden, mean_se, profile_agreement, z_score
from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import batched as B
from pymonteopt_b200 import volumes as V

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [A.PMO_FP64, A.PMO_FP32])
def test_one_layer_stack_follows_slab_batch(cuda, precision):
    slabs = [(0.3, 8.0, 0.85, 1.4, 2.0), (0.02, 15.0, 0.9, 1.33, 5.0), (1.0, 3.0, 0.7, 1.45, 1.0)]
    N = 30000
    ma, ms, g, n, t = (np.array([s[i] for s in slabs], np.float32) for i in range(5))
    sb = B.SlabBatch(ma, ms, g, n, t, np.full(3, N), nr=20, dr=0.2, seed=77,
                     precision=precision, autotune=False, block_threads=128, chunk=256,
                     tally_mode=A.PMO_BT_GLOBAL)
    ref = sb.run(use_graph=False)
    st = B.StackBatch([[s] for s in slabs], N, nr=20, dr=0.2, seed=77, precision=precision)
    got = st.run(use_graph=False)
    S, T = ref["sums"], got["sums"]
    pairs = [(A.PMO_BS_RD, A.PMO_SS_RD), (A.PMO_BS_TT, A.PMO_SS_TT), (A.PMO_BS_ABS, A.PMO_SS_ABS),
             (A.PMO_BS_WINIT, A.PMO_SS_WINIT), (A.PMO_BS_INTER, A.PMO_SS_INTER),
             (A.PMO_BS_RD_L, A.PMO_SS_LAYER0), (A.PMO_BS_RD_N, A.PMO_SS_LAYER0 + 1),
             (A.PMO_BS_TT_L, A.PMO_SS_LAYER0 + 2), (A.PMO_BS_TT_N, A.PMO_SS_LAYER0 + 3)]
    for bs, ss in pairs:
        # identical photons; sums differ only by the order of FP64 atomics
        np.testing.assert_allclose(T[:, ss], S[:, bs], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(got["dRd_dma"][:, 0], ref["dRd_dma"], rtol=1e-9)
    np.testing.assert_allclose(got["dTt_dms"][:, 0], ref["dTt_dms"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(got["Rr"], ref["Rr"], rtol=1e-5, atol=1e-9)
    # per-bin derivatives are differences of two float32 atomic sums: compare
    # them against the size of the profile
    for col in ("dRr_dma", "dRr_dms"):
        scale = np.abs(ref[col]).max(axis=1, keepdims=True)
        assert np.all(np.abs(got[col][:, :, 0] - ref[col]) <= 1e-4 * scale), col


def test_three_layer_stack_matches_reference(cuda):
    g = golden("ref_three_layer.json")
    p = g["params"]
    layers = [(p["ma"][i], p["ms"][i], p["g"][i], p["n"][i], p["thickness"][i])
              for i in range(3)]
    copies, N = 20, 100000   # 20 copies of the problem: 20 independent samples
    st = B.StackBatch([layers] * copies, N, n_ambient=p["n_air"], nr=g["nr"], dr=g["dr"],
                      seed=5)
    r = st.run(use_graph=False)
    mine = {"Rd": r["Rd"], "Tt": r["Tt"], "Rr": r["Rr"]}
    for key in ("Rd", "Tt"):
        m, s = mean_se(mine[key])
        rm, rs = mean_se(g[key])
        assert abs(z_score(m, s, rm, rs)) < 3, (key, m, s, rm, rs)
    m, s = mean_se(mine["Rr"])
    z, chi2, dof = profile_agreement(m, s, g["Rr"])
    assert dof > 20
    assert stats.chi2.sf(chi2, dof) > 1e-3, (chi2, dof, np.round(z, 2))
    assert np.max(np.abs(z)) < 4.5, np.round(z, 2)
    assert np.all(np.abs(r["balance"]) < 1e-9)


def test_stack_with_index_steps_matches_oracle(cuda):
    """Layers of different refractive index (Fresnel at the inner planes)
    against the oracle on a 40 mm wide voxel plate of the same layers."""
    layers = [(0.3, 12.0, 0.8, 1.45, 0.3), (0.05, 8.0, 0.9, 1.33, 0.5), (0.2, 15.0, 0.85, 1.5, 1.0)]
    nr, dr = 30, 0.1
    copies, N = 20, 100000
    st = B.StackBatch([layers] * copies, N, nr=nr, dr=dr, seed=31)
    r = st.run(use_graph=False)
    prob = V.plate_problem(dict(x_size=40.0, y_size=40.0, voxel_space=0.1,
                                thickness=[L[4] for L in layers], n=[L[3] for L in layers],
                                n_air=1.0, ma=[L[0] for L in layers], ms=[L[1] for L in layers],
                                g=[L[2] for L in layers]))
    area = annulus_area(nr, dr)
    ref = {"Rd": [], "Tt": [], "Rr": []}
    No = 20000
    for seed in range(20):
        o = oracle.run(prob, No, 600 + seed, precision=A.PMO_FP32, nr=nr, dr=dr)
        L = o["ledger"]
        ref["Rd"].append(L[A.PMO_L_RD] / No)
        ref["Tt"].append(L[A.PMO_L_TT] / No)
        ref["Rr"].append((o["rr"][A.PMO_RR_TOP] + o["rr"][A.PMO_RR_LAT_NEG]) / (area * No))
    for key in ("Rd", "Tt"):
        m, s = mean_se(r[key])
        rm, rs = mean_se(ref[key])
        assert abs(z_score(m, s, rm, rs)) < 3, (key, m, s, rm, rs)
    m, s = mean_se(r["Rr"])
    z, chi2, dof = profile_agreement(m, s, ref["Rr"])
    assert stats.chi2.sf(chi2, dof) > 1e-3, (chi2, dof, np.round(z, 2))
    assert np.max(np.abs(z)) < 4.5, np.round(z, 2)


def test_stack_gradients_match_pathwise_fd(cuda):
    """dRd/dmu of each layer against central differences of the stack kernel
    re-run with that layer's mu * (1 +- h), same seed (common random numbers),
    over 6 seeds."""
    base = [(0.2, 10.0, 0.85, 1.4, 0.2), (0.05, 6.0, 0.9, 1.4, 0.8), (0.1, 8.0, 0.8, 1.44, 2.0)]
    h, N = 3e-2, 400000
    est = {}
    fd = {}
    for seed in range(6):
        r = B.StackBatch([base], N, seed=40 + seed, nr=0).run(use_graph=False)
        for li in range(3):
            for which, k in (("ma", 0), ("ms", 1)):
                key = (li, which)
                est.setdefault(key, []).append(r["dRd_d" + which][0, li])
                vals = []
                for sgn in (1.0, -1.0):
                    lay = [list(L) for L in base]
                    lay[li][k] *= 1 + sgn * h
                    rr = B.StackBatch([lay], N, seed=40 + seed, nr=0).run(use_graph=False)
                    vals.append(rr["Rd"][0])
                fd.setdefault(key, []).append((vals[0] - vals[1]) / (2 * h * base[li][k]))
    for key in est:
        a, f = np.array(est[key]), np.array(fd[key])
        se = np.sqrt(a.var(ddof=1) / len(a) + f.var(ddof=1) / len(f))
        assert abs(a.mean() - f.mean()) < 3 * se + 0.02 * abs(f.mean()), \
            (key, a.mean(), f.mean(), se)


def test_stack_ledger_completion_graph_and_bad_stack(cuda):
    rng = np.random.default_rng(2)
    stacks = []
    for _ in range(40):
        nl = int(rng.integers(1, A.PMO_MAX_LAYERS + 1))
        stacks.append([(float(rng.uniform(0.01, 0.5)), float(rng.uniform(2, 20)),
                        float(rng.uniform(0.7, 0.95)), float(rng.uniform(1.33, 1.5)),
                        float(rng.uniform(0.05, 2.0))) for _ in range(nl)])
    photons = rng.integers(2000, 20000, size=40)
    st = B.StackBatch(stacks, photons, nr=16, dr=0.2, seed=3)
    direct = st.run(use_graph=False)
    assert np.all(np.abs(direct["balance"]) < 1e-9)
    assert np.all(direct["completion_ms"] > 0)
    assert np.all(st.remaining.cpu().numpy() == 0)
    # derivative slots beyond a problem's own layers stay zero
    for i, s in enumerate(stacks):
        assert np.all(direct["dRd_dma"][i, len(s):] == 0)
    graphed = st.run(use_graph=True)
    np.testing.assert_allclose(graphed["Rd"], direct["Rd"], rtol=1e-6)
    np.testing.assert_allclose(graphed["dRd_dms"], direct["dRd_dms"], rtol=1e-5, atol=1e-12)
    # a stack row that points past the layer table: its photons count as error
    # weight instead of reading outside the table
    bad = st.host_stacks.copy()
    bad[0]["first_layer"] = len(st.host_layers)
    st.stacks.copy_(torch.from_numpy(bad.view(np.uint8).copy()).to(cuda))
    r = st.run(use_graph=False)
    S = r["sums"][0]
    assert S[A.PMO_SS_ERRW] == photons[0] and S[A.PMO_SS_RD] == 0


def test_stack_sweep_against_plain_comparator(cuda):
    """The bench's layered leg on a small sweep: the batch and the reused
    plain comparator both run, the batch closes its ledger, and on the sweep's
    first problem the plain path's Rd agrees with the stack's within the
    difference a 20 mm wide plate makes (lateral escape) plus noise."""
    from pymonteopt_b200 import volumes as V
    out = B.stacks_vs_plain(count=32, plain_sample=4, device=cuda)
    assert out["problems"] == 32 and out["ratio"] > 0
    assert out["max_energy_residual"] < 1e-9
    sw = V.skin_stack_sweep(seed=0, count=32)
    layers, N = sw["stacks"][0], 400000
    ev = B.PlainStackEvaluator(V.SKIN_LAYERS, N, device=cuda)
    plain = ev.evaluate(layers, N, 7)
    stack = B.StackBatch([layers], N, seed=7, nr=32, dr=0.1).run(use_graph=False)
    assert abs(plain["Rd"] - stack["Rd"][0]) < 0.01, (plain["Rd"], stack["Rd"][0])
    # both are derivatives of the sum of the 32 R(r) bins
    for li in range(3):
        a, b = plain["dR_dma"][li], float(stack["dRr_dma"][0, :, li].sum())
        assert np.sign(a) == np.sign(b) and abs(a - b) <= 0.1 * abs(b) + 1e-3, (li, a, b)


def test_stack_autotuner_picks_a_shape_and_shapes_agree(cuda):
    """The launch shape changes neither the photons nor the results."""
    sw = V.skin_stack_sweep(seed=4, count=24)
    photons = np.maximum(2000, sw["n_photons"] // 10)
    tuned = B.StackBatch(sw["stacks"], photons, nr=16, dr=0.1, seed=8, autotune=True)
    assert (tuned.block_threads, tuned.chunk) == tuned.tune_table["best"]
    assert len(tuned.tune_table["ms"]) == 9
    fixed = B.StackBatch(sw["stacks"], photons, nr=16, dr=0.1, seed=8, block_threads=64,
                         chunk=1024)
    a, b = tuned.run(use_graph=False), fixed.run(use_graph=False)
    np.testing.assert_allclose(a["sums"], b["sums"], rtol=1e-10, atol=1e-10)
