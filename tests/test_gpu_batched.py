"""Batched slab problems (pmo_run_batched / SlabBatch).

* Problem 0 of a batch draws the Philox streams of pmo_run_plain, so in FP64
  the batched slab kernel and the plain voxel kernel on the same slab (one
  z voxel of the slab's thickness, lateral walls far away) follow the same
  photon paths: sums agree to rounding, interaction counts exactly.
* FP32 statistics of random C5-style slabs match the CPU oracle within 3
  sigma.
* The in-pass derivatives match pathwise central differences on common random
  numbers (the batched kernel itself at mu * (1 +- h)).
* Energy ledger, completion times and CUDA-graph replay.
"""
import numpy as np
import pytest
import torch

import oracle
from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import batched as B
from pymonteopt_b200 import engine as E
from pymonteopt_b200 import volumes as V
from pymonteopt_b200.problem import pencil_problem

pytestmark = pytest.mark.gpu


def _voxel_slab(ma, ms, g, n, t, half=60):
    """The slab as a reference PlateModel volume: one z voxel of size t and
    2*half+1 lateral voxels."""
    k = 2 * half + 1
    vol = np.ones((k + 2, k + 2, 3), np.uint8)
    vol[1:-1, 1:-1, 1] = 0
    return pencil_problem(vol, t, 1, [ma], [ms], [g], [n, 1.0])


def _batch(params, photons, **kw):
    ma, ms, g, n, t = (np.array([p[i] for p in params], np.float32) for i in range(5))
    return B.SlabBatch(ma, ms, g, n, t, np.array(photons), autotune=False, block_threads=128,
                       chunk=256, **kw)


def test_problem0_follows_plain_kernel_fp64(cuda):
    ma, ms, g, n, t = 0.3, 8.0, 0.85, 1.4, 2.0
    N = 20000
    sb = _batch([(ma, ms, g, n, t)], [N], precision=A.PMO_FP64, nr=20, dr=0.2, seed=77)
    res = sb.run(use_graph=False)
    prob = _voxel_slab(ma, ms, g, n, t)
    dp = E.DeviceProblem(prob, cuda)
    tal = E.run_plain(dp, N, 77, spec=E.TallySpec(nr=20, dr=0.2), precision=A.PMO_FP64)
    torch.cuda.synchronize()
    tal.check()
    L = tal.ledger.cpu().numpy()
    c = tal.host_counters()
    S = res["sums"][0]
    assert int(S[A.PMO_BS_INTER]) == int(c[A.PMO_C_INTERACT])
    for bs, ls in ((A.PMO_BS_RD, A.PMO_L_RD), (A.PMO_BS_TT, A.PMO_L_TT), (A.PMO_BS_ABS, A.PMO_L_ABS)):
        assert abs(S[bs] - L[ls]) <= 1e-9 * max(L[ls], 1.0), (bs, S[bs], L[ls])
    rr = tal.rr.cpu().numpy().astype(np.float64)
    area = np.array([2 * np.pi * (i + 0.5) * 0.2 ** 2 for i in range(20)])
    R_plain = (rr[A.PMO_RR_TOP] + rr[A.PMO_RR_LAT_NEG]) / (area * N)
    np.testing.assert_allclose(res["Rr"][0], R_plain, rtol=1e-5, atol=1e-9)


def test_batched_statistics_match_oracle(cuda):
    rng = np.random.default_rng(4)
    params = []
    for _ in range(4):
        g = rng.uniform(0.7, 0.95)
        params.append((float(np.exp(rng.uniform(np.log(0.01), np.log(1.0)))),
                       float(np.exp(rng.uniform(np.log(0.5), np.log(5.0))) / (1 - g)), g,
                       float(rng.uniform(1.33, 1.45)), float(rng.uniform(1.0, 8.0))))
    N = 50000
    reps = []
    for seed in range(6):
        sb = _batch(params, [N] * len(params), seed=500 + seed)
        r = sb.run(use_graph=False)
        reps.append(np.stack([r["Rd"], r["Tt"]]))
    reps = np.array(reps)
    gm, gs = reps.mean(0), reps.std(0, ddof=1) / np.sqrt(len(reps))
    for i, (ma, ms, g, n, t) in enumerate(params):
        prob = _voxel_slab(ma, ms, g, n, t)
        vals = []
        for seed in range(6):
            o = oracle.run(prob, 20000, 900 + seed, precision=A.PMO_FP32)
            vals.append([o["ledger"][A.PMO_L_RD] / 20000, o["ledger"][A.PMO_L_TT] / 20000])
        vals = np.array(vals)
        om, os_ = vals.mean(0), vals.std(0, ddof=1) / np.sqrt(len(vals))
        for q in range(2):
            se = np.hypot(gs[q, i], os_[q])
            assert abs(gm[q, i] - om[q]) <= 3 * se + 1e-6, (i, q, gm[q, i], om[q], se)


def test_batched_rr_matches_oracle(cuda):
    """R(r) of four C5-style slabs, 6 batched seeds against 6 oracle seeds on
    the voxel plate of each slab: chi-square over the populated bins."""
    from scipy import stats
    from helpers import annulus_area, mean_se, profile_agreement
    rng = np.random.default_rng(11)
    params = []
    for _ in range(4):
        g = rng.uniform(0.7, 0.95)
        params.append((float(np.exp(rng.uniform(np.log(0.005), np.log(0.5)))),
                       float(np.exp(rng.uniform(np.log(0.5), np.log(5.0))) / (1 - g)), g,
                       float(rng.uniform(1.33, 1.45)), float(rng.uniform(1.0, 8.0))))
    nr, dr, N, No = 20, 0.2, 100000, 40000
    mine = []
    for seed in range(6):
        sb = _batch(params, [N] * len(params), seed=700 + seed, nr=nr, dr=dr)
        mine.append(sb.run(use_graph=False)["Rr"])
    mine = np.array(mine)                      # (seeds, problems, nr)
    area = annulus_area(nr, dr)
    for i, (ma, ms, g, n, t) in enumerate(params):
        prob = _voxel_slab(ma, ms, g, n, t)
        ref = []
        for seed in range(6):
            o = oracle.run(prob, No, 1900 + seed, precision=A.PMO_FP32, nr=nr, dr=dr)
            rr = o["rr"]
            ref.append((rr[A.PMO_RR_TOP] + rr[A.PMO_RR_LAT_NEG]) / (area * No))
        m, s_ = mean_se(mine[:, i])
        z, chi2, dof = profile_agreement(m, s_, ref)
        assert dof >= 10, (i, dof)
        assert stats.chi2.sf(chi2, dof) > 1e-3, (i, chi2, dof, np.round(z, 2))
        assert np.max(np.abs(z)) < 4.5, (i, np.round(z, 2))


def test_plain_slab_evaluator_matches_batched_problem0(cuda):
    """The reused-buffer comparator of the batched benchmark gives the same
    Rd and per-label derivatives as the batched form's problem 0 (which draws
    the plain kernel's Philox streams), within statistical error."""
    ma, ms, g, n, t = 0.05, 8.0, 0.85, 1.4, 3.0
    N = 400000
    ev = B.PlainSlabEvaluator(N, nr=32, dr=0.1, device=cuda)
    got = ev.evaluate(ma, ms, g, n, t, N, 123)
    sb = _batch([(ma, ms, g, n, t)], [N], seed=123, nr=32, dr=0.1)
    r = sb.run(use_graph=False)
    assert abs(got["Rd"] - r["Rd"][0]) < 1e-3, (got["Rd"], r["Rd"][0])
    # the evaluator's derivatives are of the sum of the R(r) bins
    for key, col in (("dR_dma", "dRr_dma"), ("dR_dms", "dRr_dms")):
        ref = float(r[col][0].sum())
        assert abs(got[key] - ref) <= 0.05 * abs(ref) + 1e-6, (key, got[key], ref)


def test_batched_gradients_match_pathwise_fd(cuda):
    base = (0.05, 6.0, 0.8, 1.37, 3.0)
    h = 3e-2
    est = {"ma": [], "ms": []}
    fd = {"ma": [], "ms": []}
    for seed in range(6):
        sb = _batch([base], [400000], seed=40 + seed)
        r = sb.run(use_graph=False)
        est["ma"].append(r["dRd_dma"][0])
        est["ms"].append(r["dRd_dms"][0])
        for which, k in (("ma", 0), ("ms", 1)):
            vals = []
            for sgn in (1.0, -1.0):
                p = list(base)
                p[k] *= 1 + sgn * h
                rr = _batch([tuple(p)], [400000], seed=40 + seed).run(use_graph=False)
                vals.append(rr["Rd"][0])
            fd[which].append((vals[0] - vals[1]) / (2 * h * base[k]))
    for which in ("ma", "ms"):
        a, f = np.array(est[which]), np.array(fd[which])
        se = np.sqrt(a.var(ddof=1) / len(a) + f.var(ddof=1) / len(f))
        assert abs(a.mean() - f.mean()) < 3 * se + 0.01 * abs(f.mean()), (which, a.mean(), f.mean(), se)


def test_batch_ledger_completion_and_graph(cuda):
    b = V.c5_slab_batch(seed=3, count=64)
    photons = np.maximum(1000, b["n_photons"] // 100)
    sb = B.SlabBatch(b["ma"], b["ms"], b["g"], b["n"], b["thickness"], photons, nr=16, dr=0.2,
                     seed=1, autotune=False, block_threads=128, chunk=256)
    direct = sb.run(use_graph=False)
    assert np.all(np.abs(direct["balance"]) < 1e-6)
    assert np.all(direct["completion_ms"] > 0)
    assert np.all(sb.remaining.cpu().numpy() == 0)
    graphed = sb.run(use_graph=True)
    # same photons: identical up to the order of floating-point atomics
    np.testing.assert_allclose(graphed["Rd"], direct["Rd"], rtol=1e-6)
    np.testing.assert_allclose(graphed["dRd_dma"], direct["dRd_dma"], rtol=1e-5)
    np.testing.assert_allclose(graphed["Rr"], direct["Rr"], rtol=1e-4, atol=1e-9)
    again = sb.run(use_graph=True)
    np.testing.assert_allclose(again["Tt"], graphed["Tt"], rtol=1e-6)


def test_tally_modes_agree_and_autotuner_picks_one(cuda):
    """Per-thread privatised sums and direct global atomics see the same
    photons; the autotuner times both and keeps one."""
    b = V.c5_slab_batch(seed=5, count=48)
    photons = np.maximum(500, b["n_photons"] // 200)
    common = dict(nr=16, dr=0.2, seed=9, autotune=False, block_threads=128, chunk=64)
    runs = {}
    for mode in (A.PMO_BT_THREAD, A.PMO_BT_GLOBAL):
        sb = B.SlabBatch(b["ma"], b["ms"], b["g"], b["n"], b["thickness"], photons,
                         tally_mode=mode, **common)
        runs[mode] = sb.run(use_graph=False)
        assert np.all(sb.remaining.cpu().numpy() == 0)
        assert np.all(runs[mode]["completion_ms"] > 0)
    t, g = runs[A.PMO_BT_THREAD], runs[A.PMO_BT_GLOBAL]
    np.testing.assert_allclose(g["sums"], t["sums"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(g["Rr"], t["Rr"], rtol=1e-5, atol=1e-9)
    assert np.all(np.abs(g["balance"]) < 1e-9)
    tuned = B.SlabBatch(b["ma"], b["ms"], b["g"], b["n"], b["thickness"], photons, nr=16,
                        dr=0.2, seed=9, block_threads=128, chunk=64)
    assert tuned.tally_mode in (A.PMO_BT_THREAD, A.PMO_BT_GLOBAL)
    assert set(tuned.tune_table["mode_ms"]) == {"thread", "global"}
