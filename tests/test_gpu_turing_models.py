"""Transport on the Turing-pattern bone models, through the CUDA path.

``VoxelTuringModel`` feeds the reference's dataset driver: a bone volume
(here the seeded 60 x 40 x 60 pattern of tests/golden/ref_volumes.npz) set into
the rectangular, cylindrical or combined shells of cortical bone, subcutis
and dermis (pymopt/voxel_gpu/_classes.py:554-822).  Their volumes equal the
reference's (tests/test_host_api.py); here the transport on them is held to
the oracle:

* the FP64 build, stepping voxel by voxel, follows the oracle photon by
  photon (event counts and exit state), on identical Philox streams;
* the FP32 product through the model API (box stepping) agrees with the
  oracle's FP32 Rd, Tt and absorbed fraction within 4 combined standard
  errors, and its ledger closes.
"""
import os

import numpy as np
import pytest
import torch

import oracle
from helpers import GOLDEN
from pymonteopt_b200 import VoxelTuringModel
from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import engine as E

pytestmark = pytest.mark.gpu

VOL = np.load(os.path.join(GOLDEN, "ref_volumes.npz"))
PARAMS = {"voxel_space": 0.1, "th_cortical": 1.0, "th_subcutaneus": 1.2, "th_dermis": 0.8}
MODELS = [("TuringModel_Rectangular", {"xz_size": 6.0}),
          ("TuringModel_Cylinder", {"r_bone": 3.5}),
          ("TuringModel_RnC", {"xz_size": 6.0, "r_bone": 3.5})]


def _model(name, extra, n, cuda):
    m = VoxelTuringModel(nPh=n, model_name=name, verbose=False, keep_exits=False, device=cuda)
    m.set_model(VOL["bone"].copy())
    m.build(**PARAMS, **extra)
    return m


@pytest.mark.parametrize("name,extra", MODELS, ids=[m[0] for m in MODELS])
def test_fp64_build_follows_oracle_per_photon(cuda, name, extra):
    prob = _model(name, extra, 4000, cuda).transport_problem()
    n, seed = 4000, 23
    dp = E.DeviceProblem(prob, cuda, skip=False)
    spec = E.TallySpec(nr=30, dr=0.1, export_exits=True, photon_stats=True)
    t = E.run_plain(dp, n, seed, spec=spec, precision=A.PMO_FP64)
    torch.cuda.synchronize()
    t.check()
    ref = oracle.run(prob, n, seed, precision=A.PMO_FP64, nr=30, dr=0.1, per_photon=True)
    assert ref["status"] == 0
    same = np.all(t.ph.cpu().numpy().T.astype(np.uint32) == ref["ph_counts"][:, :3], axis=1)
    st = np.concatenate([t.exit_p.cpu().numpy().T, t.exit_v.cpu().numpy().T,
                         t.exit_w.cpu().numpy()[:, None],
                         t.exit_add.cpu().numpy().T], axis=1).astype(np.float64)
    close = np.all(np.abs(st - ref["ph_state"]) <= 1e-6 * (1 + np.abs(ref["ph_state"])), axis=1)
    share = (same & close).mean()
    assert share >= 0.995, (name, share)


@pytest.mark.parametrize("name,extra", MODELS, ids=[m[0] for m in MODELS])
def test_model_api_matches_oracle_statistics(cuda, name, extra):
    n_gpu, n_ref = 2_000_000, 200_000
    m = _model(name, extra, n_gpu, cuda)
    vals = m.start(31).getRdTtValues()
    ref = oracle.run(m.transport_problem(), n_ref, 31, precision=A.PMO_FP32, threads=8)
    assert ref["status"] == 0
    RL = ref["ledger"] / n_ref
    for key, slot in (("Rd", A.PMO_L_RD), ("Tt", A.PMO_L_TT), ("A", A.PMO_L_ABS)):
        mine, theirs = vals[key], RL[slot]
        se = np.hypot(np.sqrt(max(mine * (1 - mine), 1e-12) / n_gpu),
                      np.sqrt(max(theirs * (1 - theirs), 1e-12) / n_ref))
        assert abs(mine - theirs) < 4 * se, (name, key, mine, theirs, (mine - theirs) / se)
    L = m.get_ledger()
    assert abs(L["balance"]) < 1e-6 * (L["w_init"] + L["roulette_gain"]), L
