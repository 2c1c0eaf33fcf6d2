"""The pymopt-compatible host API on CPU: volumes, sources, params handling,
metrics.  Fixtures come from the reference's own classes
(tests/golden/make_golden.py volumes / sources)."""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN
from pymonteopt_b200 import VoxelPlateExModel, VoxelPlateModel, VoxelTuringModel
from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import metrics
from pymonteopt_b200 import voxel as VX
from pymonteopt_b200.problem import pencil_problem

VOL = np.load(os.path.join(GOLDEN, "ref_volumes.npz"))
TURING_PARAMS = {"voxel_space": 0.1, "th_cortical": 1.0, "th_subcutaneus": 1.2, "th_dermis": 0.8}


def test_plate_volume_matches_reference():
    m = VX.PlateModel()
    m.verbose = False
    m.set_params(x_size=2.1, y_size=1.6, voxel_space=0.1, thickness=[0.3, 0.5, 0.2],
                 n=[1.4, 1.37, 1.45], n_air=1.0, ma=[0.1, 0.2, 0.3], ms=[10, 20, 30],
                 g=[0.9, 0.8, 0.7])
    m.build()
    assert np.array_equal(m.voxel_model, VOL["plate"])
    assert int(m.end_point) == 3


def _plate_layer_by_layer(m):
    """The reference's fill order (pymopt/voxel_gpu/_classes.py:437-457):
    each layer's z slab, then the six shell faces."""
    vm = np.zeros((m.x_size + 2, m.y_size + 2, m.z_size + 2), np.int8)
    val = 1
    for n_, t in enumerate(m.thickness):
        k = round(t / m.voxel_space)
        vm[:, :, val:val + k] = n_
        val += k
    e = len(m.thickness)
    vm[0], vm[-1], vm[:, 0], vm[:, -1], vm[:, :, 0], vm[:, :, -1] = e, e, e, e, e, e
    return vm


def test_plate_volume_fill_matches_layer_by_layer():
    """The column-broadcast fill gives the reference's bytes for random
    stacks of one to five layers, and for the skin slab."""
    from pymonteopt_b200 import volumes as V
    rng = np.random.default_rng(3)
    cases = [dict(V.C2_PARAMS)]
    for k in rng.integers(1, 6, 12):
        vs = float(rng.choice([0.05, 0.1, 0.2]))
        cases.append(dict(x_size=float(rng.integers(3, 30)) * vs,
                          y_size=float(rng.integers(3, 30)) * vs, voxel_space=vs,
                          thickness=[float(t) * vs for t in rng.integers(1, 25, k)],
                          n=[1.4] * k, n_air=1.0, ma=[0.1] * k, ms=[10.0] * k, g=[0.9] * k))
    for c in cases:
        m = VX.PlateModel()
        m.verbose = False
        m.set_params(**c)
        m.build()
        assert m.voxel_model.dtype == np.int8
        assert np.array_equal(m.voxel_model, _plate_layer_by_layer(m)), c


def test_plate_ex_volume_matches_reference():
    m = VX.PlateExModel()
    m.verbose = False
    m.set_params(x_size=2.0, y_size=1.5, voxel_space=0.1, thickness=[0.3, 1.0],
                 n=[1.5, 1.4], n_air=1.0, ma=[1e-5, 0.02], ms=[1e-5, 1.0], g=[0.9, 0.9])
    m.build()
    assert np.array_equal(m.voxel_model, VOL["plate_ex"])
    assert m.get_second_layer_addz() == int(0.3 / 0.1) + 1   # reference formula: 3


@pytest.mark.parametrize("name,extra", [("TuringModel_Rectangular", {"xz_size": 6.0}),
                                        ("TuringModel_Cylinder", {"r_bone": 3.5}),
                                        ("TuringModel_RnC", {"xz_size": 6.0, "r_bone": 3.5})])
def test_turing_volumes_match_reference(name, extra):
    m = VoxelTuringModel(nPh=100, model_name=name, verbose=False)
    m.set_model(VOL["bone"].copy())
    m.build(**TURING_PARAMS, **extra)
    assert np.array_equal(m.model.voxel_model, VOL[name])
    prob = m.transport_problem()
    prob.validate()   # padded shell, labels in range


def test_sources_match_reference():
    cases = json.load(open(os.path.join(GOLDEN, "ref_sources.json")))["cases"]
    for c in cases:
        m = VoxelPlateModel(nPh=c["n_transported"], verbose=False, **c["kwargs"])
        m.build(**c["params"])
        if c["name"] == "first_layer_clear":
            m.model.get_second_layer_addz = lambda: 6
        src = m._source()
        assert list(src["src_add"]) == c["add"], c["name"]
        np.testing.assert_allclose(src["src_p"], c["p"], atol=1e-7)
        np.testing.assert_allclose(src["src_v"], c["v"], atol=1e-6)
        assert abs(src["src_w0"] - c["w"]) < 1e-6, (c["name"], src["src_w0"], c["w"])
        if "spec_fraction" in c:
            # the reference draws the specular photons with NumPy; the device
            # draws them per photon from Philox: compare the probability
            n = 20000
            se = np.sqrt(src["spec_prob"] * (1 - src["spec_prob"]) / n)
            assert abs(src["spec_prob"] - c["spec_fraction"]) < 4 * se
            np.testing.assert_allclose(src["spec_v"], c["spec_v"], atol=1e-6)


def test_params_and_arguments_like_the_reference():
    m = VoxelPlateModel(nPh=10, verbose=False)
    with pytest.raises(KeyError):
        m.build(not_a_key=1)
    with pytest.raises(Exception):
        VoxelPlateModel(nPh=10, threadnum=2048)
    with pytest.raises(ValueError):
        VoxelPlateModel(nPh=10, beam_type="flat")
    with pytest.raises(ValueError):
        VoxelTuringModel(nPh=10, model_name="nope")
    ex = VoxelPlateExModel(nPh=10, verbose=False)
    assert ex.first_layer_clear is True
    # default PlateModel params of the reference (pymopt/voxel_gpu/_classes.py:402-411)
    assert VX.PlateModel().params["thickness"] == [1.3, 40]


def test_problem_validation_rejects_bad_volumes():
    vol = np.zeros((5, 5, 5), np.uint8)
    vol[0], vol[-1], vol[:, 0], vol[:, -1], vol[:, :, 0], vol[:, :, -1] = 1, 1, 1, 1, 1, 1
    ok = pencil_problem(vol, 0.1, 1, [0.1], [1.0], [0.9], [1.4, 1.0])
    ok.validate()
    bad = vol.copy()
    bad[0, 2, 2] = 0
    with pytest.raises(ValueError, match="shell"):
        pencil_problem(bad, 0.1, 1, [0.1], [1.0], [0.9], [1.4, 1.0]).validate()
    with pytest.raises(ValueError):
        pencil_problem(vol, 0.1, 1, [0.1], [-1.0], [0.9], [1.4, 1.0]).validate()
    with pytest.raises(ValueError):
        pencil_problem(vol, 0.1, 1, [np.nan], [1.0], [0.9], [1.4, 1.0]).validate()
    with pytest.raises(ValueError):
        pencil_problem(vol, 0.0, 1, [0.1], [1.0], [0.9], [1.4, 1.0]).validate()


def _radial_reference(p, w, nn, dr, nPh):
    """pymopt/metrics/_scoring.py:16-25, loop per bin as the reference does."""
    alpha = np.array([i * dr for i in range(nn + 1)])
    da = np.array([2 * np.pi * (i + 0.5) * dr ** 2 for i in range(nn)])
    r = np.sqrt(p[0] ** 2 + p[1] ** 2)
    out = []
    for i in range(nn):
        idx = np.where((alpha[i] < r) & (alpha[i + 1] >= r))[0]
        out.append(w[idx].sum())
    return alpha[:-1], np.array(out) / (da * nPh)


def test_metrics_match_reference_semantics():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 1.0, (3, 5000))
    p[:, :10] = np.round(p[:, :10], 1)          # exact bin edges
    w = rng.random(5000)
    a1, r1 = metrics.radialDistance(p, w, 40, 0.1, 5000)
    a2, r2 = _radial_reference(p, w, 40, 0.1, 5000)
    np.testing.assert_allclose(a1, a2)
    np.testing.assert_allclose(r1, r2, rtol=1e-12, atol=0)
    v = rng.normal(0, 1, (3, 5000))
    v /= np.linalg.norm(v, axis=0)
    _, ra = metrics.angularyResolved(v, w, 30, 5000)
    assert ra.shape == (30,) and np.all(ra >= 0)


def test_exit_encoding_like_reference():
    m = VoxelPlateModel(nPh=1, verbose=False)
    m.build(x_size=1.0, y_size=1.0, voxel_space=0.1, thickness=[1.0], n=[1.4], n_air=1.0,
            ma=[0.1], ms=[1.0], g=[0.9])
    add = np.array([[5, 0], [5, 6], [0, 11]])
    p = np.array([[0.01, 0.05], [-0.02, 0.0], [0.05, -0.05]], np.float32)
    enc = m._encooder(p, add)
    # x = l*(add_x - cx) + p_x with cx = int((12-1)/2) = 5; z = l*(add_z-1)+p_z+l/2
    np.testing.assert_allclose(enc[0], [0.01, -0.45], atol=1e-7)
    np.testing.assert_allclose(enc[2], [0.0, 1.0], atol=1e-6)


def test_model_builds_transport_problem():
    m = VoxelPlateModel(nPh=10, verbose=False, w_beam=1.0)
    m.build(x_size=2.0, y_size=2.0, voxel_space=0.1, thickness=[0.5, 0.5], n=[1.4, 1.45],
            n_air=1.0, ma=[0.1, 0.2], ms=[10, 20], g=[0.9, 0.8])
    prob = m.transport_problem()
    prob.validate()
    assert prob.source == A.PMO_SRC_GAUSSIAN and prob.beam_sigma == 0.5
    assert prob.end_label == 2 and prob.n_labels == 3


def test_reference_kernel_library_builds_and_exports():
    """oracle/ref_gpu_build.py: the reference's cuVMC source string is found
    and compiled; the launcher is exported (no GPU call)."""
    import ctypes
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(GOLDEN), "..", "oracle"))
    try:
        import ref_gpu_build
    finally:
        sys.path.pop(0)
    root = ref_gpu_build.default_reference_root()
    if root is not None:
        src = ref_gpu_build.extract(root)
        assert "__global__ void cuVMC(" in src and "curand_init" in src
        ref_gpu_build.build(reference_root=root)
    if not ref_gpu_build.available():
        pytest.skip("reference tree absent and no prebuilt reference kernel")
    lib = ctypes.CDLL(ref_gpu_build.LIB)
    assert hasattr(lib, "ref_cuvmc_launch")
