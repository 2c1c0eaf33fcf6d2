"""On-device angle-resolved and line-profile exit tallies.

Each device histogram is checked against the host restatement of the
reference's scoring (``pymonteopt_b200.metrics``, itself checked against the
reference's functions in ``tests/test_host_api.py``).  That restatement runs
on the exit states the same run exports:

* R(alpha)/T(alpha): ``angularyResolved`` over the exits with v_z < 0 / v_z > 0
  (pymopt/metrics/_scoring.py:27-38);
* the side-face line profile: ``lineDistance`` over the exits with v_x < 0
  (pymopt/metrics/_scoring.py:40-51, as pymopt/virtualOBD.py:171-172 calls it).
"""
import numpy as np
import pytest

from pymonteopt_b200 import VoxelPlateModel
from pymonteopt_b200 import metrics

pytestmark = pytest.mark.gpu


def _model(**kw):
    m = VoxelPlateModel(nPh=200000, n_ang=30, n_line=60, line_dr=0.05, line_y_range=0.6,
                        keep_exits=True, verbose=False, **kw)
    # a narrow slab, so many photons leave through the side faces
    m.build(x_size=2.0, y_size=2.0, voxel_space=0.05, thickness=[1.0, 1.0], n=[1.37, 1.45],
            n_air=1.0, ma=[0.1, 0.05], ms=[8.0, 12.0], g=[0.85, 0.9])
    return m


def _edge_slack(v, w, nn, n):
    """Per-bin weight (in the histogram's units) of the exits whose angle lies
    within 1e-5 bin widths of a bin edge.  The device takes arccos and divides
    by the bin width in single precision (error below 4e-6 bin widths), the
    host in double, so such an exit may be counted one bin over."""
    da = np.pi / (2 * nn)
    t = np.arccos(np.abs(np.asarray(v[2], np.float64))) / da
    e = np.rint(t).astype(np.int64)
    amb = np.abs(t - e) < 1e-5
    slack = np.zeros(nn)
    for side in (e[amb] - 1, e[amb]):
        ok = (side >= 0) & (side < nn)
        np.add.at(slack, side[ok], np.asarray(w, np.float64)[amb][ok])
    alpha = (np.arange(nn) + 0.5) * da
    return slack / (4 * np.pi * np.sin(alpha) * np.sin(da / 2) * n)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_angle_resolved_matches_host_scoring(cuda, precision):
    m = _model(precision=precision).start(rand_seed=9)
    res = m.get_result()
    v, w, n = res["v"], res["w"], res["nPh"]
    for getter, sel in ((m.get_Ra, v[2] < 0), (m.get_Ta, v[2] > 0)):
        a_dev, dev = getter()
        a_host, host = metrics.angularyResolved(v[:, sel], w[sel], m.n_ang, n)
        np.testing.assert_allclose(a_dev, a_host, rtol=0, atol=1e-12)
        assert host.sum() > 0
        slack = _edge_slack(v[:, sel], w[sel], m.n_ang, n)
        assert np.all(np.abs(dev - host) <= 1e-4 * np.abs(host) + slack + 1e-9 * host.max()), \
            (np.abs(dev - host), slack)
        # only a handful of exits lie that close to an edge
        assert slack.sum() < 1e-3 * host.sum()


def test_line_profile_matches_host_scoring(cuda):
    m = _model().start(rand_seed=10)
    res = m.get_result()
    p, v, w, n = res["p"], res["v"], res["w"], res["nPh"]
    sel = v[0] < 0
    a_dev, dev = m.get_line_profile()
    a_host, host = metrics.lineDistance(p[:, sel], w[sel], m.n_line, m.line_dr, n,
                                        y_range=m.line_y_range)
    np.testing.assert_allclose(a_dev, a_host, rtol=0, atol=1e-12)
    assert host.sum() > 0 and np.count_nonzero(host) > 20
    # exit depths are encoded in single precision on the device and in
    # double on the host: a photon within 1e-6 mm of a bin edge may change bin
    np.testing.assert_allclose(dev, host, rtol=2e-3, atol=2e-3 * host.max())
    assert abs(dev.sum() - host.sum()) <= 1e-3 * host.sum()


def test_exit_tallies_off_by_default(cuda):
    m = VoxelPlateModel(nPh=1000, verbose=False)
    m.build(x_size=1.0, y_size=1.0, voxel_space=0.1, thickness=[1.0], n=[1.4], n_air=1.0,
            ma=[0.1], ms=[5.0], g=[0.9])
    m.start(rand_seed=1)
    with pytest.raises(RuntimeError):
        m.get_Ra()
    with pytest.raises(RuntimeError):
        m.get_line_profile()


def test_save_result_writes_reference_format(cuda):
    """save_result (pymopt/voxel_gpu/_classes.py:338-382): a bz2 pickle of
    get_result() and an _info.json with the reference's keys."""
    import bz2
    import json
    import os
    import pickle
    import tempfile
    m = VoxelPlateModel(nPh=5000, keep_exits=True, verbose=False)
    m.build(x_size=1.0, y_size=1.0, voxel_space=0.1, thickness=[1.0], n=[1.4], n_air=1.0,
            ma=[0.1], ms=[5.0], g=[0.9])
    m.start(rand_seed=2)
    res = m.get_result()
    with tempfile.TemporaryDirectory(dir=os.path.dirname(os.path.abspath(__file__))) as d:
        base = os.path.join(d, "run")
        m.save_result(base, coment="check")
        with bz2.open(base + "_LID.pkl.bz2", "rb") as fp:
            back = pickle.loads(fp.read())
        with open(base + "_info.json") as fp:
            info = json.load(fp)
    assert set(back) == {"p", "v", "w", "nPh"} and back["nPh"] == 5000
    for k in ("p", "v", "w"):
        np.testing.assert_array_equal(back[k], res[k])
    assert set(info) == {"Date", "coment", "number_of_photons", "calc_dtype", "model", "w_beam",
                         "beam_angle", "initial_refrect_mode", "beam_mode", "fluence_mode"}
    assert set(info["model"]) == {"model_name", "model_params", "model_voxel_space",
                                  "model_xy_size"}
    assert info["coment"] == "check" and info["number_of_photons"] == 5000
    assert info["calc_dtype"] == "32 bit" and info["model"]["model_name"] == "PlateModel"
