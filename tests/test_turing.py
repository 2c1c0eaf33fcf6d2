"""Turing-pattern generator against the reference's own generator.

``tests/golden/ref_turing.npz`` holds, for a seeded 24^3 grid, what the
reference's TuringPattern computes (pymopt/modeling/_classes.py, generated by
``tests/golden/make_golden.py``): the initial activator, the field after one
and after all steps, the threshold, the microarchitecture and the binarised,
tiled volume.  The generator runs here on the CPU through torch (the same
code as on the GPU) and, in the GPU suite, on CUDA.
"""
import json
import os
import tempfile

import numpy as np
import pytest
import torch

from helpers import GOLDEN
from pymonteopt_b200.turing import TuringPattern, _relmax_count

REF = np.load(os.path.join(GOLDEN, "ref_turing.npz"))
PARAMS = json.loads(str(REF["params_json"]))


def _check(device):
    tp = TuringPattern(device=device)
    tp.set_params(**PARAMS)
    tp._calc_kukv()
    u, v = tp._get_inital_vector()
    np.testing.assert_array_equal(u.cpu().numpy(), REF["u0"])
    u1, v1 = tp._calc_onestep(u, v)
    np.testing.assert_allclose(u1.cpu().numpy(), REF["u1"], rtol=1e-5, atol=1e-5)
    for _ in range(tp.repetition - 1):
        u1, v1 = tp._calc_onestep(u1, v1)
    # float32 FFTs of two libraries: differences stay at rounding level
    np.testing.assert_allclose(u1.cpu().numpy(), REF["u_final"], rtol=1e-4, atol=1e-4)

    tp2 = TuringPattern(device=device)
    tp2.set_params(**PARAMS)
    with tempfile.TemporaryDirectory(dir=os.path.dirname(os.path.abspath(__file__))) as d:
        vol = tp2.modeling(d)
        with open(os.path.join(d, "_info.json")) as f:
            info = json.load(f)
    assert tp2.threshold == pytest.approx(float(REF["threshold"]), rel=1e-12)
    assert vol.dtype == np.int8 and vol.shape == REF["volume"].shape
    # voxels whose field sits within rounding of the threshold may flip
    assert np.mean(vol == REF["volume"]) > 0.999
    micro = dict(zip([str(k) for k in REF["micro_keys"]], REF["micro_values"]))
    assert set(info["microarchitecture"]) == set(micro)
    for k, want in micro.items():
        assert info["microarchitecture"][k] == pytest.approx(want, rel=2e-3), k
    assert info["model_shape"] == [tp2.gridsize] * 3
    assert set(info) == {"Date", "coment", "model_params", "microarchitecture", "model_shape"}


def test_turing_generator_matches_reference_cpu():
    _check("cpu")


@pytest.mark.gpu
def test_turing_generator_matches_reference_gpu(cuda):
    _check(cuda)


def test_relmax_matches_scipy():
    from scipy.signal import argrelmax
    rng = np.random.default_rng(2)
    a = rng.normal(size=(5, 7, 40)).astype(np.float32)
    a[0, 0, :] = 1.0                    # plateau: no strict maxima
    a[1, 1, -1] = 10.0                  # end point: never a maximum under clip
    got = _relmax_count(torch.from_numpy(a)).numpy()
    want = np.array([[argrelmax(a[i, j], order=5)[0].shape[0] for j in range(7)]
                     for i in range(5)])
    np.testing.assert_array_equal(got, want)


def test_unknown_param_raises():
    tp = TuringPattern(device="cpu")
    with pytest.raises(KeyError):
        tp.set_params(gird=10)
