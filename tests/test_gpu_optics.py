"""The optical bench (OBD, SideOBD) against the reference's own NumPy bench.

``tests/golden/ref_obd.json`` holds what pymopt.optics computes on 50000
seeded synthetic exit photons (``tests/golden/make_golden.py``):
- with every Fresnel draw fixed at 0.5, so that a photon passes a surface
  when R < 0.5 (deterministic);
- over ten seeds of NumPy's generator.

The GPU bench must match the deterministic scan photon for photon and the
random one within 3 sigma.
"""
import json
import os
import sys

import numpy as np
import pytest
from scipy import stats

from helpers import GOLDEN, mean_se, z_score
from pymonteopt_b200 import optics as O

REF = json.load(open(os.path.join(GOLDEN, "ref_obd.json")))
sys.path.insert(0, GOLDEN)
from make_golden import obd_photons  # noqa: E402


def _bench(name, seed=0, fixed_u=None):
    cls = O.SideOBD if name == "side" else O.OBD
    m = cls(seed=seed, fixed_u=fixed_u)
    if name == "obd_no_ld":
        m.set_params(ld_fix_part=False)
    p, v, w = obd_photons()
    m.set_monte_data(p=p, v=v, w=w, nPh=int(w.size))
    return m


def test_grass_indices_match_reference():
    m = O.OBD(seed=0)
    assert m.params["n_1"] == pytest.approx(REF["obd"]["params"]["n_1"], rel=1e-15)
    assert m.params["n_2"] == pytest.approx(REF["obd"]["params"]["n_2"], rel=1e-15)
    for k, v in REF["obd"]["params"].items():
        assert m.params[k] == v, k
    with pytest.raises(KeyError):
        m.set_params(lens=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["obd", "obd_no_ld", "side"])
def test_fixed_draws_match_reference_scan(cuda, name):
    m = _bench(name, fixed_u=0.5)
    z, inten = m.opticalAnalysisMeth()
    ref = np.array(REF[name]["fixed"])
    np.testing.assert_allclose(z, REF[name]["z"], rtol=0, atol=0)
    assert ref.max() > 10
    # photon for photon: the same photons reach the photodiode; the reference
    # sums their float32 weights in float32, hence the 1e-6 (measured 2e-7)
    np.testing.assert_allclose(inten, ref, rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["obd", "side"])
def test_random_draws_match_reference_statistically(cuda, name):
    mine = np.array([_bench(name, seed=s).opticalAnalysisMeth()[1] for s in range(10)])
    ref = np.array(REF[name]["seeds"])
    m, s = mean_se(mine)
    rm, rs = mean_se(ref)
    keep = (rm > 0) & (rs > 0) & (s > 0)
    z = z_score(m[keep], s[keep], rm[keep], rs[keep])
    assert keep.sum() > 50
    assert stats.chi2.sf(float(np.sum(z ** 2)), int(keep.sum())) > 1e-3, np.round(z, 2)
    assert np.max(np.abs(z)) < 4.5


@pytest.mark.gpu
def test_start_and_save_result(cuda):
    import tempfile
    m = _bench("obd", seed=3)
    m.start()
    res = m.get_result()
    assert list(res.columns) == ["Z", "int", "log(int)"] and len(res) == len(REF["obd"]["z"])
    with tempfile.TemporaryDirectory(dir=os.path.dirname(os.path.abspath(__file__))) as d:
        m.save_result(os.path.join(d, "scan"))
        assert os.path.exists(os.path.join(d, "scan_opt.csv"))
