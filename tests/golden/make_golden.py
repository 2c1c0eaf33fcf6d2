"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own CPU transport path — ``pymopt.voxel`` (Numba
``vmc_kernel``, pymopt/voxel/_kernel.py:23-172, driven by
``VoxelPlateModel.build/start/get_result``, pymopt/voxel/_classes.py) — from a
checkout of pyMonteOpt, seeded through a jitted ``np.random.seed``, and stores
per-seed Rd / Tt and R(r) / T(r) (``metrics.radialDistance`` on exits with
v_z < 0 and v_z > 0, as the reference notebooks do) as JSON.

Usage::

    python tests/golden/make_golden.py /path/to/pyMonteOpt [case ...]

The reference imports pydicom, matplotlib and seaborn at module level although
the transport path never calls them; they are stubbed with empty modules.
The fixtures are committed; nothing at test time needs the reference.
"""
from __future__ import annotations

import contextlib
import io
import json
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _stub_modules():
    for name in ("pydicom", "matplotlib", "matplotlib.pyplot", "matplotlib.colors",
                 "seaborn"):
        if name not in sys.modules:
            m = types.ModuleType(name)
            sys.modules[name] = m
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.modules["matplotlib"].colors = sys.modules["matplotlib.colors"]
    sys.modules["matplotlib.colors"].LogNorm = object


# Plate cases: name -> (params, nPh, seeds, nr, dr).  'c1' is the C1 workload;
# the others are the notebook cases of the reference (test_voxelcuda.ipynb
# cells 5, 9, 23; test_voxcelplate.ipynb cells 6, 9) at CPU-sized counts.
PLATE_CASES = {
    "c1": (dict(x_size=10.1, y_size=10.1, voxel_space=0.1, thickness=[10.0], n=[1.37],
                n_air=1.0, ma=[0.1], ms=[10.0], g=[0.9]), 20000, 10, 100, 0.1),
    "thin_slab": (dict(x_size=5, y_size=5, voxel_space=0.01, thickness=[0.02], n=[1.0],
                       n_air=1.0, ma=[10.0], ms=[90.0], g=[0.75]), 20000, 10, 50, 0.05),
    "semi_inf_mismatch": (dict(x_size=10, y_size=10, voxel_space=0.1, thickness=[10.0],
                               n=[1.5], n_air=1.0, ma=[10.0], ms=[90.0], g=[0.0]),
                          20000, 10, 50, 0.02),
    "three_layer": (dict(x_size=10, y_size=10, voxel_space=0.1, thickness=[0.1, 0.1, 0.2],
                         n=[1.37, 1.37, 1.37], n_air=1.0, ma=[1.0, 1.0, 2.0],
                         ms=[100.0, 10.0, 10.0], g=[0.9, 0.0, 0.7]), 20000, 10, 100, 0.05),
    "c2_pencil": (dict(x_size=20.0, y_size=20.0, voxel_space=0.05, thickness=[0.1, 2.0, 17.9],
                       n=[1.4, 1.4, 1.44], n_air=1.0, ma=[0.5, 0.05, 0.01],
                       ms=[20.0, 15.0, 10.0], g=[0.8, 0.85, 0.9]), 2000, 10, 100, 0.2),
}


def _radial(p, w, nn, dr, nph, metrics):
    _, r = metrics.radialDistance(p, w, nn, dr, nph)
    return r


def run_plate_case(ref_root: str, name: str) -> dict:
    _stub_modules()
    sys.path.insert(0, ref_root)
    from numba import njit
    from pymopt import metrics
    from pymopt.voxel import VoxelPlateModel

    @njit
    def _seed(s):
        np.random.seed(s)

    params, nph, seeds, nr, dr = PLATE_CASES[name]
    out = {"case": name, "params": params, "nPh": nph, "seeds": list(range(seeds)),
           "nr": nr, "dr": dr, "Rd": [], "Tt": [], "Rr": [], "Tr": [], "seconds": []}
    for s in range(seeds):
        model = VoxelPlateModel(nPh=nph)
        with contextlib.redirect_stdout(io.StringIO()):
            model.build(**params)
            _seed(s)
            t0 = time.time()
            model.start()
            out["seconds"].append(time.time() - t0)
        res = model.get_result()
        v, w, p = res["v"], res["w"], res["p"]
        rd = v[2] < 0
        tt = v[2] > 0
        out["Rd"].append(float(w[rd].sum() / nph))
        out["Tt"].append(float(w[tt].sum() / nph))
        out["Rr"].append(_radial(p[:, rd], w[rd], nr, dr, nph, metrics).tolist())
        out["Tr"].append(_radial(p[:, tt], w[tt], nr, dr, nph, metrics).tolist())
    return out


def run_c3_case(ref_root: str, nph: int = 2000, seeds: int = 10, nr: int = 100,
                dr: float = 0.2) -> dict:
    """C3 through the reference kernel directly: there is no reference model
    class for a raw label volume, so ``vmc_kernel`` is called on the padded
    volume with the state the reference's start() would build
    (pymopt/voxel/_classes.py:63-81)."""
    _stub_modules()
    sys.path.insert(0, ref_root)
    sys.path.insert(0, REPO)
    from numba import njit
    from pymopt import metrics
    from pymopt.voxel import vmc_kernel
    from pymonteopt_b200.volumes import c3_ct_like

    @njit
    def _seed(s):
        np.random.seed(s)

    prob = c3_ct_like(0)
    vol = prob.labels.astype(np.int8)
    end = prob.end_label
    cx, cy = prob.center
    out = {"case": "c3", "volume_seed": 0, "nPh": nph, "seeds": [], "failed_seeds": [],
           "nr": nr, "dr": dr, "Rd": [], "Tt": [], "Rr": [], "Tr": [], "seconds": []}
    l = prob.voxel_space
    s = -1
    while len(out["seeds"]) < seeds:
        s += 1
        add = np.zeros((3, nph), np.int32)
        add[0], add[1], add[2] = cx, cy, 1
        p = np.zeros((3, nph), np.float32)
        p[2] = -l / 2
        v = np.zeros((3, nph), np.float32)
        v[2] = 1
        w = np.full(nph, prob.src_w0, np.float32)
        _seed(s)
        t0 = time.time()
        try:
            with contextlib.redirect_stdout(io.StringIO()):
                add, p, v, w = vmc_kernel(add, p, v, w, prob.ma[:end].copy(),
                                          prob.ms[:end].copy(), prob.n.copy(),
                                          prob.g[:end].copy(), vol, l, np.int32(nph),
                                          np.int8(end))
        except ZeroDivisionError:
            # the reference kernel divides by zero on some histories of this
            # heterogeneous volume (Numba's Python error model raises); such
            # seeds are recorded and skipped
            out["failed_seeds"].append(s)
            continue
        out["seeds"].append(s)
        out["seconds"].append(time.time() - t0)
        enc = p.astype(np.float64).copy()
        enc[0] = l * (add[0] - cx) + p[0]
        enc[1] = l * (add[1] - cy) + p[1]
        rd, tt = v[2] < 0, v[2] > 0
        out["Rd"].append(float(w[rd].sum() / nph))
        out["Tt"].append(float(w[tt].sum() / nph))
        out["Rr"].append(_radial(enc[:, rd], w[rd], nr, dr, nph, metrics).tolist())
        out["Tr"].append(_radial(enc[:, tt], w[tt], nr, dr, nph, metrics).tolist())
    return out


def main():
    ref_root = sys.argv[1]
    cases = sys.argv[2:] or list(PLATE_CASES) + ["c3"]
    for name in cases:
        t0 = time.time()
        res = run_c3_case(ref_root) if name == "c3" else run_plate_case(ref_root, name)
        res["generator"] = "tests/golden/make_golden.py (reference pymopt.voxel, Numba)"
        path = os.path.join(HERE, f"ref_{name}.json")
        with open(path, "w") as f:
            json.dump(res, f, indent=0)
        print(f"{name}: Rd {np.mean(res['Rd']):.6f} +- {np.std(res['Rd'])/np.sqrt(len(res['Rd'])):.6f}"
              f"  Tt {np.mean(res['Tt']):.6f}  ({time.time()-t0:.1f} s) -> {path}")


if __name__ == "__main__":
    main()
