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
The "turing" case runs the reference's CPU Turing-pattern generator
(pymopt/modeling/_classes.py) on a small grid; the "obd" case runs its OBD
ray tracing (pymopt/optics/_classes.py) on seeded synthetic exit photons.
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
    sys.modules["seaborn"].set_style = lambda *a, **k: None
    for sub in ("pydicom.uid", "pydicom.dataset"):
        sys.modules.setdefault(sub, types.ModuleType(sub))
    sys.modules["pydicom.uid"].ImplicitVRLittleEndian = None
    sys.modules["pydicom.dataset"].Dataset = sys.modules["pydicom.dataset"].FileDataset = object


# Plate cases: name -> (params, photons per seed, seeds, nr, dr[, model kwargs[,
# model class[, chunks per seed]]]).  'c1' is the C1 workload; 'c2_pencil' /
# 'c2_gaussian' the C2 skin slab with a pencil and with the 1 mm 1/e^2
# Gaussian beam the benchmark runs; the notebook cases of the reference
# (test_voxelcuda.ipynb cells 5, 9, 23; test_voxcelplate.ipynb cells 6, 9) at
# CPU-sized counts; and the source options of BaseVoxelMonteCarlo
# (pymopt/voxel/_classes.py:111-203): an oblique beam and first_layer_clear on
# the glass-covered VoxelPlateExModel.  The oblique beam with its specular part
# as photons (initial_refrect_by_angle) is not run: the reference deletes those
# photons from its state arrays but still passes the original nPh to the
# kernel (pymopt/voxel/_classes.py:133-146 with :75-80), which then reads and
# writes past the arrays' ends (glibc aborted with heap corruption here).  Its
# expected results follow from the "oblique" case: the specular photons add
# their fraction to Rd and fall in no R(r) bin (they are recorded at r = 0).
#
# A seed's photons run as `chunks` reference runs of photons/chunks each, with
# the generators seeded per run.  The cases below keep one run per seed and
# many seeds, so that a fixture's standard error comes from 40-160 samples
# (with 10, z-scores follow a t distribution and a chi-square over 50-100
# bins is too easily exceeded).  The reference kernel raises
# ZeroDivisionError on rare histories (its theta() lets cos(theta) round above
# 1, the direction turns NaN, and Numba's fastmath zero-divisor check trips on
# the renormalisation, pymopt/voxel/_kernel.py:12-21, :165); a run that raises
# is recorded in "failed_runs" and replaced by the next run seed.
C2 = dict(x_size=20.0, y_size=20.0, voxel_space=0.05, thickness=[0.1, 2.0, 17.9],
          n=[1.4, 1.4, 1.44], n_air=1.0, ma=[0.5, 0.05, 0.01], ms=[20.0, 15.0, 10.0],
          g=[0.8, 0.85, 0.9])
OBLIQUE = dict(x_size=10.0, y_size=10.0, voxel_space=0.1, thickness=[2.0], n=[1.4],
               n_air=1.0, ma=[0.1], ms=[10.0], g=[0.8])
PLATE_CASES = {
    "c1": (dict(x_size=10.1, y_size=10.1, voxel_space=0.1, thickness=[10.0], n=[1.37],
                n_air=1.0, ma=[0.1], ms=[10.0], g=[0.9]), 5000, 40, 100, 0.1),
    "thin_slab": (dict(x_size=5, y_size=5, voxel_space=0.01, thickness=[0.02], n=[1.0],
                       n_air=1.0, ma=[10.0], ms=[90.0], g=[0.75]), 5000, 40, 50, 0.05),
    "semi_inf_mismatch": (dict(x_size=10, y_size=10, voxel_space=0.1, thickness=[10.0],
                               n=[1.5], n_air=1.0, ma=[10.0], ms=[90.0], g=[0.0]),
                          5000, 40, 50, 0.02),
    "three_layer": (dict(x_size=10, y_size=10, voxel_space=0.1, thickness=[0.1, 0.1, 0.2],
                         n=[1.37, 1.37, 1.37], n_air=1.0, ma=[1.0, 1.0, 2.0],
                         ms=[100.0, 10.0, 10.0], g=[0.9, 0.0, 0.7]), 5000, 40, 100, 0.05),
    "c2_pencil": (C2, 5000, 40, 100, 0.2, {}, "VoxelPlateModel", 1),
    "c2_gaussian": (C2, 10000, 160, 100, 0.1, {"w_beam": 1.0}, "VoxelPlateModel", 1),
    "oblique": (OBLIQUE, 2500, 80, 50, 0.1, {"beam_angle": 0.5}, "VoxelPlateModel", 1),
    "ex_first_layer": (dict(x_size=8.0, y_size=8.0, voxel_space=0.1, thickness=[0.5, 3.0],
                            n=[1.5, 1.33], n_air=1.0, ma=[1e-5, 0.05], ms=[1e-5, 5.0],
                            g=[0.9, 0.8]), 5000, 40, 50, 0.1, {}, "VoxelPlateExModel", 1),
}


def run_plate_case(ref_root: str, name: str) -> dict:
    """Per-seed Rd / Tt / R(r) / T(r) of the reference's own model class
    (oracle/ref_cpu.py runs it on spawned processes)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref_cpu
    case = PLATE_CASES[name]
    params, nph, seeds, nr, dr = case[:5]
    model_kwargs = case[5] if len(case) > 5 else {}
    model_class = case[6] if len(case) > 6 else "VoxelPlateModel"
    chunks = case[7] if len(case) > 7 else 1
    per_run = nph // chunks
    need = seeds * chunks
    done, failed, nxt = [], [], 0
    while len(done) < need:
        batch = list(range(nxt, nxt + need - len(done)))
        nxt = batch[-1] + 1
        runs = ref_cpu.run_plate_seeds(params, per_run, batch, model_kwargs, nr, dr,
                                       path=ref_root, model_class=model_class)
        for s, r in zip(batch, runs):
            (failed.append(s) if r is None else done.append(r))
    out = {"case": name, "params": params, "nPh": per_run * chunks, "seeds": list(range(seeds)),
           "model_class": model_class, "model_kwargs": model_kwargs, "runs_per_seed": chunks,
           "run_seeds": [], "failed_runs": failed,
           "nr": nr, "dr": dr, "Rd": [], "Tt": [], "Rr": [], "Tr": [], "seconds": []}
    for i in range(seeds):
        part = done[i * chunks:(i + 1) * chunks]
        out["run_seeds"].append([r["seed"] for r in part])
        out["seconds"].append(sum(r["seconds"] for r in part))
        for k in ("Rd", "Tt"):
            out[k].append(float(np.mean([r[k] for r in part])))
        for k in ("Rr", "Tr"):
            out[k].append(np.mean([r[k] for r in part], axis=0).tolist())
    return out


def _c3_chunk(args):
    """One chunk of C3 photons through the reference's ``vmc_kernel`` with
    Numba's generator seeded by ``chunk``; None when the kernel raises."""
    ref_root, chunk, nph, nr, dr = args
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, REPO)
    import ref_cpu
    from pymonteopt_b200.volumes import c3_ct_like
    ref_cpu.stub_modules()
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    from pymopt import metrics
    from pymopt.voxel import vmc_kernel
    prob = c3_ct_like(0)
    vol = prob.labels.astype(np.int8)
    end = prob.end_label
    cx, cy = prob.center
    l = prob.voxel_space
    add = np.zeros((3, nph), np.int32)
    add[0], add[1], add[2] = cx, cy, 1
    p = np.zeros((3, nph), np.float32)
    p[2] = -l / 2
    v = np.zeros((3, nph), np.float32)
    v[2] = 1
    w = np.full(nph, prob.src_w0, np.float32)
    ref_cpu.seed_all(chunk)
    t0 = time.time()
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            add, p, v, w = vmc_kernel(add, p, v, w, prob.ma[:end].copy(), prob.ms[:end].copy(),
                                      prob.n.copy(), prob.g[:end].copy(), vol, l,
                                      np.int32(nph), np.int8(end))
    except ZeroDivisionError:
        return None
    dt = time.time() - t0
    enc = p.astype(np.float64).copy()
    enc[0] = l * (add[0] - cx) + p[0]
    enc[1] = l * (add[1] - cy) + p[1]
    rd, tt = v[2] < 0, v[2] > 0
    return {"chunk": chunk, "seconds": dt, "w_rd": float(w[rd].sum()), "w_tt": float(w[tt].sum()),
            "rr": metrics.radialDistance(enc[:, rd], w[rd], nr, dr, nph)[1] * nph,
            "tr": metrics.radialDistance(enc[:, tt], w[tt], nr, dr, nph)[1] * nph}


def run_c3_case(ref_root: str, nph: int = 2000, chunks_per_seed: int = 1, seeds: int = 100,
                nr: int = 100, dr: float = 0.2) -> dict:
    """C3 through the reference kernel directly: there is no reference model
    class for a raw label volume, so ``vmc_kernel`` is called on the padded
    volume with the state the reference's start() would build
    (pymopt/voxel/_classes.py:63-81).

    The reference kernel raises ZeroDivisionError on rare histories of this
    volume (Numba's Python error model), so photons run in chunks of ``nph``
    with Numba's generator seeded per chunk; a chunk that raises is recorded
    and skipped, and each fixture seed is the sum of ``chunks_per_seed``
    chunks that completed."""
    import multiprocessing as mp
    need = chunks_per_seed * seeds
    done, failed, nxt = [], [], 0
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        while len(done) < need:
            batch = list(range(nxt, nxt + (need - len(done)) + 4))
            nxt = batch[-1] + 1
            for c, r in zip(batch, pool.map(_c3_chunk, [(ref_root, c, nph, nr, dr) for c in batch])):
                (failed.append(c) if r is None else done.append(r))
    done = sorted(done, key=lambda r: r["chunk"])[:need]
    n_seed = nph * chunks_per_seed
    out = {"case": "c3", "volume_seed": 0, "nPh": n_seed, "chunk_photons": nph,
           "seeds": [], "chunks": [], "failed_chunks": failed,
           "nr": nr, "dr": dr, "Rd": [], "Tt": [], "Rr": [], "Tr": [], "seconds": []}
    for i in range(seeds):
        part = done[i * chunks_per_seed:(i + 1) * chunks_per_seed]
        out["seeds"].append(i)
        out["chunks"].append([r["chunk"] for r in part])
        out["seconds"].append(sum(r["seconds"] for r in part))
        out["Rd"].append(sum(r["w_rd"] for r in part) / n_seed)
        out["Tt"].append(sum(r["w_tt"] for r in part) / n_seed)
        out["Rr"].append((sum(r["rr"] for r in part) / n_seed).tolist())
        out["Tr"].append((sum(r["tr"] for r in part) / n_seed).tolist())
    return out


TURING_PARAMS = {"voxel_space": 0.1, "th_cortical": 1.0, "th_subcutaneus": 1.2, "th_dermis": 0.8}


def bone_volume(seed: int = 0, shape=(60, 40, 60)) -> np.ndarray:
    """Seeded binary stand-in for a Turing-pattern bone volume."""
    rng = np.random.default_rng(seed)
    return (rng.random(shape) < 0.3).astype(np.int8)


def run_volumes_case(ref_root: str) -> str:
    """Volumes built by the reference's own model classes (PlateModel,
    PlateExModel, TuringModel_*; pymopt/voxel/_classes.py:343-782, identical
    to pymopt/voxel_gpu/_classes.py:387-821), saved as an npz."""
    _stub_modules()
    sys.path.insert(0, ref_root)
    if not hasattr(np, "int"):
        np.int = int  # the reference's Turing models use the removed alias
    from pymopt.voxel import _classes as RC
    # pymopt/voxel/_classes.py calls tqdm without importing it
    RC.tqdm = getattr(RC, "tqdm", lambda it: it)
    out = {}
    with contextlib.redirect_stdout(io.StringIO()):
        m = RC.PlateModel()
        m.set_params(x_size=2.1, y_size=1.6, voxel_space=0.1, thickness=[0.3, 0.5, 0.2],
                     n=[1.4, 1.37, 1.45], n_air=1.0, ma=[0.1, 0.2, 0.3], ms=[10, 20, 30],
                     g=[0.9, 0.8, 0.7])
        m.build()
        out["plate"] = m.voxel_model
        m = RC.PlateExModel()
        m.set_params(x_size=2.0, y_size=1.5, voxel_space=0.1, thickness=[0.3, 1.0],
                     n=[1.5, 1.4], n_air=1.0, ma=[1e-5, 0.02], ms=[1e-5, 1.0], g=[0.9, 0.9])
        m.build()
        out["plate_ex"] = m.voxel_model
        u = bone_volume()
        out["bone"] = u
        for name, extra in (("TuringModel_Rectangular", {"xz_size": 6.0}),
                            ("TuringModel_Cylinder", {"r_bone": 3.5}),
                            ("TuringModel_RnC", {"xz_size": 6.0, "r_bone": 3.5})):
            m = getattr(RC, name)()
            m.set_params(**TURING_PARAMS, **extra)
            m.build(u.copy())
            out[name] = m.voxel_model
    path = os.path.join(HERE, "ref_volumes.npz")
    np.savez_compressed(path, **out)
    return path


def run_sources_case(ref_root: str) -> str:
    """Initial photon state the reference builds on the host
    (_generate_initial_coodinate, pymopt/voxel/_classes.py:102-203) for the
    beam options that do not draw random numbers, and the specular fraction
    of initial_refrect_by_angle."""
    _stub_modules()
    sys.path.insert(0, ref_root)
    from pymopt.voxel import _classes as RC
    cases = []
    base = dict(x_size=2.1, y_size=2.1, voxel_space=0.1, thickness=[0.5, 1.0],
                n=[1.4, 1.5], n_air=1.0, ma=[0.1, 0.2], ms=[10, 20], g=[0.9, 0.8])
    with contextlib.redirect_stdout(io.StringIO()):
        for name, cls, kw in (
                ("default", RC.VoxelPlateModel, {}),
                ("angle", RC.VoxelPlateModel, {"beam_angle": 0.3}),
                ("angle_refrect", RC.VoxelPlateModel,
                 {"beam_angle": 0.3, "initial_refrect_by_angle": True}),
                ("first_layer_clear", RC.VoxelPlateModel, {"first_layer_clear": True})):
            m = cls(nPh=20000, **kw)
            m.build(**base)
            if name == "first_layer_clear":
                m.model.get_second_layer_addz = lambda: 6
            np.random.seed(0)
            m._reset_results()
            m._generate_initial_coodinate(m.nPh)
            rec = {"name": name, "kwargs": kw, "params": base,
                   "add": m.add[:, -1].tolist(), "p": m.p[:, -1].astype(float).tolist(),
                   "v": m.v[:, -1].astype(float).tolist(), "w": float(m.w[-1]),
                   "n_transported": int(m.w.size)}
            if name == "angle_refrect":
                rec["spec_fraction"] = float(m.inital_del_num / m.nPh)
                rec["spec_v"] = m.v_result[:, -1].astype(float).tolist()
            cases.append(rec)
    path = os.path.join(HERE, "ref_sources.json")
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)
    return path


# Turing-pattern generator case: small grid, few steps, seeded
TURING_GEN = dict(grid=8, dx=1 / 8, dt=1, du=0.0002, dv=0.01, length=3, repetition=12,
                  bv_tv=0.138, voxelsize=0.0295, seed=3, ct_coef=4.5e4, tile_num_xz=1,
                  tile_num_y=2)


def run_turing_case(ref_root: str) -> str:
    """The reference's CPU Turing-pattern generator (pymopt/modeling/_classes.py,
    the scipy.fftpack twin of pymopt/modeling_gpu/_classes.py) on a 24^3 grid:
    the field after the reaction-diffusion steps, the thresholded
    microarchitecture and the binarised, tiled volume."""
    import tempfile
    _stub_modules()
    sys.path.insert(0, ref_root)
    from pymopt.modeling import _classes as MC
    MC.tqdm = lambda it: it
    tp = MC.TuringPattern()
    tp.set_params(**TURING_GEN)
    with contextlib.redirect_stdout(io.StringIO()):
        tp._calc_kukv()
        u, v = tp._get_inital_vector()
        fields = {"u0": u.copy(), "v0": v.copy()}
        for i in range(tp.repetition):
            u, v = tp._calc_onestep(u, v)
            if i == 0:
                fields["u1"] = u.copy()
        fields["u_final"] = u.copy()
        tp2 = MC.TuringPattern()
        tp2.set_params(**TURING_GEN)
        with tempfile.TemporaryDirectory(dir=HERE) as d:
            vol = tp2.modeling(d)
            with open(os.path.join(d, "_info.json")) as f:
                info = json.load(f)
    path = os.path.join(HERE, "ref_turing.npz")
    micro = info["microarchitecture"]
    fields.pop("v0")
    np.savez_compressed(path, volume=vol, threshold=np.float64(tp2.threshold),
                        micro_keys=np.array(list(micro.keys())),
                        micro_values=np.array([float(x) for x in micro.values()]),
                        params_json=np.array(json.dumps(TURING_GEN)), **fields)
    return path


def obd_photons(seed: int = 0, n: int = 50000):
    """Seeded synthetic exit photons for the OBD stage: positions N(0, 1 mm)
    in x and y, Lambertian directions leaving through the top (v_z < 0),
    weights U[0.5, 1], plus 10 % going the other way; float32 like
    get_result()."""
    rng = np.random.default_rng(seed)
    p = np.zeros((3, n), np.float32)
    p[0], p[1] = rng.normal(0, 1.0, n), rng.normal(0, 1.0, n)
    cos_t = np.sqrt(rng.random(n))
    phi = 2 * np.pi * rng.random(n)
    sin_t = np.sqrt(1 - cos_t ** 2)
    v = np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), -cos_t]).astype(np.float32)
    v[2, rng.random(n) < 0.1] *= -1
    w = rng.uniform(0.5, 1.0, n).astype(np.float32)
    return p, v, w


def run_obd_case(ref_root: str) -> str:
    """The reference's OBD ray tracing (pymopt/optics/_classes.py:381-566) on
    seeded synthetic exit photons: OBD (with and without the LD fixing part)
    and SideOBD, once with np.random.rand replaced by a constant 0.5 (every
    Fresnel decision becomes R < 0.5, deterministic) and over ten seeds of
    the real generator."""
    _stub_modules()
    sys.path.insert(0, ref_root)
    from pymopt.optics import _classes as OC
    OC.tqdm = lambda it: it
    OC.calTime = lambda *a, **k: None
    p, v, w = obd_photons()
    out = {"n": int(w.size)}
    real_rand = np.random.rand
    with contextlib.redirect_stdout(io.StringIO()):
        for name, cls, extra in (("obd", OC.OBD, {}),
                                 ("obd_no_ld", OC.OBD, {"ld_fix_part": False}),
                                 ("side", OC.SideOBD, {})):
            runs = []
            for mode in ["fixed"] + list(range(10)):
                m = cls()
                if extra:
                    m.set_params(**extra)
                m.set_monte_data(p=p.copy(), v=v.copy(), w=w.copy(), nPh=int(w.size))
                if mode == "fixed":
                    np.random.rand = lambda k: np.full(k, 0.5)
                else:
                    np.random.rand = real_rand
                    np.random.seed(100 + mode)
                try:
                    z, inten = m.opticalAnalysisMeth()
                finally:
                    np.random.rand = real_rand
                runs.append(inten)
            out[name] = {"z": np.asarray(z).tolist(), "fixed": np.asarray(runs[0]).tolist(),
                         "seeds": [np.asarray(r).tolist() for r in runs[1:]],
                         "params": {k: (v_ if not isinstance(v_, np.generic) else v_.item())
                                    for k, v_ in m.params.items()}}
    out["generator"] = "tests/golden/make_golden.py (reference pymopt.optics, NumPy)"
    path = os.path.join(HERE, "ref_obd.json")
    with open(path, "w") as f:
        json.dump(out, f)
    return path


def main():
    ref_root = sys.argv[1]
    cases = sys.argv[2:] or list(PLATE_CASES) + ["c3", "volumes", "sources", "turing", "obd"]
    for name in cases:
        t0 = time.time()
        if name == "turing":
            print("turing ->", run_turing_case(ref_root))
            continue
        if name == "obd":
            print("obd ->", run_obd_case(ref_root))
            continue
        if name == "volumes":
            print("volumes ->", run_volumes_case(ref_root))
            continue
        if name == "sources":
            print("sources ->", run_sources_case(ref_root))
            continue
        res = run_c3_case(ref_root) if name == "c3" else run_plate_case(ref_root, name)
        res["generator"] = "tests/golden/make_golden.py (reference pymopt.voxel, Numba)"
        path = os.path.join(HERE, f"ref_{name}.json")
        with open(path, "w") as f:
            json.dump(res, f, indent=0)
        print(f"{name}: Rd {np.mean(res['Rd']):.6f} +- {np.std(res['Rd'])/np.sqrt(len(res['Rd'])):.6f}"
              f"  Tt {np.mean(res['Tt']):.6f}  ({time.time()-t0:.1f} s) -> {path}")


if __name__ == "__main__":
    main()
