"""Seeded synthetic workloads (C1-C5).

Each generator returns host arrays only; nothing here touches the GPU.  All
randomness comes from ``numpy.random.Generator(PCG64(seed))``.

* :func:`plate_volume` — the reference PlateModel volume
  (pymopt/voxel_gpu/_classes.py:416-459): layers along z, labels 0..L-1, a
  one-voxel shell of ``end_label = L``.
* :func:`c1_slab` — homogeneous 10 mm slab, 101x101x100 voxels at 0.1 mm.
* :func:`c2_skin` — three-layer skin slab, 400x400x400 voxels at 0.05 mm.
* :func:`c3_ct_like` — 256^3 voxels at 0.2 mm, five classes thresholded from a
  Gaussian random field with 3 mm correlation length.
* :func:`c4_voxel_props` — 64^3 voxels at 0.25 mm with per-voxel ma/ms.
* :func:`c5_slab_batch` — 4096 independent single-layer slab problems.
"""
from __future__ import annotations

import numpy as np

from . import _abi as A
from .problem import TransportProblem, center_add, pencil_problem


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def plate_volume(x_size: float, y_size: float, voxel_space: float, thickness) -> tuple:
    """Padded layered volume exactly as PlateModel._make_voxel_model builds it
    (pymopt/voxel_gpu/_classes.py:424-459).  Returns ``(labels, end_label)``."""
    nx = int(np.int32(round(x_size / voxel_space)))
    ny = int(np.int32(round(y_size / voxel_space)))
    nz = int(np.int32(round(np.array(thickness).sum() / voxel_space)))
    vol = np.empty((nx + 2, ny + 2, nz + 2), np.uint8)
    val = 1
    for k, t in enumerate(thickness):
        n = round(t / voxel_space)
        vol[:, :, val:val + n] = k
        val += n
    end = len(thickness)
    vol[0], vol[-1] = end, end
    vol[:, 0], vol[:, -1] = end, end
    vol[:, :, 0], vol[:, :, -1] = end, end
    return vol, end


def plate_problem(params: dict, *, beam_sigma: float = 0.0) -> TransportProblem:
    """Problem for a PlateModel params dict (keys of PlateModel.params,
    pymopt/voxel_gpu/_classes.py:402-411)."""
    vol, end = plate_volume(params["x_size"], params["y_size"], params["voxel_space"],
                            params["thickness"])
    n = list(params["n"]) + [params["n_air"]]
    return pencil_problem(vol, params["voxel_space"], end, params["ma"], params["ms"],
                          params["g"], n, beam_sigma=beam_sigma)


C1_PARAMS = {
    "x_size": 10.1, "y_size": 10.1, "voxel_space": 0.1, "thickness": [10.0],
    "n": [1.37], "n_air": 1.0, "ma": [0.1], "ms": [10.0], "g": [0.9],
}

C2_PARAMS = {
    "x_size": 20.0, "y_size": 20.0, "voxel_space": 0.05, "thickness": [0.1, 2.0, 17.9],
    "n": [1.4, 1.4, 1.44], "n_air": 1.0, "ma": [0.5, 0.05, 0.01], "ms": [20.0, 15.0, 10.0],
    "g": [0.8, 0.85, 0.9],
}
C2_W_BEAM = 1.0  # 1/e^2 radius [mm]; sigma = w_beam / 2 (gaussianBeam, :267-273)


def c1_slab() -> TransportProblem:
    """C1: 101x101x100 voxels at 0.1 mm, ma 0.1, ms 10, g 0.9, n 1.37, pencil."""
    return plate_problem(C1_PARAMS)


def c2_skin(*, gaussian: bool = True) -> TransportProblem:
    """C2: three-layer skin slab, 400^3 voxels at 0.05 mm, Gaussian beam of
    1 mm 1/e^2 radius (pencil when ``gaussian`` is False)."""
    return plate_problem(C2_PARAMS, beam_sigma=C2_W_BEAM / 2 if gaussian else 0.0)


def gaussian_random_field(shape, corr_vox: float, rng: np.random.Generator) -> np.ndarray:
    """White noise low-pass filtered by a Gaussian of ``corr_vox`` voxels (FFT)."""
    noise = rng.standard_normal(shape, dtype=np.float32)
    f = np.fft.rfftn(noise)
    kx = np.fft.fftfreq(shape[0]).astype(np.float32)
    ky = np.fft.fftfreq(shape[1]).astype(np.float32)
    kz = np.fft.rfftfreq(shape[2]).astype(np.float32)
    s2 = np.float32((2 * np.pi * corr_vox) ** 2 / 2)
    f *= np.exp(-s2 * kx[:, None, None] ** 2)
    f *= np.exp(-s2 * ky[None, :, None] ** 2)
    f *= np.exp(-s2 * kz[None, None, :] ** 2)
    return np.fft.irfftn(f, s=shape, axes=(0, 1, 2)).astype(np.float32)


C3_CLASSES = ("air", "fat", "soft tissue", "muscle", "bone")


def c3_ct_like(seed: int = 0, n: int = 256, voxel_space: float = 0.2,
               corr_mm: float = 3.0) -> TransportProblem:
    """C3: n^3 interior voxels, five classes from a seeded Gaussian random field
    thresholded at its quintiles; per-class ma log-U[0.005, 0.5], ms U[5, 30],
    g U[0.8, 0.95], n U[1.0, 1.55] (air n = 1.0); ambient shell n = 1.0."""
    rng = _rng(seed)
    field = gaussian_random_field((n, n, n), corr_mm / voxel_space, rng)
    q = np.quantile(field, [0.2, 0.4, 0.6, 0.8])
    cls = np.searchsorted(q, field).astype(np.uint8)
    end = len(C3_CLASSES)
    vol = np.full((n + 2, n + 2, n + 2), end, np.uint8)
    vol[1:-1, 1:-1, 1:-1] = cls
    k = len(C3_CLASSES)
    ma = np.exp(rng.uniform(np.log(0.005), np.log(0.5), k)).astype(np.float32)
    ms = rng.uniform(5.0, 30.0, k).astype(np.float32)
    g = rng.uniform(0.8, 0.95, k).astype(np.float32)
    nn = rng.uniform(1.0, 1.55, k).astype(np.float32)
    nn[0] = 1.0
    n_tab = np.concatenate([nn, np.float32([1.0])])
    prob = pencil_problem(vol, voxel_space, end, ma, ms, g, n_tab)
    prob.meta.update({"workload": "c3_ct_like", "seed": seed, "classes": C3_CLASSES})
    return prob


def c4_voxel_props(seed: int = 0, n: int = 64, voxel_space: float = 0.25) -> TransportProblem:
    """C4: n^3 voxels at 0.25 mm, per-voxel ma log-U[0.01, 0.2], ms U[5, 20],
    g 0.9, n 1.4, ambient n 1.0, pencil beam."""
    rng = _rng(seed)
    vol = np.ones((n + 2, n + 2, n + 2), np.uint8)
    vol[1:-1, 1:-1, 1:-1] = 0
    vma = np.zeros(vol.shape, np.float32)
    vms = np.zeros(vol.shape, np.float32)
    vma[1:-1, 1:-1, 1:-1] = np.exp(rng.uniform(np.log(0.01), np.log(0.2), (n, n, n)))
    vms[1:-1, 1:-1, 1:-1] = rng.uniform(5.0, 20.0, (n, n, n))
    prob = pencil_problem(vol, voxel_space, 1, [0.0], [0.0], [0.9], [1.4, 1.0])
    prob.vox_ma, prob.vox_ms = vma, vms
    prob.__post_init__()
    prob.meta.update({"workload": "c4_voxel_props", "seed": seed})
    return prob


def c5_slab_batch(seed: int = 0, count: int = 4096) -> dict:
    """C5: ``count`` single-layer slabs: ma log-U[0.001, 1], ms' log-U[0.5, 5]
    (ms = ms' / (1 - g)), g U[0.7, 0.95], n U[1.33, 1.45], thickness U[1, 20] mm,
    photon budgets log-U[1e4, 1e6]; ambient n = 1.0."""
    rng = _rng(seed)
    ma = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), count))
    msp = np.exp(rng.uniform(np.log(0.5), np.log(5.0), count))
    g = rng.uniform(0.7, 0.95, count)
    ms = msp / (1 - g)
    n = rng.uniform(1.33, 1.45, count)
    th = rng.uniform(1.0, 20.0, count)
    nph = np.exp(rng.uniform(np.log(1e4), np.log(1e6), count)).astype(np.int64)
    return {"ma": ma.astype(np.float32), "ms": ms.astype(np.float32),
            "g": g.astype(np.float32), "n": n.astype(np.float32),
            "thickness": th.astype(np.float32), "n_photons": nph, "n_ambient": 1.0}


SKIN_LAYERS = [(0.5, 20.0, 0.8, 1.4, 0.1), (0.05, 15.0, 0.85, 1.4, 1.5),
               (0.02, 10.0, 0.9, 1.44, 1.4)]   # (ma, ms, g, n, thickness)


def skin_stack_sweep(seed: int = 0, count: int = 1024) -> dict:
    """A parameter sweep of three-layer skin stacks, as the reference's
    dataset driver sweeps PlateModel optics (pymopt/virtualOBD.py:139-147):
    the layers of the C2 slab (epidermis 0.1 mm, dermis 1.5 mm, subcutis
    1.4 mm), each layer's mu_a scaled by a log-uniform factor in [1/2, 2] and
    mu_s by one in [e^-0.5, e^0.5], photon budgets log-uniform in [1e4, 1e5].
    Returns ``stacks`` (count x 3 layer tuples) and ``n_photons``."""
    rng = _rng(seed)
    fa = np.exp(rng.uniform(-np.log(2.0), np.log(2.0), (count, 3)))
    fs = np.exp(rng.uniform(-0.5, 0.5, (count, 3)))
    stacks = [[(ma * fa[i, j], ms * fs[i, j], g, n, t)
               for j, (ma, ms, g, n, t) in enumerate(SKIN_LAYERS)] for i in range(count)]
    photons = np.exp(rng.uniform(np.log(1e4), np.log(1e5), count)).astype(np.int64)
    return {"stacks": stacks, "n_photons": photons}

