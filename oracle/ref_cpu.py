"""The reference's own CPU transport path, run unmodified (test and baseline
infrastructure).

``pymopt.voxel.VoxelPlateModel`` (pymopt/voxel/_classes.py) drives the Numba
kernel ``vmc_kernel`` (pymopt/voxel/_kernel.py:23-172), one photon after
another on one core.  The reference has no installable package (no setup.py
or pyproject.toml), so :func:`install` copies the Python sources of the
subpackages that path imports, unchanged, into ``baseline/_ref/pymopt``.
That folder is git-ignored: no reference source enters the history.  It
travels with the working tree to machines that have no reference checkout,
where ``bench.py``'s CPU baseline and reference arm import it from there.

The reference imports pydicom, matplotlib and seaborn at module level, and
its Gaussian beam draws plots while it samples (``gaussianBeam``,
pymopt/voxel/_classes.py:219-240).  None of these is installed, and none
takes part in the transport, so :func:`stub_modules` puts inert stand-ins in
``sys.modules`` before the import.

Seeding: the Gaussian beam draws from NumPy's global generator
(``scipy.stats.norm.rvs``) on the host; the kernel draws from Numba's own
generator, which only a jitted ``np.random.seed`` seeds.  :func:`run_plate`
seeds both.
"""
from __future__ import annotations

import contextlib
import io
import os
import shutil
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_DIR = os.path.join(REPO, "baseline", "_ref")
# the subpackages pymopt.voxel imports (voxel -> utils, fluence, optics;
# metrics for R(r))
SUBPACKAGES = ("voxel", "utils", "metrics", "fluence", "optics")


def default_reference_root() -> str | None:
    """A reference checkout named by ``PMO_REFERENCE_ROOT``, else a checkout
    called ``reference`` beside this repository, else None."""
    for cand in (os.environ.get("PMO_REFERENCE_ROOT"),
                 os.path.join(os.path.dirname(REPO), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "pymopt", "voxel")):
            return cand
    return None


def install(reference_root: str | None = None) -> str | None:
    """Copy the ``.py`` files of the reference subpackages into
    ``baseline/_ref/pymopt`` (sources only; the reference's compiled
    extensions are not copied).  Returns the folder, or None when no
    reference checkout is given or found."""
    root = reference_root or default_reference_root()
    if root is None:
        return REF_DIR if available() else None
    for sub in SUBPACKAGES:
        src = os.path.join(root, "pymopt", sub)
        dst = os.path.join(REF_DIR, "pymopt", sub)
        os.makedirs(dst, exist_ok=True)
        for name in sorted(os.listdir(src)):
            if name.endswith(".py"):
                shutil.copy2(os.path.join(src, name), os.path.join(dst, name))
    with open(os.path.join(REF_DIR, "SOURCE.txt"), "w") as f:
        f.write("Unmodified .py files of pyMonteOpt's pymopt/{%s}, copied by "
                "oracle/ref_cpu.py.\n" % ",".join(SUBPACKAGES))
    return REF_DIR


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "pymopt", "voxel", "_kernel.py"))


class _Inert:
    """Stands in for any plotting object: every attribute, call and item is
    another inert object; unpacking gives two of them (``fig, ax = ...``)."""

    def __getattr__(self, name):
        return _Inert()

    def __call__(self, *a, **k):
        return _Inert()

    def __getitem__(self, k):
        return _Inert()

    def __iter__(self):
        return iter((_Inert(), _Inert()))


def stub_modules() -> None:
    """Inert pydicom / matplotlib / seaborn modules for the reference's
    module-level imports and its plotting calls."""
    for name in ("pydicom", "pydicom.uid", "pydicom.dataset", "matplotlib",
                 "matplotlib.pyplot", "matplotlib.colors", "seaborn"):
        if name in sys.modules:
            continue
        m = types.ModuleType(name)
        m.__getattr__ = lambda attr: _Inert()   # module-level __getattr__ (PEP 562)
        sys.modules[name] = m
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.modules["matplotlib"].colors = sys.modules["matplotlib.colors"]
    sys.modules["pydicom"].uid = sys.modules["pydicom.uid"]
    sys.modules["pydicom"].dataset = sys.modules["pydicom.dataset"]


def import_reference(path: str | None = None):
    """Import ``pymopt`` (voxel and metrics) from ``path`` (a checkout or the
    copy in baseline/_ref) and return (pymopt.voxel, pymopt.metrics)."""
    path = path or REF_DIR
    stub_modules()
    if path not in sys.path:
        sys.path.insert(0, path)
    import pymopt.metrics as metrics
    import pymopt.voxel as voxel
    return voxel, metrics


_SEED_FN = None


def seed_all(s: int) -> None:
    """Seed NumPy's global generator (host-side beam sampling) and Numba's
    generator (the kernel's draws)."""
    global _SEED_FN
    if _SEED_FN is None:
        from numba import njit

        @njit
        def _seed(x):
            np.random.seed(x)
        _SEED_FN = _seed
    np.random.seed(s)
    _SEED_FN(s)


def run_plate(params: dict, nph: int, seed: int, model_kwargs: dict | None = None,
              nr: int = 100, dr: float = 0.1, path: str | None = None,
              model_class: str = "VoxelPlateModel") -> dict:
    """One ``VoxelPlateModel(nPh).build(**params).start()`` of the reference
    (or another model class of pymopt/voxel/_classes.py, e.g.
    ``VoxelPlateExModel``) with both generators seeded.  Returns Rd, Tt (by
    the sign of v_z, as getRdTtRate does, pymopt/voxel/_classes.py:259-266),
    R(r) and T(r) (metrics.radialDistance on the exits with v_z < 0 and
    v_z > 0) and the seconds spent in start()."""
    voxel, metrics = import_reference(path)
    model = getattr(voxel._classes, model_class)(nPh=nph, **(model_kwargs or {}))
    with contextlib.redirect_stdout(io.StringIO()):
        model.build(**params)
        seed_all(seed)
        t0 = time.perf_counter()
        model.start()
        dt = time.perf_counter() - t0
    res = model.get_result()
    v, w, p = res["v"], res["w"], res["p"]
    rd, tt = v[2] < 0, v[2] > 0
    out = {"Rd": float(w[rd].sum() / nph), "Tt": float(w[tt].sum() / nph), "seconds": dt,
           "nPh": nph, "seed": seed}
    if nr > 0:
        out["Rr"] = metrics.radialDistance(p[:, rd], w[rd], nr, dr, nph)[1].tolist()
        out["Tr"] = metrics.radialDistance(p[:, tt], w[tt], nr, dr, nph)[1].tolist()
    return out


def _plate_worker(args):
    try:
        return run_plate(*args)
    except ZeroDivisionError:
        # vmc_kernel's theta() (pymopt/voxel/_kernel.py:12-21) clamps cos(theta)
        # at -1 but not at +1; when float32 rounding pushes it above 1 the
        # direction becomes NaN and, under fastmath, Numba's zero-divisor
        # check on the renormalisation (:165) raises
        return None


def run_plate_seeds(params: dict, nph: int, seeds, model_kwargs: dict | None = None,
                    nr: int = 100, dr: float = 0.1, path: str | None = None,
                    model_class: str = "VoxelPlateModel", processes: int = 0) -> list:
    """:func:`run_plate` for each seed, on spawned worker processes; None for
    a seed whose run raised ZeroDivisionError in the reference kernel."""
    import multiprocessing as mp
    jobs = [(params, nph, s, model_kwargs, nr, dr, path, model_class) for s in seeds]
    processes = processes or min(len(jobs), os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(processes) as pool:
        return pool.map(_plate_worker, jobs)


_POOL_CASE = None


def _pool_init(params, model_kwargs, path):
    """Per worker process: import the reference and compile its kernel once."""
    global _POOL_CASE
    _POOL_CASE = (params, model_kwargs, path)
    # Numba JIT warm-up (vmc_kernel takes idx % (nPh // 10), so nPh >= 10)
    run_plate(params, 20, 7919, model_kwargs, nr=0, path=path)


def _pool_task(args):
    nph, seed = args
    params, model_kwargs, path = _POOL_CASE
    for attempt in range(8):
        try:
            r = run_plate(params, nph, seed + 100003 * attempt, model_kwargs, nr=0, path=path)
            return r["seconds"], r["Rd"], attempt
        except ZeroDivisionError:
            continue   # the reference kernel's NaN direction (see _plate_worker)
    raise RuntimeError("the reference kernel raised on 8 seeds in a row")


class RefPool:
    """``processes`` spawned workers running the reference's
    ``VoxelPlateModel.build(**params).start()``; each has compiled the Numba
    kernel before the first timed step."""

    def __init__(self, params: dict, processes: int, model_kwargs: dict | None = None,
                 path: str | None = None):
        import multiprocessing as mp
        self.processes = int(processes)
        self.pool = mp.get_context("spawn").Pool(
            self.processes, initializer=_pool_init, initargs=(params, model_kwargs, path))

    def step(self, nph_per_process: int, seed: int) -> dict:
        """Every process runs ``nph_per_process`` photons (distinct seeds) and
        times its own start(); the step's rate is all photons over the slowest
        process's seconds."""
        jobs = [(int(nph_per_process), seed + 7919 * i) for i in range(self.processes)]
        res = self.pool.map(_pool_task, jobs, chunksize=1)
        secs = [r[0] for r in res]
        return {"photons": self.processes * int(nph_per_process), "seconds": max(secs),
                "seconds_min": min(secs), "value": self.processes * nph_per_process / max(secs),
                "Rd_mean": float(np.mean([r[1] for r in res])),
                "rerun_seeds": int(sum(r[2] for r in res))}

    def close(self) -> None:
        self.pool.close()
        self.pool.join()


def host_cpu() -> dict:
    """CPU model and logical CPU count of this host (from /proc/cpuinfo)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return {"model": model, "logical_cpus": n}


def _timed_worker(args):
    params, model_kwargs, nph, seed, path = args
    # Numba JIT warm-up (vmc_kernel takes idx % (nPh // 10), so nPh >= 10)
    run_plate(params, 20, seed + 7919, model_kwargs, nr=0, path=path)
    r = run_plate(params, nph, seed, model_kwargs, nr=0, path=path)
    return r["seconds"], r["Rd"]


def rate(params: dict, nph: int, processes: int = 1, model_kwargs: dict | None = None,
         seed: int = 0, path: str | None = None) -> dict:
    """Photons/s of the reference's start() on ``processes`` independent
    processes (distinct seeds, ``nph`` photons each), JIT warm-up excluded.
    Each process times its own start(); the rate is the photons of all
    processes over the slowest process's time.  Processes are spawned, so a
    caller that already initialised CUDA is safe."""
    import multiprocessing as mp
    jobs = [(params, model_kwargs, nph, seed + 1000 * i, path) for i in range(processes)]
    if processes == 1:
        res = [_timed_worker(jobs[0])]
    else:
        with mp.get_context("spawn").Pool(processes) as pool:
            res = pool.map(_timed_worker, jobs)
    secs = [r[0] for r in res]
    return {"value": processes * nph / max(secs), "photons": processes * nph,
            "seconds_max": max(secs), "seconds_min": min(secs), "processes": processes,
            "Rd_mean": float(np.mean([r[1] for r in res]))}


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else None
    print(install(root))
