"""Turing-pattern trabecular-bone volumes on the GPU (torch.fft / cuFFT).

Produces the binary bone volumes that :class:`VoxelTuringModel.set_model`
takes, like the reference's ``TuringPattern``
(pymopt/modeling_gpu/_classes.py:24-236 on CuPy, and its scipy twin
pymopt/modeling/_classes.py:26-170).  The algorithm is the reference's:

* **Reaction-diffusion.**
  - Activator ``u`` and inhibitor ``v`` live on a periodic
    ``(length*grid)^3`` grid.
  - They start from ``1 - rand`` drawn by NumPy's legacy generator: seed
    ``seed`` for u and ``2*seed`` for v, unseeded when ``seed`` is falsy.
  - Each step is one semi-implicit diffusion step in Fourier space:
    ``u <- Re ifftn(K_u * Re fftn(f(u, v)))`` with
    ``K_u = 1 / Re fftn(k_u)``, where ``k_u`` is the 7-point implicit
    Laplacian stencil ``1 + 6 dt du/dx^2`` at the origin and
    ``-dt du/dx^2`` at the six neighbours.  ``v`` is updated the same way.
  - As in the reference, only the real part of the forward transform is kept.
* **Threshold.**
  - The threshold is a cubic in the target BV/TV (coefficients ``coef``).
  - Voxels at or below it are set to 0, and BV/TV real is the remaining
    fraction.
* **Microarchitecture.**
  - Tb.N* counts, along the last axis, the strict local maxima of
    order 5 (``scipy.signal.argrelmax`` with its clipped ends), averaged per
    row, summed over the first axis, over ``voxelsize * gridsize^2``.
  - Tb.Th, Tb.Sp and Dtorb are derived from Tb.N*.
* **Binarisation and tiling.** Voxels > 0 become 1 (int8), and the volume is
  tiled ``(tile_num_xz, tile_num_y, tile_num_xz)``.

The grids here are float32 and complex64 on the device, the reference's
precision.  At the reference's default size (520^3) a step is four 3-D FFTs
of 1.1 GB complex arrays.
"""
from __future__ import annotations

import datetime
import json
import os

import numpy as np
import torch

from .utils import ToJsonEncoder, set_params

__all__ = ["TuringPattern"]


def _relmax_count(u: torch.Tensor, order: int = 5) -> torch.Tensor:
    """Strict local maxima of ``order`` along the last axis, counted per row,
    with the index clipping of scipy.signal.argrelmax (mode='clip')."""
    n = u.shape[-1]
    idx = torch.arange(n, device=u.device)
    peak = torch.ones_like(u, dtype=torch.bool)
    for k in range(1, order + 1):
        plus = u.index_select(-1, torch.clamp(idx + k, max=n - 1))
        minus = u.index_select(-1, torch.clamp(idx - k, min=0))
        peak &= (u > plus) & (u > minus)
    return peak.sum(dim=-1)


class TuringPattern:
    """Drop-in for the reference's TuringPattern (same params, methods and
    return values), computed with torch on ``device`` (default: CUDA)."""

    def __init__(self, device=None):
        self.dtype = "float32"
        self.save_dicom = False
        self.params = {
            "grid": 40,
            "dx": 1 / 40,
            "dt": 1,
            "du": 0.0002,
            "dv": 0.01,
            "length": 13,
            "repetition": 100,
            "bv_tv": 0.138,
            "voxelsize": 0.0295,
            "seed": False,
            "ct_coef": 4.5e4,
            "tile_num_xz": 1,
            "tile_num_y": 1,
        }
        self.coef = np.array([-7.67681281, 1.65199492, -0.45314158, 0.60424417])
        self.keys_params = list(self.params.keys())
        self._setatter_params()
        self.f = lambda u, v: u + self.dt * (0.6 * u - v - u ** 3)
        self.g = lambda u, v: v + self.dt * (1.5 * u - 2 * v)
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("TuringPattern runs on a CUDA device; pass device= "
                                   "explicitly to run elsewhere")
            device = "cuda"
        self.device = torch.device(device)

    # ---- parameters (pymopt/modeling_gpu/_classes.py:78-100) ---------------
    def set_threshold_func_coef(self, coef):
        self.coef = np.array(coef)

    def set_params(self, *initial_data, **kwargs):
        set_params(self.params, self.keys_params, *initial_data, **kwargs)
        self._setatter_params()

    def set_inhibitor_function(self, g):
        self.g = g

    def set_activator_function(self, f):
        self.f = f

    def _setatter_params(self):
        for k in self.params:
            setattr(self, k, self.params[k])
        self.gridsize = self.length * self.grid

    # ---- reaction-diffusion --------------------------------------------------
    def _kernel_vector3(self, dd):
        gs = self.gridsize
        ke = np.float32(-self.dt * dd / self.dx ** 2)
        k = torch.zeros((gs, gs, gs), dtype=torch.float32, device=self.device)
        k[0, 0, 0] = float(np.float32(1 + 6 * self.dt * dd / self.dx ** 2))
        for i in ((1, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
            k[i] = float(ke)
        return k

    def _calc_kukv(self):
        self.ku = 1 / torch.fft.fftn(self._kernel_vector3(self.du)).real
        self.kv = 1 / torch.fft.fftn(self._kernel_vector3(self.dv)).real

    def _calc_onestep(self, u, v):
        a = torch.fft.ifftn(self.ku * torch.fft.fftn(self.f(u, v)).real).real
        b = torch.fft.ifftn(self.kv * torch.fft.fftn(self.g(u, v)).real).real
        return a, b

    def _get_inital_vector(self):
        gs = self.gridsize
        if self.seed:
            np.random.seed(seed=int(self.seed))
        ui = 1 - np.random.rand(gs, gs, gs).astype(self.dtype)
        if self.seed:
            np.random.seed(seed=int(self.seed * 2))
        vi = 1 - np.random.rand(gs, gs, gs).astype(self.dtype)
        return (torch.from_numpy(ui).to(self.device), torch.from_numpy(vi).to(self.device))

    # ---- post-processing -----------------------------------------------------
    def _get_threshold(self):
        self.threshold = np.poly1d(self.coef)(self.bv_tv)

    def _adjust_vbtv(self, u):
        self._get_threshold()
        low = u <= float(self.threshold)
        u = torch.where(low, torch.zeros((), dtype=u.dtype, device=u.device), u)
        self.bv_tv_real = 1 - int(low.sum()) / u.numel()
        return u

    def _calc_microarchitecture(self, u):
        # per first-axis slice: peaks per row averaged over its rows, summed
        per_slice = _relmax_count(u).double().mean(dim=-1)
        self.num_peak = float(per_slice.sum())
        tbn = self.num_peak / (self.voxelsize * self.gridsize ** 2)
        self.microarchitecture = {
            "BV/TV": self.bv_tv,
            "BV/TV real": self.bv_tv_real,
            "Tb.N* [/mm]": tbn,
            "Tb.Th [mm]": (self.bv_tv_real / tbn),
            "Tb.Sp [mm]": ((1 - self.bv_tv_real) / tbn),
            "Dtorb [mg/cm3]": (self.bv_tv_real * 1200),
        }

    def _model_binarization(self, u):
        return (u > 0).to(torch.int8)

    def _save_info(self, path, coment=""):
        info = {
            "Date": datetime.datetime.now().isoformat(),
            "coment": coment,
            "model_params": self.params,
            "microarchitecture": self.microarchitecture,
            "model_shape": self.model_shape,
        }
        with open(os.path.join(path, "_info.json"), "w") as fp:
            json.dump(info, fp, indent=4, cls=ToJsonEncoder)

    def _save_dicom(self, u, path):
        try:
            import pydicom  # noqa: F401
        except ImportError as e:
            raise ImportError("save_dicom=True needs pydicom, which is not installed") from e
        raise NotImplementedError("DICOM export is not part of this package")

    # ---- driver (pymopt/modeling_gpu/_classes.py:51-76) ----------------------
    def modeling(self, path, save_dicom=False):
        """Grow the pattern, write ``path/_info.json`` and return the binary
        int8 volume (NumPy, tiled)."""
        self.save_dicom = save_dicom
        self._calc_kukv()
        u, v = self._get_inital_vector()
        for _ in range(self.repetition):
            u, v = self._calc_onestep(u, v)
        self.model_shape = tuple(u.shape)
        del v, self.ku, self.kv
        if save_dicom:
            self._save_dicom(u, path)
        u = self._adjust_vbtv(u)
        self._calc_microarchitecture(u)
        self._save_info(path)
        vol = self._model_binarization(u).cpu().numpy()
        if self.tile_num_xz != 0:
            vol = np.tile(vol, (self.tile_num_xz, self.tile_num_y, self.tile_num_xz))
        return vol


def main(argv=None) -> int:
    """``python -m pymonteopt_b200.turing``: time TuringPattern.modeling at
    the reference's default size (520^3, 100 steps) and print one JSON line."""
    import argparse
    import tempfile
    import time
    ap = argparse.ArgumentParser(description=main.__doc__.split("\n")[0])
    ap.add_argument("--grid", type=int, default=40)
    ap.add_argument("--length", type=int, default=13)
    ap.add_argument("--repetition", type=int, default=100)
    args = ap.parse_args(argv)
    tp = TuringPattern()
    tp.set_params(grid=args.grid, dx=1 / args.grid, length=args.length,
                  repetition=args.repetition, seed=1)
    with tempfile.TemporaryDirectory() as d:
        tp.modeling(d)                                   # warm-up (cuFFT plans)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        vol = tp.modeling(d)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    print(json.dumps({"gridsize": tp.gridsize, "repetition": tp.repetition, "seconds": dt,
                      "steps_per_s": tp.repetition / dt, "bv_tv_real": tp.bv_tv_real,
                      "volume_shape": list(vol.shape)}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
