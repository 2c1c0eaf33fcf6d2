"""The reference's own GPU kernel ``cuVMC`` as a statistical oracle and as a
baseline (test and baseline infrastructure; never part of the product).

``oracle/_ref/libcuvmc_ref.so`` comes from ``oracle/ref_gpu_build.py``.  It
holds the reference's kernel source (pymopt/voxel_gpu/_cukernel.py:27-227),
compiled unchanged for sm_100a.  Photons are prepared here as
``VoxelModel.start()`` prepares them for the TEM00 pencil beam
(pymopt/voxel_gpu/_classes.py:75-112, 155-221):

* voxel ``(int((nx-1)/2), int((ny-1)/2), 1)``;
* offset ``(0, 0, -l/2)``, direction ``(0, 0, 1)``;
* weight ``1 - Rsp``;
* int8 labels, ``M = ny``, ``L = nz``, ``threadnum`` threads per block.

Results are read back as the reference reads them:
* ``Rd = sum w[v_z < 0] / nPh`` and ``Tt = sum w[v_z > 0] / nPh``
  (pymopt/voxel_gpu/_classes.py:326-337);
* exit positions encoded against the beam-axis voxel
  (pymopt/voxel_gpu/_classes.py:302-310);
* annulus bins ``(i dr, (i+1) dr]`` over ``2 pi (i + 1/2) dr^2 nPh``
  (pymopt/metrics/_scoring.py:16-25).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libcuvmc_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB} is not built (oracle/ref_gpu_build.py)")
        lib = C.CDLL(LIB)
        f = lib.ref_cuvmc_launch
        f.restype = C.c_int
        f.argtypes = [C.c_void_p] * 9 + [C.c_float, C.c_int, C.c_int, C.c_int, C.c_byte,
                                         C.c_int, C.c_int, C.c_void_p]
        _lib = lib
    return _lib


class RefVolume:
    """The reference's device-side inputs of one pencil-beam problem."""

    def __init__(self, prob, device="cuda"):
        e = int(prob.end_label)
        prob.validate()
        if prob.vox_ma is not None:
            raise ValueError("the reference kernel has per-label optics only")
        present = np.unique(prob.labels)
        inner = present[present != e]
        # cuVMC steps voxel to voxel while st >= db * mt: with mt == 0 a photon
        # trapped by total internal reflection would never leave its loop
        if np.any(prob.ma[inner] + prob.ms[inner] <= 0) or np.any(prob.ma[inner] < 0):
            raise ValueError("every label inside the volume needs ma + ms > 0")
        if int(prob.n_labels) > 127:
            raise ValueError("the reference indexes labels through a signed char")
        self.prob = prob
        self.device = torch.device(device)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)  # noqa: E731
        # ma, ms, g: one entry per layer label; n: one more, the ambient
        # index at end_point (pymopt/voxel_gpu/_classes.py:416-426)
        self.ma = t(prob.ma[:e].astype(np.float32))
        self.ms = t(prob.ms[:e].astype(np.float32))
        self.g = t(prob.g[:e].astype(np.float32))
        self.n = t(prob.n.astype(np.float32))
        self.model = t(prob.labels.view(np.int8))
        self.M, self.L = int(prob.labels.shape[1]), int(prob.labels.shape[2])

    def initial_state(self, n_photons: int):
        """Pencil-beam state arrays (SoA, reference layout), on the device."""
        pr = self.prob
        cx, cy, cz = pr.src_add
        dev = self.device
        add = torch.empty((3, n_photons), dtype=torch.int32, device=dev)
        add[0].fill_(int(cx))
        add[1].fill_(int(cy))
        add[2].fill_(int(cz))
        p = torch.zeros((3, n_photons), dtype=torch.float32, device=dev)
        p[2].fill_(float(np.float32(-pr.voxel_space / 2)))
        v = torch.zeros((3, n_photons), dtype=torch.float32, device=dev)
        v[2].fill_(1.0)
        w = torch.full((n_photons,), float(np.float32(pr.src_w0)), dtype=torch.float32,
                       device=dev)
        return add, p, v, w

    def launch(self, add, p, v, w, seed: int, threadnum: int = 128, stream=None) -> None:
        n = int(w.numel())
        s = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        st = load().ref_cuvmc_launch(
            add.data_ptr(), p.data_ptr(), v.data_ptr(), w.data_ptr(), self.ma.data_ptr(),
            self.ms.data_ptr(), self.n.data_ptr(), self.g.data_ptr(), self.model.data_ptr(),
            float(np.float32(self.prob.voxel_space)), self.M, self.L, n,
            int(self.prob.end_label), int(seed), int(threadnum), s)
        if st != 0:
            raise RuntimeError(f"reference cuVMC launch failed: CUDA error {st}")

    def results(self, add, p, v, w, nr: int, dr: float) -> dict:
        """Rd, Tt, R(r), T(r) read the reference's way (FP64 sums)."""
        n = int(w.numel())
        pr = self.prob
        l = float(np.float32(pr.voxel_space))
        cx, cy = pr.center
        wd = w.double()
        vz = v[2]
        rd, tt = vz < 0, vz > 0
        x = l * (add[0] - int(cx)).double() + p[0].double()
        y = l * (add[1] - int(cy)).double() + p[1].double()
        r = torch.sqrt(x * x + y * y)
        idx = torch.ceil(r / dr).long() - 1
        ok = (r > 0) & (idx >= 0) & (idx < nr)
        area = torch.tensor([2 * np.pi * (i + 0.5) * dr ** 2 for i in range(nr)],
                            dtype=torch.float64, device=w.device)
        out = {"Rd": float(wd[rd].sum()) / n, "Tt": float(wd[tt].sum()) / n}
        for key, sel in (("Rr", rd), ("Tr", tt)):
            m = sel & ok
            h = torch.bincount(idx[m], weights=wd[m], minlength=nr)[:nr]
            out[key] = (h / (area * n)).cpu().numpy()
        return out

    def run(self, n_photons: int, seed: int, nr: int = 100, dr: float = 0.1,
            threadnum: int = 128) -> dict:
        add, p, v, w = self.initial_state(n_photons)
        self.launch(add, p, v, w, seed, threadnum)
        return self.results(add, p, v, w, nr, dr)
