"""Host-side description of one transport problem.

A :class:`TransportProblem` holds everything a run needs besides the photon
range and seed: the padded label volume, the per-label (or per-voxel) optical
properties and the photon source.  The model classes of
:mod:`pymonteopt_b200.voxel` build one from the reference's params dicts; the
engine (:mod:`pymonteopt_b200.engine`) uploads it to the GPU.

Conventions follow the reference voxel path:

* ``labels`` is a C-order ``(nx, ny, nz)`` uint8 array padded by a one-voxel
  shell of ``end_label`` (pymopt/voxel_gpu/_classes.py:439-459);
* ``ma, ms, g`` are indexed by label, ``n`` by label with ``n[end_label]`` the
  ambient index (pymopt/voxel_gpu/_classes.py:416-426);
* the pencil source starts at voxel ``(int((nx-1)/2), int((ny-1)/2), 1)`` with
  in-voxel offset ``(0, 0, -l/2)`` and direction ``(0, 0, 1)``
  (pymopt/voxel_gpu/_classes.py:155-202);
* exit positions are encoded relative to voxel ``(center_ix, center_iy)``
  (pymopt/voxel_gpu/_classes.py:302-310).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi as A


def center_add(length: int) -> int:
    """Beam-axis voxel index of a padded axis (pymopt/voxel_gpu/_classes.py:165-169)."""
    return int((length - 1) / 2)


def check_volume(shell_broken: bool, max_label: int, n_labels: int) -> None:
    """Raise for a volume without a complete end_label shell, or with a label
    that has no optical properties."""
    if shell_broken:
        raise ValueError("the volume must be enclosed by a one-voxel shell of end_label")
    if max_label >= n_labels:
        raise ValueError(f"label {max_label} has no optical properties "
                         f"(n_labels = {n_labels})")


@dataclass
class TransportProblem:
    labels: np.ndarray                      # (nx, ny, nz) uint8, padded
    voxel_space: float                      # l [mm]
    end_label: int
    ma: np.ndarray                          # (n_labels,) float32
    ms: np.ndarray
    g: np.ndarray
    n: np.ndarray
    # source
    source: int = A.PMO_SRC_PENCIL
    src_add: tuple = (0, 0, 1)
    src_p: tuple = (0.0, 0.0, 0.0)
    src_v: tuple = (0.0, 0.0, 1.0)
    src_w0: float = 1.0
    beam_sigma: float = 0.0
    spec_prob: float = 0.0
    spec_v: tuple = (0.0, 0.0, -1.0)
    center: tuple = (0, 0)
    # per-voxel optics (PMO_PROPS_VOXEL)
    vox_ma: Optional[np.ndarray] = None
    vox_ms: Optional[np.ndarray] = None
    # PMO_SRC_STATE initial state (SoA, reference layout)
    state_add: Optional[np.ndarray] = None   # (3, N) int32
    state_p: Optional[np.ndarray] = None     # (3, N) float32
    state_v: Optional[np.ndarray] = None     # (3, N) float32
    state_w: Optional[np.ndarray] = None     # (N,) float32
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        self.labels = np.ascontiguousarray(self.labels, dtype=np.uint8)
        n_lab = len(self.n)
        pad = lambda a: np.ascontiguousarray(  # noqa: E731
            np.concatenate([np.asarray(a, np.float32).ravel(),
                            np.zeros(max(0, n_lab - len(a)), np.float32)]))
        self.ma = pad(self.ma)
        self.ms = pad(self.ms)
        self.g = pad(self.g)
        self.n = np.ascontiguousarray(np.asarray(self.n, np.float32))
        if self.vox_ma is not None:
            self.vox_ma = np.ascontiguousarray(self.vox_ma, dtype=np.float32)
            self.vox_ms = np.ascontiguousarray(self.vox_ms, dtype=np.float32)

    # ------------------------------------------------------------------
    @property
    def shape(self):
        return self.labels.shape

    @property
    def n_labels(self) -> int:
        return len(self.n)

    @property
    def props_mode(self) -> int:
        return A.PMO_PROPS_VOXEL if self.vox_ma is not None else A.PMO_PROPS_LABEL

    def validate(self, labels: bool = True) -> None:
        """Host-side checks that the device kernels rely on.

        The reference never checks its volume; an unpadded volume would let
        cuVMC read outside ``voxel_model``.  Here the shell, the label range
        and the source voxel are checked once per problem.  ``labels=False``
        leaves out the two checks that read the whole volume (the shell and
        the label range); the engine runs those on the uploaded copy instead
        (:func:`check_volume`).
        """
        lab = self.labels
        if lab.ndim != 3 or min(lab.shape) < 3:
            raise ValueError("labels must be a 3-D volume of at least 3 voxels per axis")
        if lab.size >= 2**32:
            raise ValueError("label volume larger than 2^32 voxels")
        e = int(self.end_label)
        if not (0 <= e < self.n_labels <= 256):
            raise ValueError(
                f"end_label {e} must index n (len {self.n_labels}), n_labels <= 256")
        if labels:
            faces = (lab[0], lab[-1], lab[:, 0], lab[:, -1], lab[:, :, 0], lab[:, :, -1])
            check_volume(any(np.any(f != e) for f in faces), int(lab.max()), self.n_labels)
        if self.voxel_space <= 0 or not np.isfinite(self.voxel_space):
            raise ValueError("voxel_space must be positive")
        for name in ("ma", "ms", "g", "n"):
            a = getattr(self, name)
            if not np.all(np.isfinite(a)):
                raise ValueError(f"{name} contains non-finite values")
        if np.any(self.ma < 0) or np.any(self.ms < 0):
            raise ValueError("ma and ms must be non-negative")
        if np.any(np.abs(self.g) > 1):
            raise ValueError("g must lie in [-1, 1]")
        if np.any(self.n <= 0):
            raise ValueError("n must be positive")
        if self.vox_ma is not None:
            if self.vox_ma.shape != lab.shape or self.vox_ms.shape != lab.shape:
                raise ValueError("vox_ma / vox_ms must have the label volume's shape")
            if not (np.all(np.isfinite(self.vox_ma)) and np.all(np.isfinite(self.vox_ms))):
                raise ValueError("vox_ma / vox_ms contain non-finite values")
            if np.any(self.vox_ma < 0) or np.any(self.vox_ms < 0):
                raise ValueError("vox_ma and vox_ms must be non-negative")
        if self.source != A.PMO_SRC_STATE:
            ix, iy, iz = self.src_add
            if not (0 < ix < lab.shape[0] - 1 and 0 < iy < lab.shape[1] - 1
                    and 0 < iz < lab.shape[2] - 1):
                raise ValueError(f"source voxel {self.src_add} is not inside the volume")
            if int(lab[ix, iy, iz]) == e:
                raise ValueError("source voxel lies in the end_label shell")

    def fill_struct(self, s: A.PmoProblem) -> None:
        """Copy the scalar fields into a ctypes :class:`PmoProblem`."""
        s.nx, s.ny, s.nz = (int(x) for x in self.labels.shape)
        s.voxel_space = float(self.voxel_space)
        s.end_label = int(self.end_label)
        s.props_mode = self.props_mode
        s.n_labels = self.n_labels
        s.source = int(self.source)
        s.src_ix, s.src_iy, s.src_iz = (int(x) for x in self.src_add)
        for i in range(3):
            s.src_p[i] = float(self.src_p[i])
            s.src_v[i] = float(self.src_v[i])
            s.spec_v[i] = float(self.spec_v[i])
        s.src_w0 = float(self.src_w0)
        s.beam_sigma = float(self.beam_sigma)
        s.spec_prob = float(self.spec_prob)
        s.center_ix, s.center_iy = (int(x) for x in self.center)


def pencil_problem(labels: np.ndarray, voxel_space: float, end_label: int,
                   ma, ms, g, n, *, beam_sigma: float = 0.0) -> TransportProblem:
    """A problem with the reference's default TEM00 pencil source and specular
    loss ``w = 1 - Rsp`` (pymopt/voxel_gpu/_classes.py:204-221)."""
    nx, ny, _ = labels.shape
    cx, cy = center_add(nx), center_add(ny)
    n = np.asarray(n, np.float32)
    n1, n2 = n[end_label], n[int(labels[cx, cy, 1])]
    rsp = ((n1 - n2) / (n1 + n2)) ** 2 if n1 != n2 else np.float32(0.0)
    return TransportProblem(
        labels=labels, voxel_space=voxel_space, end_label=end_label,
        ma=ma, ms=ms, g=g, n=n,
        source=A.PMO_SRC_GAUSSIAN if beam_sigma > 0 else A.PMO_SRC_PENCIL,
        src_add=(cx, cy, 1), src_p=(0.0, 0.0, -voxel_space / 2),
        src_v=(0.0, 0.0, 1.0), src_w0=np.float32(1.0) - np.float32(rsp),
        beam_sigma=beam_sigma, center=(cx, cy),
    )
