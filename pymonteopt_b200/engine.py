"""GPU engine: upload a :class:`~pymonteopt_b200.problem.TransportProblem`,
run photon ranges through the C ABI, read tallies back.

PyTorch supplies device memory and the current CUDA stream; all compute is in
``libpmo_b200.so``.  Every call is stream-ordered on the current stream and
asynchronous until a tally is read on the host.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _abi as A
from ._lib import PmoError, check, load
from .problem import check_volume


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


def _stream_handle(stream: Optional[torch.cuda.Stream] = None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def require_cuda(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("pymonteopt_b200 needs a CUDA device (B200, sm_100a); "
                           "there is no CPU fallback")
    d = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if d.type != "cuda":
        raise RuntimeError(f"device {d} is not a CUDA device")
    return d


SKIP_CAP = 15   # z half-extent of the uniform boxes (lateral: up to 192 voxels)


def check_labels(labels: torch.Tensor, end_label: int, n_labels: int) -> None:
    """The volume checks of ``TransportProblem.validate`` (a complete shell of
    ``end_label``, every label below ``n_labels``) on a device copy of the
    labels: a few reductions and one read-back, instead of host passes over
    the whole volume."""
    e = int(end_label)
    faces = (labels[0], labels[-1], labels[:, 0], labels[:, -1], labels[:, :, 0],
             labels[:, :, -1])
    shell = torch.stack([(f != e).any() for f in faces]).any()
    flags = torch.stack([shell.to(torch.int32), labels.max().to(torch.int32)]).tolist()
    check_volume(bool(flags[0]), int(flags[1]), int(n_labels))


class DeviceProblem:
    """A problem whose volume and optical tables are resident on one GPU.

    ``skip`` builds the uniform-box map (``pmo_build_voxel_words``) so that
    photons in per-label optics step from box face to box face; the path is
    the same as voxel-by-voxel stepping up to rounding.  ``skip=False`` keeps
    the reference's voxel-by-voxel stepping (the FP64 oracle comparisons use
    it)."""

    def __init__(self, prob, device=None, *, skip: bool = True, skip_cap: int = SKIP_CAP):
        load()
        self.device = require_cuda(device)
        prob.validate(labels=False)
        self.host = prob
        dev = self.device
        self.labels = torch.from_numpy(prob.labels).to(dev)
        check_labels(self.labels, prob.end_label, prob.n_labels)
        self.words = None
        self.skip_cap = int(skip_cap)
        if skip and prob.vox_ma is None:
            self.words = torch.empty(prob.labels.shape, dtype=torch.int16, device=dev)
            self.build_words()
        self.ma = torch.from_numpy(prob.ma).to(dev)
        self.ms = torch.from_numpy(prob.ms).to(dev)
        self.g = torch.from_numpy(prob.g).to(dev)
        self.n = torch.from_numpy(prob.n).to(dev)
        self.vox_ma = self.vox_ms = None
        if prob.vox_ma is not None:
            self.vox_ma = torch.from_numpy(prob.vox_ma).to(dev)
            self.vox_ms = torch.from_numpy(prob.vox_ms).to(dev)
        self.workspace = torch.empty(int(load().pmo_workspace_bytes()), dtype=torch.uint8,
                                     device=dev)

    def build_words(self, stream=None) -> None:
        """(Re)build the uniform-box map from the resident labels."""
        scratch = torch.empty(A.PMO_VOXEL_WORDS_SCRATCH * self.labels.numel(), dtype=torch.uint8,
                              device=self.device)
        nx, ny, nz = self.labels.shape
        st = load().pmo_build_voxel_words(self.labels.data_ptr(), nx, ny, nz, self.skip_cap,
                                          self.words.data_ptr(), scratch.data_ptr(),
                                          scratch.numel(), _stream_handle(stream))
        check(st, "pmo_build_voxel_words")

    def set_optics(self, ma=None, ms=None, vox_ma=None, vox_ms=None) -> None:
        """Replace optical properties in place (same shapes)."""
        for name, val in (("ma", ma), ("ms", ms), ("vox_ma", vox_ma), ("vox_ms", vox_ms)):
            if val is None:
                continue
            dst = getattr(self, name)
            src = torch.as_tensor(val, dtype=torch.float32).reshape(dst.shape)
            dst.copy_(src.to(self.device))

    def struct(self, seed: int, begin: int, count: int, precision: int, flags: int = 0,
               max_events: int = 0, state=None) -> A.PmoProblem:
        s = A.PmoProblem()
        self.host.fill_struct(s)
        s.labels = self.labels.data_ptr()
        s.voxel_words = self.words.data_ptr() if self.words is not None else None
        s.ma, s.ms, s.g, s.n = (t.data_ptr() for t in (self.ma, self.ms, self.g, self.n))
        if self.vox_ma is not None:
            s.vox_ma, s.vox_ms = self.vox_ma.data_ptr(), self.vox_ms.data_ptr()
        if state is not None:
            s.source = A.PMO_SRC_STATE
            s.state_add, s.state_p, s.state_v, s.state_w = (t.data_ptr() for t in state)
        s.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        s.photon_begin = int(begin)
        s.photon_count = int(count)
        s.max_events = int(max_events)
        s.precision = int(precision)
        s.flags = int(flags)
        return s


@dataclass
class TallySpec:
    nr: int = 0
    dr: float = 0.1
    fluence: int = A.PMO_FLU_NONE
    window: Optional[tuple] = None      # ((lo_x, lo_y, lo_z), (dim_x, dim_y, dim_z))
    export_exits: bool = False
    photon_stats: bool = False
    # angle-resolved exits: bins of arccos|v_z| over [0, pi/2]
    n_ang: int = 0
    # line profile of exits moving towards -x: depth bins for |y| < line_y_range
    n_line: int = 0
    line_dr: float = 0.1
    line_y_range: float = 5.0


class Tallies:
    """Device tally buffers of one run (accumulated across photon ranges)."""

    def __init__(self, dprob: DeviceProblem, spec: TallySpec, n_photons: int):
        dev = dprob.device
        self.spec = spec
        self.n_photons = 0
        self.capacity = int(n_photons)
        self.ledger = torch.zeros(A.PMO_LEDGER_N, dtype=torch.float64, device=dev)
        self.counters = torch.zeros(A.PMO_COUNTERS_N, dtype=torch.int64, device=dev)
        self.rr = (torch.zeros(A.PMO_RR_CATS, spec.nr, dtype=torch.float32, device=dev)
                   if spec.nr > 0 else None)
        # absorbed weight per voxel in 64-bit fixed point (2^PMO_ABSORBED_SHIFT
        # per unit weight; int64 storage of the kernel's unsigned sums)
        self.absorbed = (torch.zeros(dprob.labels.shape, dtype=torch.int64, device=dev)
                         if spec.fluence != A.PMO_FLU_NONE else None)
        self.ang = (torch.zeros(2, spec.n_ang, dtype=torch.float32, device=dev)
                    if spec.n_ang > 0 else None)
        self.line = (torch.zeros(spec.n_line, dtype=torch.float32, device=dev)
                     if spec.n_line > 0 else None)
        N = self.capacity
        if spec.export_exits:
            self.exit_add = torch.zeros(3, N, dtype=torch.int32, device=dev)
            self.exit_p = torch.zeros(3, N, dtype=torch.float32, device=dev)
            self.exit_v = torch.zeros(3, N, dtype=torch.float32, device=dev)
            self.exit_w = torch.zeros(N, dtype=torch.float32, device=dev)
        else:
            self.exit_add = self.exit_p = self.exit_v = self.exit_w = None
        if spec.photon_stats:
            self.ph = torch.zeros(3, N, dtype=torch.int32, device=dev)
        else:
            self.ph = None

    def zero_(self) -> "Tallies":
        for t in (self.ledger, self.counters, self.rr, self.absorbed, self.ang, self.line):
            if t is not None:
                t.zero_()
        self.n_photons = 0
        return self

    def struct(self) -> A.PmoTallies:
        sp = self.spec
        t = A.PmoTallies()
        t.ledger = self.ledger.data_ptr()
        t.counters = self.counters.data_ptr()
        t.rr = _ptr(self.rr)
        t.nr = int(sp.nr)
        t.dr = float(sp.dr)
        t.fluence_mode = int(sp.fluence)
        t.absorbed = _ptr(self.absorbed)
        if sp.fluence == A.PMO_FLU_SHARED:
            lo, dim = sp.window
            for a in range(3):
                t.win_lo[a] = int(lo[a])
                t.win_dim[a] = int(dim[a])
        t.exit_add, t.exit_p = _ptr(self.exit_add), _ptr(self.exit_p)
        t.exit_v, t.exit_w = _ptr(self.exit_v), _ptr(self.exit_w)
        t.ang, t.n_ang = _ptr(self.ang), int(sp.n_ang)
        t.line, t.n_line = _ptr(self.line), int(sp.n_line)
        t.line_dr, t.line_y_range = float(sp.line_dr), float(sp.line_y_range)
        if self.ph is not None:
            t.ph_interact = self.ph[0].data_ptr()
            t.ph_cross = self.ph[1].data_ptr()
            t.ph_fresnel = self.ph[2].data_ptr()
        return t

    # ---- host views -------------------------------------------------------
    def host_counters(self) -> np.ndarray:
        return self.counters.cpu().numpy().view(np.uint64)

    def check(self) -> None:
        """Synchronise and raise if any photon ended in an error."""
        c = np.ascontiguousarray(self.host_counters())
        status = load().pmo_check_counters(c.ctypes.data)
        if status != A.PMO_OK:
            raise PmoError(status, "transport")

    def summary(self) -> dict:
        L = self.ledger.cpu().numpy()
        c = self.host_counters()
        n = max(self.n_photons, 1)
        return {
            "nPh": self.n_photons,
            "Rd": L[A.PMO_L_RD] / n,
            "Tt": L[A.PMO_L_TT] / n,
            "A": L[A.PMO_L_ABS] / n,
            "ledger": L,
            "counters": c,
        }


def run_plain(dprob: DeviceProblem, n_photons: int, seed: int, *, tallies: Tallies = None,
              spec: TallySpec = None, begin: int = 0, precision: int = A.PMO_FP32,
              block_threads: int = 0, blocks_per_sm: int = 0, max_events: int = 0,
              stream=None) -> Tallies:
    """Trace photons ``[begin, begin + n_photons)`` and accumulate into
    ``tallies`` (created when None).  Asynchronous on the current stream."""
    lib = load()
    if tallies is None:
        tallies = Tallies(dprob, spec or TallySpec(), n_photons)
    sp = tallies.spec
    flags = (A.PMO_FLAG_EXPORT_EXITS if sp.export_exits else 0) | \
            (A.PMO_FLAG_PHOTON_STATS if sp.photon_stats else 0)
    if flags and n_photons > tallies.capacity:
        raise ValueError("per-photon outputs were sized for fewer photons")
    s = dprob.struct(seed, begin, n_photons, precision, flags, max_events)
    t = tallies.struct()
    launch = A.PmoLaunch(int(block_threads), int(blocks_per_sm))
    st = lib.pmo_run_plain(C.byref(s), C.byref(t), C.byref(launch),
                           C.c_void_p(dprob.workspace.data_ptr()),
                           dprob.workspace.numel(), _stream_handle(stream))
    check(st, "pmo_run_plain")
    tallies.n_photons += int(n_photons)
    return tallies


def absorbed_weight(tallies: Tallies) -> torch.Tensor:
    """The absorbed-weight grid as FP64 weight (fixed point / 2^32)."""
    if tallies.absorbed is None:
        raise ValueError("the run did not tally fluence")
    return tallies.absorbed.double() * (2.0 ** -A.PMO_ABSORBED_SHIFT)


def normalize_fluence(dprob: DeviceProblem, tallies: Tallies, stream=None) -> torch.Tensor:
    """FP64 fluence of the interior voxels, phi = absorbed / (nPh * l^3 * mu_a)."""
    if tallies.absorbed is None:
        raise ValueError("the run did not tally fluence")
    nx, ny, nz = dprob.labels.shape
    phi = torch.empty((nx - 2, ny - 2, nz - 2), dtype=torch.float64, device=dprob.device)
    s = dprob.struct(0, 0, 0, A.PMO_FP32)
    st = load().pmo_normalize_fluence(C.byref(s), C.c_void_p(tallies.absorbed.data_ptr()),
                                      float(max(tallies.n_photons, 1)),
                                      C.c_void_p(phi.data_ptr()), _stream_handle(stream))
    check(st, "pmo_normalize_fluence")
    return phi


def cuvmc(add: torch.Tensor, p: torch.Tensor, v: torch.Tensor, w: torch.Tensor,
          ma: torch.Tensor, ms: torch.Tensor, n: torch.Tensor, g: torch.Tensor,
          voxel_model: torch.Tensor, l: float, nPh: int, end_point: int, rand_seed: int,
          workspace: torch.Tensor, stream=None) -> None:
    """Drop-in for the reference kernel launch ``func(grid, block, (add, p, v,
    w, ma, ms, n, g, voxel_model, l, M, L, nPh, end_point, rand_seed))``
    (pymopt/voxel_gpu/_classes.py:105-111): updates add/p/v/w in place."""
    lib = load()
    K, M, L = voxel_model.shape
    for t, dt in ((add, torch.int32), (p, torch.float32), (v, torch.float32),
                  (w, torch.float32), (ma, torch.float32), (ms, torch.float32),
                  (n, torch.float32), (g, torch.float32), (voxel_model, torch.int8)):
        if t.dtype != dt or not t.is_cuda or not t.is_contiguous():
            raise ValueError(f"cuvmc expects contiguous CUDA {dt} tensors")
    st = lib.pmo_cuvmc(add.data_ptr(), p.data_ptr(), v.data_ptr(), w.data_ptr(),
                       ma.data_ptr(), ms.data_ptr(), n.data_ptr(), g.data_ptr(),
                       voxel_model.data_ptr(), float(l), int(M), int(L), int(nPh),
                       int(end_point), int(rand_seed), int(K),
                       C.c_void_p(workspace.data_ptr()), workspace.numel(),
                       _stream_handle(stream))
    check(st, "pmo_cuvmc")


def main(argv=None) -> int:
    """``python -m pymonteopt_b200.engine``: time plain launches on one of the
    synthetic volumes and print one JSON line (photons/s of the best launch).
    The volume stays resident and L2 is not flushed between launches; the
    benchmark of record is ``bench.py``."""
    import argparse
    import json
    from . import volumes as V
    vols = {"c1": V.c1_slab, "c2": V.c2_skin, "c3": V.c3_ct_like, "c4": V.c4_voxel_props}
    flu = {"none": A.PMO_FLU_NONE, "global": A.PMO_FLU_GLOBAL}
    ap = argparse.ArgumentParser(description=main.__doc__.split("\n")[0])
    ap.add_argument("--volume", choices=sorted(vols), default="c3")
    ap.add_argument("--photons", type=float, default=1e7)
    ap.add_argument("--fluence", choices=sorted(flu), default="none")
    ap.add_argument("--nr", type=int, default=100)
    ap.add_argument("--dr", type=float, default=0.1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--block-threads", type=int, default=0)
    ap.add_argument("--words-reps", type=int, default=0,
                    help="time this many uniform-box map builds instead of transport")
    args = ap.parse_args(argv)
    n = int(args.photons)
    dp = DeviceProblem(vols[args.volume]())
    if args.words_reps > 0:
        # the box map's build alone (the volume was uploaded and built once)
        ts = []
        for _ in range(args.words_reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dp.build_words()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        nvox = dp.labels.numel()
        print(json.dumps({"volume": args.volume, "voxels": nvox, "words_seconds": min(ts),
                          "voxels_per_s": nvox / min(ts)}))
        return 0
    spec = TallySpec(nr=args.nr, dr=args.dr, fluence=flu[args.fluence])
    tallies = Tallies(dp, spec, n)
    best = float("inf")
    for r in range(args.warmup + args.reps):
        tallies.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run_plain(dp, n, 1 + r, tallies=tallies, block_threads=args.block_threads)
        e1.record()
        torch.cuda.synchronize()
        tallies.check()
        if r >= args.warmup:
            best = min(best, e0.elapsed_time(e1) / 1e3)
    s = tallies.summary()
    c = s["counters"]
    print(json.dumps({"volume": args.volume, "photons": n, "fluence": args.fluence,
                      "seconds": best, "photons_per_s": n / best,
                      "Rd": float(s["Rd"]), "Tt": float(s["Tt"]), "A": float(s["A"]),
                      "interactions_per_photon": float(c[A.PMO_C_INTERACT]) / n,
                      "crossings_per_photon": float(c[A.PMO_C_CROSS]) / n,
                      "fresnel_per_photon": float(c[A.PMO_C_FRESNEL]) / n}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
