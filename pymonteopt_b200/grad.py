"""Differentiable R(r): forward transport plus Philox-replay backward.

:class:`DifferentiableRr` maps optical properties to the radially resolved
diffuse reflectance R(r) (the reference's ``radialDistance`` of exits with
v_z < 0, pymopt/metrics/_scoring.py:16-25) as a ``torch.autograd.Function``:

* forward: one transport run (``pmo_run_plain``) that also writes, per
  photon, the R(r) bin its exit weight went to and that weight (8 bytes per
  photon; no paths are stored);
* backward: ``pmo_run_grad`` replays every photon whose bin has a non-zero
  loss gradient from its Philox counters and accumulates the perturbation
  Monte Carlo derivatives of implicit-capture weighting,
  dR/dmu_a(v) = -E[w L_v], dR/dmu_s(v) = E[w (n_v / mu_s(v) - L_v)],
  per voxel (voxel-by-voxel stepping) and per label.

Parameters are either per label (``props='label'``: tensors of n_labels) or
per voxel (``props='voxel'``: tensors shaped like the padded volume; needs a
problem with per-voxel optics).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _abi as A
from . import engine as E
from ._lib import PmoError, check, load


def annulus_area(nr: int, dr: float) -> np.ndarray:
    """2 pi (i + 1/2) dr^2 (pymopt/metrics/_scoring.py:18)."""
    return np.array([2 * np.pi * (i + 0.5) * dr ** 2 for i in range(nr)])


class ReplayResult:
    def __init__(self, d_ma_voxel, d_ms_voxel, d_ma_label, d_ms_label, counters):
        self.d_ma_voxel = d_ma_voxel
        self.d_ms_voxel = d_ms_voxel
        self.d_ma_label = d_ma_label
        self.d_ms_label = d_ms_label
        self.counters = counters

    @property
    def replayed(self) -> int:
        return int(self.counters[A.PMO_G_REPLAYED])

    @property
    def mismatches(self) -> int:
        return int(self.counters[A.PMO_G_MISMATCH])


def run_forward_scored(dp: E.DeviceProblem, n: int, seed: int, nr: int, dr: float,
                       precision: int = A.PMO_FP32, block_threads: int = 0) -> E.Tallies:
    """Forward run that also records each photon's exit bin and weight."""
    spec = E.TallySpec(nr=nr, dr=dr)
    t = E.Tallies(dp, spec, n)
    t.score_bin = torch.empty(n, dtype=torch.int32, device=dp.device)
    t.score_w = torch.empty(n, dtype=torch.float32, device=dp.device)
    lib = load()
    s = dp.struct(seed, 0, n, precision, A.PMO_FLAG_SCORE_RECORD)
    ts = t.struct()
    ts.score_bin = t.score_bin.data_ptr()
    ts.score_w = t.score_w.data_ptr()
    st = lib.pmo_run_plain(C.byref(s), C.byref(ts), C.byref(A.PmoLaunch(block_threads, 0)),
                           C.c_void_p(dp.workspace.data_ptr()), dp.workspace.numel(),
                           E._stream_handle())
    check(st, "pmo_run_plain (scored)")
    t.n_photons = n
    return t


def run_replay(dp: E.DeviceProblem, fwd: E.Tallies, coef: torch.Tensor, seed: int, *,
               per_voxel: bool, per_label: bool = True, precision: int = A.PMO_FP32,
               block_threads: int = 0) -> ReplayResult:
    """Backward replay of the photons of ``fwd`` with loss weights ``coef``
    ([PMO_RR_CATS, nr] float32: dLoss/d(bin weight sum))."""
    if per_voxel and dp.words is not None:
        raise ValueError("per-voxel derivatives need voxel-by-voxel stepping: "
                         "build the DeviceProblem with skip=False")
    dev = dp.device
    n = fwd.n_photons
    nr = fwd.spec.nr
    coef = coef.to(device=dev, dtype=torch.float32).contiguous()
    assert coef.numel() == A.PMO_RR_CATS * nr
    g = A.PmoGrad()
    g.coef = coef.data_ptr()
    g.nr = nr
    g.dr = float(fwd.spec.dr)
    g.score_bin = fwd.score_bin.data_ptr()
    g.score_w = fwd.score_w.data_ptr()
    d_ma_v = d_ms_v = d_ma_l = d_ms_l = None
    if per_voxel:
        d_ma_v = torch.zeros(dp.labels.shape, dtype=torch.float32, device=dev)
        d_ms_v = torch.zeros_like(d_ma_v)
        g.d_ma_voxel, g.d_ms_voxel = d_ma_v.data_ptr(), d_ms_v.data_ptr()
    if per_label:
        nl = len(dp.host.n)
        d_ma_l = torch.zeros(nl, dtype=torch.float64, device=dev)
        d_ms_l = torch.zeros_like(d_ma_l)
        g.d_ma_label, g.d_ms_label = d_ma_l.data_ptr(), d_ms_l.data_ptr()
    cnt = torch.zeros(A.PMO_G_COUNTERS_N, dtype=torch.int64, device=dev)
    g.counters = cnt.data_ptr()
    s = dp.struct(seed, 0, n, precision)
    st = load().pmo_run_grad(C.byref(s), C.byref(g), C.byref(A.PmoLaunch(block_threads, 0)),
                             C.c_void_p(dp.workspace.data_ptr()), dp.workspace.numel(),
                             E._stream_handle())
    check(st, "pmo_run_grad")
    return ReplayResult(d_ma_v, d_ms_v, d_ma_l, d_ms_l, cnt.cpu().numpy().view(np.uint64))


class _RrFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ma, ms, model):
        model._set_optics(ma, ms)
        fwd = run_forward_scored(model.dp, model.n_photons, model.seed, model.nr, model.dr,
                                 model.precision, model.block_threads)
        fwd.check()
        rr = fwd.rr.to(torch.float64)
        R = (rr[A.PMO_RR_TOP] + rr[A.PMO_RR_LAT_NEG]) / (model.area * model.n_photons)
        ctx.model = model
        ctx.fwd = fwd
        model.last_forward = fwd
        return R

    @staticmethod
    def backward(ctx, grad_R):
        model, fwd = ctx.model, ctx.fwd
        w = (grad_R.to(torch.float64) / (model.area * model.n_photons)).to(torch.float32)
        coef = torch.zeros(A.PMO_RR_CATS, model.nr, dtype=torch.float32, device=w.device)
        coef[A.PMO_RR_TOP] = w
        coef[A.PMO_RR_LAT_NEG] = w
        # only the gradients this model returns are accumulated
        res = run_replay(model.dp, fwd, coef, model.seed, per_voxel=model.props == "voxel",
                         per_label=model.props != "voxel", precision=model.precision,
                         block_threads=model.block_threads)
        model.last_replay = res
        if res.mismatches:
            raise PmoError(A.PMO_ERR_NUMERIC,
                           f"gradient replay left the forward path for {res.mismatches} photons")
        if model.props == "voxel":
            return res.d_ma_voxel.to(grad_R.dtype), res.d_ms_voxel.to(grad_R.dtype), None
        return res.d_ma_label.to(grad_R.dtype), res.d_ms_label.to(grad_R.dtype), None


class DifferentiableRr:
    """R(r) [mm^-2] as a differentiable function of the optical properties.

    ``props='label'``: ``ma``, ``ms`` are n_labels tensors (the problem's
    per-label tables); uniform-box stepping stays on.
    ``props='voxel'``: ``ma``, ``ms`` are padded-volume tensors (per-voxel
    optics); stepping is voxel by voxel so the derivatives resolve voxels.
    """

    def __init__(self, prob, *, n_photons: int, seed: int = 0, nr: int = 50, dr: float = 0.1,
                 props: str = "label", precision: int = A.PMO_FP32, block_threads: int = 0,
                 device=None):
        if props not in ("label", "voxel"):
            raise ValueError("props must be 'label' or 'voxel'")
        if props == "voxel" and prob.vox_ma is None:
            raise ValueError("props='voxel' needs a problem with per-voxel optics (vox_ma/vox_ms)")
        self.props = props
        self.dp = E.DeviceProblem(prob, device, skip=(props == "label"))
        self.n_photons = int(n_photons)
        self.seed = int(seed)
        self.nr, self.dr = int(nr), float(dr)
        self.precision = precision
        self.block_threads = block_threads
        self.area = torch.tensor(annulus_area(self.nr, self.dr), dtype=torch.float64,
                                 device=self.dp.device)
        self.last_forward: Optional[E.Tallies] = None
        self.last_replay: Optional[ReplayResult] = None

    def _set_optics(self, ma, ms):
        if self.props == "voxel":
            self.dp.set_optics(vox_ma=ma.detach(), vox_ms=ms.detach())
        else:
            self.dp.set_optics(ma=ma.detach(), ms=ms.detach())

    def __call__(self, ma: torch.Tensor, ms: torch.Tensor) -> torch.Tensor:
        return _RrFunction.apply(ma, ms, self)

    def initial_params(self):
        """The problem's own optical properties as float64 leaf tensors."""
        h = self.dp.host
        if self.props == "voxel":
            ma, ms = h.vox_ma, h.vox_ms
        else:
            ma, ms = h.ma, h.ms
        dev = self.dp.device
        return (torch.tensor(ma, dtype=torch.float64, device=dev),
                torch.tensor(ms, dtype=torch.float64, device=dev))

    def fd_gradient(self, loss_fn, ma, ms, which: str, index, rel_step: float = 1e-3):
        """Central finite difference of ``loss_fn(R)`` with common random
        numbers (same seed and photons in both runs) with respect to
        ``ma`` or ``ms`` at ``index``; relative step ``rel_step``."""
        base = (ma if which == "ma" else ms).detach().clone()
        h = rel_step * float(base[index])
        vals = []
        for sign in (1.0, -1.0):
            p = base.clone()
            p[index] += sign * h
            with torch.no_grad():
                R = self(p, ms.detach()) if which == "ma" else self(ma.detach(), p)
            vals.append(float(loss_fn(R)))
        self._set_optics(ma.detach(), ms.detach())
        return (vals[0] - vals[1]) / (2 * h)


def reweighted_fd(dp: E.DeviceProblem, fwd: E.Tallies, coef: torch.Tensor, seed: int,
                  targets, param: str = "ma", rel_step: float = 1e-3,
                  precision: int = A.PMO_FP32) -> np.ndarray:
    """Central finite differences of the loss with ``coef`` = dLoss/d(bin weight
    sum), relative step ``rel_step``, on the photons of ``fwd`` (common random
    numbers): each target's mu is scaled by (1 +- h) and the photons are
    reweighted by the perturbation Monte Carlo factor instead of re-traced.

    ``targets``: voxel index triples (padded volume; the problem must step
    voxel by voxel) or label ints.  Returns dLoss/dmu per target."""
    targets = list(targets)
    if not 0 < len(targets) <= A.PMO_FD_MAX:
        raise ValueError(f"1..{A.PMO_FD_MAX} targets")
    by_label = all(isinstance(t, (int, np.integer)) for t in targets)
    if not by_label and dp.words is not None:
        raise ValueError("voxel targets need voxel-by-voxel stepping (skip=False)")
    host = dp.host
    tmap = np.full(host.labels.shape, -1, np.int16)
    theta = []
    for i, t in enumerate(targets):
        if by_label:
            tmap[host.labels == t] = i
            tab = host.ma if param == "ma" else host.ms
            theta.append(float(tab[t]))
        else:
            tmap[tuple(t)] = i
            if host.vox_ma is not None:
                grid = host.vox_ma if param == "ma" else host.vox_ms
                theta.append(float(grid[tuple(t)]))
            else:
                tab = host.ma if param == "ma" else host.ms
                theta.append(float(tab[int(host.labels[tuple(t)])]))
    dev = dp.device
    d_map = torch.from_numpy(tmap).to(dev)
    out = torch.zeros(2 * len(targets), dtype=torch.float64, device=dev)
    nr = fwd.spec.nr
    coef = coef.to(device=dev, dtype=torch.float32).contiguous()
    g = A.PmoGrad()
    g.coef = coef.data_ptr()
    g.nr = nr
    g.dr = float(fwd.spec.dr)
    g.score_bin = fwd.score_bin.data_ptr()
    g.score_w = fwd.score_w.data_ptr()
    nl = len(host.n)
    d_ma_l = torch.zeros(nl, dtype=torch.float64, device=dev)
    d_ms_l = torch.zeros_like(d_ma_l)
    g.d_ma_label, g.d_ms_label = d_ma_l.data_ptr(), d_ms_l.data_ptr()
    cnt = torch.zeros(A.PMO_G_COUNTERS_N, dtype=torch.int64, device=dev)
    g.counters = cnt.data_ptr()
    g.fd_target = d_map.data_ptr()
    g.fd_n = len(targets)
    g.fd_param = 0 if param == "ma" else 1
    g.fd_h = float(rel_step)
    g.fd_out = out.data_ptr()
    s = dp.struct(seed, 0, fwd.n_photons, precision)
    st = load().pmo_run_grad(C.byref(s), C.byref(g), C.byref(A.PmoLaunch(0, 0)),
                             C.c_void_p(dp.workspace.data_ptr()), dp.workspace.numel(),
                             E._stream_handle())
    check(st, "pmo_run_grad (reweighted finite difference)")
    d = out.cpu().numpy().reshape(-1, 2)
    if int(cnt.cpu()[A.PMO_G_MISMATCH]):
        raise PmoError(A.PMO_ERR_NUMERIC, "replay left the forward path")
    return (d[:, 0] - d[:, 1]) / (2 * rel_step * np.asarray(theta))
