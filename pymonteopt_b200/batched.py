"""Thousands of independent slab problems in one persistent launch.

:class:`SlabBatch` runs a batch of laterally infinite single-layer slabs (the
reference's one-layer PlateModel with x_size, y_size taken to infinity,
pymopt/voxel_gpu/_classes.py:396-459) through ``pmo_run_batched``: one
persistent kernel drains a device work queue of (problem, photon range)
items, computing in the same pass Rd, Tt, A, R(r) and their perturbation
Monte Carlo derivatives with respect to mu_a and mu_s.  The launch sequence
(clearing the sums, the kernel, the FP64 finalisation) is captured in a CUDA
graph and replayed.

:class:`StackBatch` does the same for layered slabs (PlateModel stacks of up to
``PMO_MAX_LAYERS`` layers with unbounded lateral size) through
``pmo_run_stack_batch``, with the derivatives of every output with respect to
each layer's mu_a and mu_s.

The launch shape (threads per block, photons per work item) and where the
per-problem sums gather (privatised per thread in shared memory, or straight
to global memory) are chosen by a small autotuner. It times candidates on a
down-scaled copy of the batch and caches the winner per device and batch
signature.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Optional

import numpy as np
import torch

from . import _abi as A
from . import engine as E
from ._lib import check, load

SLAB_DTYPE = np.dtype([("ma", "<f4"), ("ms", "<f4"), ("g", "<f4"), ("n_tissue", "<f4"),
                       ("n_ambient", "<f4"), ("thickness", "<f4"), ("dr", "<f4"),
                       ("photons", "<u4")])
ITEM_DTYPE = np.dtype([("problem", "<u4"), ("begin", "<u4"), ("count", "<u4")])

_TUNE_CACHE: dict = {}


def build_items(photons: np.ndarray, chunk: int, order: Optional[np.ndarray] = None) -> np.ndarray:
    """Work queue: each problem's photons in chunks of ``chunk``, problems in
    ``order`` (default: ascending budget, so small problems finish early)."""
    photons = np.asarray(photons, np.int64)
    if order is None:
        order = np.argsort(photons, kind="stable")
    counts = (photons[order] + chunk - 1) // chunk
    items = np.empty(int(counts.sum()), ITEM_DTYPE)
    prob = np.repeat(order, counts)
    first = np.repeat(np.cumsum(counts) - counts, counts)
    k = np.arange(items.size) - first
    items["problem"] = prob
    items["begin"] = k * chunk
    items["count"] = np.minimum(chunk, photons[prob] - k * chunk)
    return items


class SlabBatch:
    """A batch of slab problems resident on one GPU.

    Parameters are arrays of equal length: ``ma``, ``ms`` [1/mm], ``g``, ``n``
    (tissue index), ``thickness`` [mm], ``photons`` (budget per problem).
    ``dr`` [mm] and ``nr`` set the R(r) bins of every problem.
    """

    def __init__(self, ma, ms, g, n, thickness, photons, *, n_ambient=1.0, nr: int = 32,
                 dr=0.1, seed: int = 0, precision: int = A.PMO_FP32, device=None,
                 block_threads: int = 0, chunk: int = 0, tally_mode: Optional[int] = None,
                 autotune: bool = True):
        load()
        self.device = E.require_cuda(device)
        P = len(ma)
        slabs = np.zeros(P, SLAB_DTYPE)
        slabs["ma"], slabs["ms"], slabs["g"] = ma, ms, g
        slabs["n_tissue"] = n
        slabs["n_ambient"] = n_ambient
        slabs["thickness"] = thickness
        slabs["dr"] = dr
        slabs["photons"] = photons
        if np.any(slabs["thickness"] <= 0) or np.any(slabs["ma"] < 0) or np.any(slabs["ms"] < 0):
            raise ValueError("thickness must be positive and ma, ms non-negative")
        if np.any(slabs["photons"] < 1) or np.any(np.abs(slabs["g"]) > 1):
            raise ValueError("photon budgets must be >= 1 and |g| <= 1")
        self.host_slabs = slabs
        self.P = P
        self.nr = int(nr)
        self.seed = int(seed)
        self.precision = precision
        dev = self.device
        self.slabs = torch.from_numpy(slabs.view(np.uint8).copy()).to(dev)
        self.sums = torch.zeros(P, A.PMO_BS_N, dtype=torch.float64, device=dev)
        self.bins = torch.zeros(P, max(self.nr, 1), 3, dtype=torch.float32, device=dev)
        self.remaining = torch.zeros(P, dtype=torch.int32, device=dev)
        self.budget = torch.from_numpy(slabs["photons"].astype(np.int32)).to(dev)
        self.t_done = torch.zeros(P, dtype=torch.int64, device=dev)
        self.results = torch.zeros(P, A.PMO_BR_N, dtype=torch.float64, device=dev)
        self.rr = torch.zeros(P, max(self.nr, 1), 3, dtype=torch.float64, device=dev)
        self.workspace = torch.zeros(int(load().pmo_workspace_bytes()), dtype=torch.uint8,
                                     device=dev)
        self.graph = None
        if tally_mode not in (None, A.PMO_BT_THREAD, A.PMO_BT_GLOBAL):
            raise ValueError("tally_mode must be PMO_BT_THREAD or PMO_BT_GLOBAL")
        if autotune and not (block_threads and chunk and tally_mode is not None):
            block_threads, chunk, tally_mode = self.autotune(
                block_threads=block_threads, chunk=chunk, tally_mode=tally_mode)
        self.block_threads = block_threads or 128
        self.tally_mode = A.PMO_BT_THREAD if tally_mode is None else int(tally_mode)
        self.set_chunk(chunk or 256)

    # ------------------------------------------------------------------
    def set_chunk(self, chunk: int) -> None:
        self.chunk = int(chunk)
        items = build_items(self.host_slabs["photons"], self.chunk)
        self.items = torch.from_numpy(items.view(np.uint8).copy()).to(self.device)
        self.n_items = len(items)
        self.graph = None

    def _struct(self, slabs=None, items=None, n_items=None, sums=None, bins=None,
                remaining=None, t_done=None, P=None, tally_mode=None) -> A.PmoBatch:
        b = A.PmoBatch()
        b.slabs = (slabs if slabs is not None else self.slabs).data_ptr()
        b.n_problems = P or self.P
        b.items = (items if items is not None else self.items).data_ptr()
        b.n_items = n_items if n_items is not None else self.n_items
        b.seed = self.seed & 0xFFFFFFFFFFFFFFFF
        b.nr = self.nr
        b.sums = (sums if sums is not None else self.sums).data_ptr()
        b.bins = (bins if bins is not None else self.bins).data_ptr()
        b.remaining = (remaining if remaining is not None else self.remaining).data_ptr()
        b.t_done = (t_done if t_done is not None else self.t_done).data_ptr()
        b.precision = self.precision
        b.tally_mode = self.tally_mode if tally_mode is None else int(tally_mode)
        return b

    def launch(self, stream=None) -> None:
        """Enqueue one evaluation: clear sums, run the batch, finalise."""
        self.sums.zero_()
        self.bins.zero_()
        self.remaining.copy_(self.budget)
        self.t_done.zero_()
        b = self._struct()
        lib = load()
        st = lib.pmo_run_batched(C.byref(b), C.byref(A.PmoLaunch(self.block_threads, 0)),
                                 C.c_void_p(self.workspace.data_ptr()), self.workspace.numel(),
                                 E._stream_handle(stream))
        check(st, "pmo_run_batched")
        st = lib.pmo_batch_finalize(C.byref(b), C.c_void_p(self.results.data_ptr()),
                                    C.c_void_p(self.rr.data_ptr()) if self.nr > 0 else None,
                                    E._stream_handle(stream))
        check(st, "pmo_batch_finalize")

    def capture(self) -> "torch.cuda.CUDAGraph":
        """Capture :meth:`launch` in a CUDA graph (warms up once first)."""
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.launch()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        self.graph = g
        return g

    def run(self, use_graph: bool = True) -> dict:
        """One evaluation; returns host results (synchronises)."""
        if use_graph:
            if self.graph is None:
                self.capture()
            self.graph.replay()
        else:
            self.launch()
        return self.fetch()

    def fetch(self) -> dict:
        res = self.results.cpu().numpy()
        rr = self.rr.cpu().numpy()
        ws = self.workspace[8:16].cpu().numpy().view(np.uint64)[0]
        td = self.t_done.cpu().numpy().view(np.uint64)
        done_ms = (td.astype(np.float64) - float(ws)) / 1e6
        return {
            "Rd": res[:, A.PMO_BR_RD], "Tt": res[:, A.PMO_BR_TT], "A": res[:, A.PMO_BR_A],
            "dRd_dma": res[:, A.PMO_BR_DRD_DMA], "dRd_dms": res[:, A.PMO_BR_DRD_DMS],
            "dTt_dma": res[:, A.PMO_BR_DTT_DMA], "dTt_dms": res[:, A.PMO_BR_DTT_DMS],
            "balance": res[:, A.PMO_BR_BALANCE],
            "Rr": rr[:, :, 0], "dRr_dma": rr[:, :, 1], "dRr_dms": rr[:, :, 2],
            "completion_ms": done_ms,
            "sums": self.sums.cpu().numpy(),
        }

    # ------------------------------------------------------------------
    def autotune(self, candidates=None, scale: float = 1 / 64, mode_scale: float = 1 / 8,
                 block_threads: int = 0, chunk: int = 0,
                 tally_mode: Optional[int] = None) -> tuple:
        """Pick (threads per block, photons per work item, tally mode).

        The shapes are timed with per-thread privatised sums on the batch with
        every budget scaled by ``scale``.  The tally modes are then timed on
        the best shape at ``mode_scale``: contention on one problem's sums
        grows with the photons of that problem in flight at once, so the
        comparison needs budgets closer to the real ones (measured on C5:
        equal at 1/64, 1.3 % apart at 1/8, global atomics 25 % slower at
        full size).  Arguments
        that are set (non-zero, not None) are kept as given."""
        sig = (torch.cuda.get_device_name(self.device), self.P,
               int(self.host_slabs["photons"].sum()), round(float(self.host_slabs["ma"].mean()), 6),
               block_threads, chunk, tally_mode)
        if sig in _TUNE_CACHE:
            self.tune_table = _TUNE_CACHE[sig]
            return self.tune_table["best"]
        if candidates is None:
            candidates = [(t, c) for t in ((block_threads,) if block_threads else (64, 128, 256))
                          for c in ((chunk,) if chunk else (64, 512, 4096))]
        modes = (tally_mode,) if tally_mode is not None else (A.PMO_BT_THREAD, A.PMO_BT_GLOBAL)
        dev = self.device
        sums = torch.zeros_like(self.sums)
        bins = torch.zeros_like(self.bins)
        rem = torch.zeros_like(self.remaining)
        tdone = torch.zeros_like(self.t_done)
        lib = load()

        def scaled(f):
            small = self.host_slabs.copy()
            small["photons"] = np.maximum(1, (small["photons"] * f).astype(np.int64))
            return small["photons"], torch.from_numpy(small.view(np.uint8).copy()).to(dev)

        def timed(photons, slabs, threads, chunk, mode):
            items = build_items(photons, chunk)
            d_items = torch.from_numpy(items.view(np.uint8).copy()).to(dev)
            b = self._struct(slabs=slabs, items=d_items, n_items=len(items), sums=sums,
                             bins=bins, remaining=rem, t_done=tdone, tally_mode=mode)
            times = []
            for rep in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                st = lib.pmo_run_batched(C.byref(b), C.byref(A.PmoLaunch(threads, 0)),
                                         C.c_void_p(self.workspace.data_ptr()),
                                         self.workspace.numel(), E._stream_handle())
                e1.record()
                check(st, "pmo_run_batched (autotune)")
                torch.cuda.synchronize()
                if rep:
                    times.append(e0.elapsed_time(e1))
            return min(times)

        small = scaled(scale)
        shapes = {(t, c): timed(*small, t, c, modes[0]) for t, c in candidates}
        shape = min(shapes, key=shapes.get)
        if len(modes) > 1:
            mid = scaled(mode_scale)
            by_mode = {m: timed(*mid, *shape, m) for m in modes}
        else:
            by_mode = {modes[0]: shapes[shape]}
        # contention only grows with the budgets, so the down-scaled timing
        # flatters global atomics (on C5: 1-3 % ahead at 1/8, 25 % behind at
        # full size): they must win by 10 % to be kept
        mode = modes[0]
        if len(modes) > 1 and by_mode[A.PMO_BT_GLOBAL] < 0.90 * by_mode[A.PMO_BT_THREAD]:
            mode = A.PMO_BT_GLOBAL
        best = (*shape, mode)
        self.tune_table = {"best": best, "shape_ms": {str(k): v for k, v in shapes.items()},
                           "mode_ms": {("thread" if m == A.PMO_BT_THREAD else "global"): v
                                       for m, v in by_mode.items()}}
        _TUNE_CACHE[sig] = self.tune_table
        return best


LAYER_DTYPE = np.dtype([("ma", "<f4"), ("ms", "<f4"), ("g", "<f4"), ("n", "<f4"),
                        ("thickness", "<f4")])
STACK_DTYPE = np.dtype([("first_layer", "<u4"), ("n_layers", "<u4"), ("n_ambient", "<f4"),
                        ("dr", "<f4"), ("photons", "<u4")])


class StackBatch:
    """A batch of layered slab problems resident on one GPU: PlateModel stacks
    (pymopt/voxel_gpu/_classes.py:396-459) with unbounded lateral size, run by
    ``pmo_run_stack_batch`` in one persistent launch with forward and
    per-layer gradient together.

    ``stacks``: one sequence of layers per problem, top layer first, each
    layer ``(ma, ms, g, n, thickness)`` [1/mm, 1/mm, -, -, mm], at most
    ``PMO_MAX_LAYERS`` layers; ``photons``: budget per problem;
    ``n_ambient``: scalar or per problem.  ``dr`` [mm] and ``nr`` set the R(r)
    bins of every problem.  A stack of one layer follows the photons of
    :class:`SlabBatch` on the same seed.
    """

    def __init__(self, stacks, photons, *, n_ambient=1.0, nr: int = 32, dr: float = 0.1,
                 seed: int = 0, precision: int = A.PMO_FP32, device=None,
                 block_threads: int = 0, chunk: int = 0, autotune: bool = False):
        load()
        self.device = E.require_cuda(device)
        P = len(stacks)
        photons = np.broadcast_to(np.asarray(photons, np.int64), (P,))
        n_amb = np.broadcast_to(np.asarray(n_ambient, np.float32), (P,))
        rows = []
        st = np.zeros(P, STACK_DTYPE)
        for i, layers in enumerate(stacks):
            layers = [tuple(float(v) for v in L) for L in layers]
            if not 1 <= len(layers) <= A.PMO_MAX_LAYERS:
                raise ValueError(f"problem {i}: 1 to {A.PMO_MAX_LAYERS} layers")
            for ma, ms, g, n, t in layers:
                if not (t > 0 and ma >= 0 and ms >= 0 and abs(g) <= 1 and n > 0):
                    raise ValueError(f"problem {i}: thickness > 0, ma, ms >= 0, |g| <= 1, n > 0")
            st[i] = (len(rows), len(layers), n_amb[i], dr, photons[i])
            rows.extend(layers)
        if np.any(photons < 1) or np.any(photons >= 2**32):
            raise ValueError("photon budgets must lie in [1, 2^32)")
        table = np.array(rows, LAYER_DTYPE)
        self.host_stacks, self.host_layers = st, table
        self.n_layers = st["n_layers"].astype(int)
        self.P = P
        self.nr = int(nr)
        self.seed = int(seed)
        self.precision = precision
        dev = self.device
        self.stacks = torch.from_numpy(st.view(np.uint8).copy()).to(dev)
        self.layers = torch.from_numpy(table.view(np.uint8).copy()).to(dev)
        self.sums = torch.zeros(P, A.PMO_SS_N, dtype=torch.float64, device=dev)
        self.bins = torch.zeros(P, max(self.nr, 1), A.PMO_SB_N, dtype=torch.float32, device=dev)
        self.remaining = torch.zeros(P, dtype=torch.int32, device=dev)
        self.budget = torch.from_numpy(photons.astype(np.int32)).to(dev)
        self.t_done = torch.zeros(P, dtype=torch.int64, device=dev)
        self.results = torch.zeros(P, A.PMO_SR_N, dtype=torch.float64, device=dev)
        self.rr = torch.zeros(P, max(self.nr, 1), A.PMO_SB_N, dtype=torch.float64, device=dev)
        self.workspace = torch.zeros(int(load().pmo_workspace_bytes()), dtype=torch.uint8,
                                     device=dev)
        self.photons = photons
        self.graph = None
        if autotune and not (block_threads and chunk):
            block_threads, chunk = self.autotune(block_threads=block_threads, chunk=chunk)
        self.block_threads = int(block_threads or 128)
        self.set_chunk(chunk or 256)

    def set_chunk(self, chunk: int) -> None:
        self.chunk = int(chunk)
        items = build_items(self.photons, self.chunk)
        self.items = torch.from_numpy(items.view(np.uint8).copy()).to(self.device)
        self.n_items = len(items)
        self.graph = None

    def autotune(self, scale: float = 1 / 16, block_threads: int = 0, chunk: int = 0) -> tuple:
        """Pick (threads per block, photons per work item) by timing the
        candidates (64, 128, 256) x (64, 256, 1024) on a copy of the batch
        with every budget scaled by ``scale``; cached per device and batch
        signature.  Arguments that are set (non-zero) are kept as given."""
        sig = ("stack", torch.cuda.get_device_name(self.device), self.P,
               int(self.photons.sum()), len(self.host_layers),
               round(float(self.host_layers["ma"].mean()), 6), block_threads, chunk)
        if sig in _TUNE_CACHE:
            self.tune_table = _TUNE_CACHE[sig]
            return self.tune_table["best"]
        cands = [(t, c) for t in ((block_threads,) if block_threads else (64, 128, 256))
                 for c in ((chunk,) if chunk else (64, 256, 1024))]
        small = np.maximum(1, (self.photons * scale).astype(np.int64))
        st = self.host_stacks.copy()
        st["photons"] = small
        d_st = torch.from_numpy(st.view(np.uint8).copy()).to(self.device)
        lib = load()
        times = {}
        for t, c in cands:
            items = build_items(small, c)
            d_items = torch.from_numpy(items.view(np.uint8).copy()).to(self.device)
            b = self._struct(stacks=d_st, items=d_items, n_items=len(items))
            best = float("inf")
            for rep in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                check(lib.pmo_run_stack_batch(C.byref(b), C.byref(A.PmoLaunch(t, 0)),
                                              C.c_void_p(self.workspace.data_ptr()),
                                              self.workspace.numel(), E._stream_handle()),
                      "pmo_run_stack_batch (autotune)")
                e1.record()
                torch.cuda.synchronize()
                if rep:
                    best = min(best, e0.elapsed_time(e1))
            times[(t, c)] = best
        choice = min(times, key=times.get)
        self.tune_table = {"best": choice, "ms": {f"{t}x{c}": v for (t, c), v in times.items()},
                           "scale": scale}
        _TUNE_CACHE[sig] = self.tune_table
        return choice

    def _struct(self, stacks=None, items=None, n_items=None) -> A.PmoStackBatch:
        b = A.PmoStackBatch()
        b.stacks = (stacks if stacks is not None else self.stacks).data_ptr()
        b.n_problems = self.P
        b.layers, b.n_layer_rows = self.layers.data_ptr(), len(self.host_layers)
        b.items = (items if items is not None else self.items).data_ptr()
        b.n_items = n_items if n_items is not None else self.n_items
        b.seed = self.seed & 0xFFFFFFFFFFFFFFFF
        b.nr = self.nr
        b.sums, b.bins = self.sums.data_ptr(), self.bins.data_ptr()
        b.remaining, b.t_done = self.remaining.data_ptr(), self.t_done.data_ptr()
        b.precision = self.precision
        return b

    def launch(self, stream=None) -> None:
        """Enqueue one evaluation: clear sums, run the batch, finalise."""
        self.sums.zero_()
        self.bins.zero_()
        self.remaining.copy_(self.budget)
        self.t_done.zero_()
        b = self._struct()
        lib = load()
        check(lib.pmo_run_stack_batch(C.byref(b), C.byref(A.PmoLaunch(self.block_threads, 0)),
                                      C.c_void_p(self.workspace.data_ptr()),
                                      self.workspace.numel(), E._stream_handle(stream)),
              "pmo_run_stack_batch")
        check(lib.pmo_stack_batch_finalize(
            C.byref(b), C.c_void_p(self.results.data_ptr()),
            C.c_void_p(self.rr.data_ptr()) if self.nr > 0 else None, E._stream_handle(stream)),
            "pmo_stack_batch_finalize")

    def capture(self) -> "torch.cuda.CUDAGraph":
        """Capture :meth:`launch` in a CUDA graph (warms up once first)."""
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.launch()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        self.graph = g
        return g

    def run(self, use_graph: bool = True) -> dict:
        """One evaluation; returns host results (synchronises)."""
        if use_graph:
            if self.graph is None:
                self.capture()
            self.graph.replay()
        else:
            self.launch()
        return self.fetch()

    def fetch(self) -> dict:
        res = self.results.cpu().numpy()
        rr = self.rr.cpu().numpy()
        ws = self.workspace[8:16].cpu().numpy().view(np.uint64)[0]
        td = self.t_done.cpu().numpy().view(np.uint64)
        K = A.PMO_MAX_LAYERS
        lay = res[:, A.PMO_SR_LAYER0:A.PMO_SR_LAYER0 + 4 * K].reshape(self.P, K, 4)
        return {
            "Rd": res[:, A.PMO_SR_RD], "Tt": res[:, A.PMO_SR_TT], "A": res[:, A.PMO_SR_A],
            "balance": res[:, A.PMO_SR_BALANCE],
            # per problem and layer (layers beyond a problem's own are 0)
            "dRd_dma": lay[:, :, 0], "dRd_dms": lay[:, :, 1],
            "dTt_dma": lay[:, :, 2], "dTt_dms": lay[:, :, 3],
            "Rr": rr[:, :, 0], "dRr_dma": rr[:, :, 1::2][:, :, :K],
            "dRr_dms": rr[:, :, 2::2][:, :, :K],
            "completion_ms": (td.astype(np.float64) - float(ws)) / 1e6,
            "sums": self.sums.cpu().numpy(), "n_layers": self.n_layers,
        }


def time_batch(batch: SlabBatch, reps: int = 3) -> dict:
    """Wall and device time of graph replays of the batch."""
    if batch.graph is None:
        batch.capture()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.graph.replay()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    return {"seconds": min(times), "evals_per_s": batch.P / min(times)}


def voxel_slab_problem(ma, ms, g, n, thickness, n_ambient=1.0, half: int = 60):
    """One slab as the reference builds it with PlateModel: one z voxel of the
    slab's thickness, 2*half+1 lateral voxels, end-label shell."""
    from .problem import pencil_problem
    k = 2 * half + 1
    vol = np.ones((k + 2, k + 2, 3), np.uint8)
    vol[1:-1, 1:-1, 1] = 0
    return pencil_problem(vol, float(thickness), 1, [ma], [ms], [g], [n, n_ambient])


def plain_eval(ma, ms, g, n, thickness, photons, *, nr=32, dr=0.1, seed=0, device=None) -> dict:
    """One forward + gradient evaluation of one slab through the per-problem
    API (upload, scored forward run, gradient replay): the path the batched
    form replaces."""
    from . import grad as G
    prob = voxel_slab_problem(ma, ms, g, n, thickness)
    dp = E.DeviceProblem(prob, device)
    fwd = G.run_forward_scored(dp, int(photons), seed, nr, dr)
    area = torch.tensor(G.annulus_area(nr, dr), dtype=torch.float64, device=dp.device)
    coef = torch.zeros(A.PMO_RR_CATS, nr, dtype=torch.float32, device=dp.device)
    coef[A.PMO_RR_TOP] = (1.0 / (area * photons)).float()
    coef[A.PMO_RR_LAT_NEG] = coef[A.PMO_RR_TOP]
    rep = G.run_replay(dp, fwd, coef, seed, per_voxel=False)
    L = fwd.ledger.cpu().numpy()
    return {"Rd": L[A.PMO_L_RD] / photons, "dR_dma": float(rep.d_ma_label[0]),
            "dR_dms": float(rep.d_ms_label[0])}


class PlainSlabEvaluator:
    """Forward + gradient of one slab at a time through the per-problem plain
    API with every device buffer reused: the fastest way to run C5's problems
    one by one.

    Every slab is the same label volume (one z voxel whose size is the slab's
    thickness, see :func:`voxel_slab_problem`), so one resident
    :class:`~pymonteopt_b200.engine.DeviceProblem` with its box map serves all
    of them.  Per problem only the optical tables are rewritten (four small
    host-to-device copies) and the voxel size and entry weight change in the
    launch parameters; the tallies, score record, gradient sums and counters
    are preallocated for the largest budget.  Each evaluation runs the scored
    forward transport (``pmo_run_plain``) and the Philox replay
    (``pmo_run_grad``) and reads Rd and the two per-label derivatives back."""

    def __init__(self, max_photons: int, nr: int = 32, dr: float = 0.1, device=None):
        self.dp = E.DeviceProblem(voxel_slab_problem(0.1, 10.0, 0.9, 1.4, 1.0), device)
        dev = self.dp.device
        self.nr, self.dr = int(nr), float(dr)
        self.tal = E.Tallies(self.dp, E.TallySpec(nr=nr, dr=dr), 0)
        self.score_bin = torch.empty(int(max_photons), dtype=torch.int32, device=dev)
        self.score_w = torch.empty(int(max_photons), dtype=torch.float32, device=dev)
        # loss weights: R(r) of the exits with v_z < 0 per unit bin weight;
        # the 1/nPh of the estimator is applied to the read-back sums
        area = torch.tensor(annulus_area_mm2(nr, dr), dtype=torch.float64, device=dev)
        self.coef = torch.zeros(A.PMO_RR_CATS, nr, dtype=torch.float32, device=dev)
        self.coef[A.PMO_RR_TOP] = (1.0 / area).float()
        self.coef[A.PMO_RR_LAT_NEG] = self.coef[A.PMO_RR_TOP]
        self.grad_sums = torch.zeros(2, len(self.dp.host.n), dtype=torch.float64, device=dev)
        self.gcnt = torch.zeros(A.PMO_G_COUNTERS_N, dtype=torch.int64, device=dev)
        self.max_photons = int(max_photons)

    def evaluate(self, ma, ms, g, n, thickness, photons: int, seed: int) -> dict:
        photons = int(photons)
        if photons > self.max_photons:
            raise ValueError("more photons than the evaluator was sized for")
        lib = load()
        dp = self.dp
        dp.host = voxel_slab_problem(ma, ms, g, n, thickness)   # host fields only
        for dst, val in ((dp.ma, ma), (dp.ms, ms), (dp.g, g)):
            dst[:1].copy_(torch.tensor([val], dtype=torch.float32), non_blocking=True)
        dp.n.copy_(torch.tensor([n, 1.0], dtype=torch.float32), non_blocking=True)
        self.tal.zero_()
        self.grad_sums.zero_()
        self.gcnt.zero_()
        stream = E._stream_handle()
        s = dp.struct(seed, 0, photons, A.PMO_FP32, A.PMO_FLAG_SCORE_RECORD)
        ts = self.tal.struct()
        ts.score_bin = self.score_bin.data_ptr()
        ts.score_w = self.score_w.data_ptr()
        launch = A.PmoLaunch(0, 0)
        ws = C.c_void_p(dp.workspace.data_ptr())
        check(lib.pmo_run_plain(C.byref(s), C.byref(ts), C.byref(launch), ws,
                                dp.workspace.numel(), stream), "pmo_run_plain (scored)")
        gr = A.PmoGrad()
        gr.coef = self.coef.data_ptr()
        gr.nr, gr.dr = self.nr, self.dr
        gr.score_bin, gr.score_w = self.score_bin.data_ptr(), self.score_w.data_ptr()
        gr.d_ma_label = self.grad_sums[0].data_ptr()
        gr.d_ms_label = self.grad_sums[1].data_ptr()
        gr.counters = self.gcnt.data_ptr()
        s = dp.struct(seed, 0, photons, A.PMO_FP32)
        check(lib.pmo_run_grad(C.byref(s), C.byref(gr), C.byref(launch), ws,
                               dp.workspace.numel(), stream), "pmo_run_grad")
        led = self.tal.ledger.cpu().numpy()          # synchronises
        gs = self.grad_sums[:, 0].cpu().numpy() / photons
        return {"Rd": led[A.PMO_L_RD] / photons, "dR_dma": float(gs[0]),
                "dR_dms": float(gs[1])}


def annulus_area_mm2(nr: int, dr: float) -> np.ndarray:
    """2 pi (i + 1/2) dr^2 (pymopt/metrics/_scoring.py:18)."""
    return np.array([2 * np.pi * (i + 0.5) * dr ** 2 for i in range(nr)])


def batched_vs_plain(count: int = 4096, plain_sample: int = 48, seed: int = 0, nr: int = 32,
                     dr: float = 0.1, device=None) -> dict:
    """C5: ``count`` slabs with log-uniform budgets in one graph-captured
    persistent launch (forward + gradient), against per-problem plain
    evaluations of a random sample of the same problems."""
    from . import volumes as V
    b = V.c5_slab_batch(seed=seed, count=count)
    t0 = time.perf_counter()
    sb = SlabBatch(b["ma"], b["ms"], b["g"], b["n"], b["thickness"], b["n_photons"], nr=nr,
                   dr=dr, seed=seed + 1, device=device)
    tune_s = time.perf_counter() - t0
    sb.capture()
    tb = time_batch(sb, reps=2)
    res = sb.fetch()
    comp = res["completion_ms"]
    rng = np.random.default_rng(seed + 7)
    pick = rng.choice(count, size=min(plain_sample, count), replace=False)
    # per-problem plain API, every buffer reused (the comparator of record)
    ev = PlainSlabEvaluator(int(b["n_photons"].max()), nr=nr, dr=dr, device=device)
    for i in pick[:2]:                                  # warm-up
        ev.evaluate(b["ma"][i], b["ms"][i], b["g"][i], b["n"][i], b["thickness"][i],
                    1000, seed + 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in pick:
        ev.evaluate(b["ma"][i], b["ms"][i], b["g"][i], b["n"][i], b["thickness"][i],
                    int(b["n_photons"][i]), seed + 1)
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    plain_rate = len(pick) / plain_s
    # the same with a fresh upload per problem (plain_eval)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in pick:
        plain_eval(b["ma"][i], b["ms"][i], b["g"][i], b["n"][i], b["thickness"][i],
                   int(b["n_photons"][i]), nr=nr, dr=dr, seed=seed + 1, device=device)
    torch.cuda.synchronize()
    fresh_rate = len(pick) / (time.perf_counter() - t0)
    # the same slab kernel launched once per problem (no batching, no graph)
    singles = [SlabBatch([b["ma"][i]], [b["ms"][i]], [b["g"][i]], [b["n"][i]],
                         [b["thickness"][i]], [int(b["n_photons"][i])], nr=nr, dr=dr,
                         seed=seed + 1, device=device, autotune=False,
                         block_threads=sb.block_threads, chunk=sb.chunk,
                         tally_mode=sb.tally_mode) for i in pick]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for one in singles:
        one.launch()
        one.results.cpu()
    torch.cuda.synchronize()
    single_rate = len(pick) / (time.perf_counter() - t0)
    photons = float(b["n_photons"].sum())
    return {
        "problems": count,
        "photons": photons,
        "batched_seconds": tb["seconds"],
        "batched_evals_per_s": tb["evals_per_s"],
        "batched_photons_per_s": photons / tb["seconds"],
        "plain_evals_per_s": plain_rate,
        "plain_path": "PlainSlabEvaluator: one resident volume, tables rewritten per problem, "
                      "scored forward + replay + read-back per problem",
        "plain_sample": len(pick),
        "ratio": tb["evals_per_s"] / plain_rate,
        "plain_fresh_upload_evals_per_s": fresh_rate,
        "ratio_vs_fresh_upload": tb["evals_per_s"] / fresh_rate,
        "single_launch_evals_per_s": single_rate,
        "ratio_vs_single_launches": tb["evals_per_s"] / single_rate,
        "p50_completion_ms": float(np.percentile(comp, 50)),
        "p99_completion_ms": float(np.percentile(comp, 99)),
        "launch_shape": {"block_threads": sb.block_threads, "photons_per_item": sb.chunk,
                         "tally_mode": "thread" if sb.tally_mode == A.PMO_BT_THREAD
                         else "global"},
        "autotune_seconds": tune_s,
        "max_energy_residual": float(np.max(np.abs(res["balance"]))),
    }


class PlainStackEvaluator:
    """Forward + per-layer gradient of one skin stack at a time through the
    per-problem plain API with every buffer reused: the comparator of the
    layered batch.  All problems of the sweep share the layer thicknesses, so
    one resident voxel plate (20 x 20 mm, 0.05 mm voxels, its box map built
    once) serves them all; per problem the three layers' mu_a and mu_s are
    copied in, then the scored forward run and the per-label replay run and
    Rd and its six derivatives are read back."""

    def __init__(self, layers, max_photons: int, nr: int = 32, dr: float = 0.1, device=None,
                 lateral_mm: float = 20.0, voxel_mm: float = 0.05):
        from . import volumes as V
        prob = V.plate_problem(dict(x_size=lateral_mm, y_size=lateral_mm, voxel_space=voxel_mm,
                                    thickness=[L[4] for L in layers], n=[L[3] for L in layers],
                                    n_air=1.0, ma=[L[0] for L in layers],
                                    ms=[L[1] for L in layers], g=[L[2] for L in layers]))
        self.nl = len(layers)
        self.dp = E.DeviceProblem(prob, device)
        dev = self.dp.device
        self.nr, self.dr = int(nr), float(dr)
        self.tal = E.Tallies(self.dp, E.TallySpec(nr=nr, dr=dr), 0)
        self.score_bin = torch.empty(int(max_photons), dtype=torch.int32, device=dev)
        self.score_w = torch.empty(int(max_photons), dtype=torch.float32, device=dev)
        area = torch.tensor(annulus_area_mm2(nr, dr), dtype=torch.float64, device=dev)
        self.coef = torch.zeros(A.PMO_RR_CATS, nr, dtype=torch.float32, device=dev)
        self.coef[A.PMO_RR_TOP] = (1.0 / area).float()
        self.coef[A.PMO_RR_LAT_NEG] = self.coef[A.PMO_RR_TOP]
        self.grad_sums = torch.zeros(2, len(self.dp.host.n), dtype=torch.float64, device=dev)
        self.gcnt = torch.zeros(A.PMO_G_COUNTERS_N, dtype=torch.int64, device=dev)
        self.tabs = torch.zeros(2, len(self.dp.host.n), dtype=torch.float32)
        self.max_photons = int(max_photons)

    def evaluate(self, layers, photons: int, seed: int) -> dict:
        photons = int(photons)
        lib = load()
        dp = self.dp
        for i, L in enumerate(layers):
            self.tabs[0, i], self.tabs[1, i] = float(L[0]), float(L[1])
        dp.ma.copy_(self.tabs[0], non_blocking=True)
        dp.ms.copy_(self.tabs[1], non_blocking=True)
        self.tal.zero_()
        self.grad_sums.zero_()
        self.gcnt.zero_()
        stream = E._stream_handle()
        launch = A.PmoLaunch(0, 0)
        ws = C.c_void_p(dp.workspace.data_ptr())
        s = dp.struct(seed, 0, photons, A.PMO_FP32, A.PMO_FLAG_SCORE_RECORD)
        ts = self.tal.struct()
        ts.score_bin, ts.score_w = self.score_bin.data_ptr(), self.score_w.data_ptr()
        check(lib.pmo_run_plain(C.byref(s), C.byref(ts), C.byref(launch), ws,
                                dp.workspace.numel(), stream), "pmo_run_plain (scored)")
        gr = A.PmoGrad()
        gr.coef = self.coef.data_ptr()
        gr.nr, gr.dr = self.nr, self.dr
        gr.score_bin, gr.score_w = self.score_bin.data_ptr(), self.score_w.data_ptr()
        gr.d_ma_label = self.grad_sums[0].data_ptr()
        gr.d_ms_label = self.grad_sums[1].data_ptr()
        gr.counters = self.gcnt.data_ptr()
        s = dp.struct(seed, 0, photons, A.PMO_FP32)
        check(lib.pmo_run_grad(C.byref(s), C.byref(gr), C.byref(launch), ws,
                               dp.workspace.numel(), stream), "pmo_run_grad")
        led = self.tal.ledger.cpu().numpy()          # synchronises
        g = self.grad_sums[:, :self.nl].cpu().numpy() / photons
        return {"Rd": led[A.PMO_L_RD] / photons, "dR_dma": g[0], "dR_dms": g[1]}


def stacks_vs_plain(count: int = 1024, plain_sample: int = 48, seed: int = 0, nr: int = 32,
                    dr: float = 0.1, device=None) -> dict:
    """The layered batch on a skin sweep (volumes.skin_stack_sweep): ``count``
    three-layer stacks, forward + per-layer gradient in one graph-captured
    launch, against the per-problem plain path with reused buffers on a
    random sample of the same problems."""
    from . import volumes as V
    sw = V.skin_stack_sweep(seed=seed, count=count)
    stacks, photons = sw["stacks"], sw["n_photons"]
    t0 = time.perf_counter()
    sb = StackBatch(stacks, photons, nr=nr, dr=dr, seed=seed + 1, device=device, autotune=True)
    tune_s = time.perf_counter() - t0
    sb.capture()
    tb = time_batch(sb, reps=3)
    res = sb.fetch()
    comp = res["completion_ms"]
    rng = np.random.default_rng(seed + 11)
    pick = rng.choice(count, size=min(plain_sample, count), replace=False)
    ev = PlainStackEvaluator(V.SKIN_LAYERS, int(photons.max()), nr=nr, dr=dr, device=device)
    for i in pick[:2]:
        ev.evaluate(stacks[i], 1000, seed + 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in pick:
        ev.evaluate(stacks[i], int(photons[i]), seed + 1)
    torch.cuda.synchronize()
    plain_rate = len(pick) / (time.perf_counter() - t0)
    total = float(photons.sum())
    return {
        "problems": count, "layers_per_problem": 3, "photons": total,
        "batched_seconds": tb["seconds"], "batched_evals_per_s": tb["evals_per_s"],
        "batched_photons_per_s": total / tb["seconds"],
        "plain_evals_per_s": plain_rate,
        "plain_path": "PlainStackEvaluator: one resident 20 x 20 mm plate at 0.05 mm, optics "
                      "rewritten per problem, scored forward + per-label replay + read-back",
        "launch_shape": {"block_threads": sb.block_threads, "photons_per_item": sb.chunk},
        "autotune_seconds": tune_s,
        "plain_sample": len(pick), "ratio": tb["evals_per_s"] / plain_rate,
        "p50_completion_ms": float(np.percentile(comp, 50)),
        "p99_completion_ms": float(np.percentile(comp, 99)),
        "max_energy_residual": float(np.max(np.abs(res["balance"]))),
    }


def main(argv=None) -> int:
    """``python -m pymonteopt_b200.batched``: time graph replays of the C5
    slab batch (forward + gradient), or with ``--stacks`` of the layered skin
    sweep, and print one JSON line."""
    import argparse
    import json
    from . import volumes as V
    ap = argparse.ArgumentParser(description=main.__doc__.split("\n")[0])
    ap.add_argument("--count", type=int, default=4096, help="slab problems")
    ap.add_argument("--photon-scale", type=float, default=1.0,
                    help="multiplies every photon budget")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--block-threads", type=int, default=0)
    ap.add_argument("--chunk", type=int, default=0, help="photons per work item")
    ap.add_argument("--tally-mode", choices=["auto", "thread", "global"], default="auto",
                    help="per-problem sums privatised per thread, or straight to global memory")
    ap.add_argument("--stacks", action="store_true",
                    help="the layered batch on the skin sweep (volumes.skin_stack_sweep) instead")
    args = ap.parse_args(argv)
    if args.stacks:
        sw = V.skin_stack_sweep(seed=0, count=args.count)
        photons = np.maximum(1, (sw["n_photons"] * args.photon_scale).astype(np.int64))
        st = StackBatch(sw["stacks"], photons, nr=32, dr=0.1, seed=1,
                        block_threads=args.block_threads, chunk=args.chunk, autotune=True)
        tb = time_batch(st, reps=args.reps)
        res = st.fetch()
        print(json.dumps({"problems": st.P, "layers_per_problem": 3,
                          "photons": float(photons.sum()), "seconds": tb["seconds"],
                          "evals_per_s": tb["evals_per_s"],
                          "photons_per_s": float(photons.sum()) / tb["seconds"],
                          "block_threads": st.block_threads, "photons_per_item": st.chunk,
                          "autotune": getattr(st, "tune_table", None),
                          "p99_completion_ms": float(np.percentile(res["completion_ms"], 99)),
                          "max_energy_residual": float(np.max(np.abs(res["balance"])))}))
        return 0
    b = V.c5_slab_batch(seed=0, count=args.count)
    photons = np.maximum(1, (b["n_photons"] * args.photon_scale).astype(np.int64))
    mode = {"auto": None, "thread": A.PMO_BT_THREAD, "global": A.PMO_BT_GLOBAL}[args.tally_mode]
    sb = SlabBatch(b["ma"], b["ms"], b["g"], b["n"], b["thickness"], photons, nr=32, dr=0.1,
                   seed=1, block_threads=args.block_threads, chunk=args.chunk, tally_mode=mode)
    tb = time_batch(sb, reps=args.reps)
    res = sb.fetch()
    print(json.dumps({"problems": sb.P, "photons": float(photons.sum()),
                      "seconds": tb["seconds"], "evals_per_s": tb["evals_per_s"],
                      "photons_per_s": float(photons.sum()) / tb["seconds"],
                      "block_threads": sb.block_threads, "photons_per_item": sb.chunk,
                      "tally_mode": "thread" if sb.tally_mode == A.PMO_BT_THREAD else "global",
                      "autotune": getattr(sb, "tune_table", None),
                      "p50_completion_ms": float(np.percentile(res["completion_ms"], 50)),
                      "p99_completion_ms": float(np.percentile(res["completion_ms"], 99)),
                      "max_energy_residual": float(np.max(np.abs(res["balance"])))}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
