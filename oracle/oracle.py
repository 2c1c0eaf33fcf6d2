"""Python driver for the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only to check or to time the CPU
restatement; the product package never imports it.

:func:`run` traces photons ``[begin, begin + n)`` of a
:class:`pymonteopt_b200.problem.TransportProblem` with the C restatement in
``vmc_oracle.c`` and returns host tallies with the same meaning as the device
ones (ledger, counters, R(r) histograms, absorbed-weight grid) plus optional
per-photon final states and event counts.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))

from pymonteopt_b200 import _abi as A  # noqa: E402

_LIB = None


class OracleTallies(C.Structure):
    _fields_ = [
        ("ledger", C.c_double * A.PMO_LEDGER_N),
        ("counters", C.c_ulonglong * A.PMO_COUNTERS_N),
        ("rr", C.c_void_p),
        ("nr", C.c_int32),
        ("dr", C.c_double),
        ("absorbed", C.c_void_p),
        ("ph_state", C.c_void_p),
        ("ph_counts", C.c_void_p),
        ("grad_coef", C.c_void_p),
        ("g_ma_voxel", C.c_void_p), ("g_ms_voxel", C.c_void_p),
        ("g_ma_label", C.c_void_p), ("g_ms_label", C.c_void_p),
    ]


def load():
    global _LIB
    if _LIB is None:
        sys.path.insert(0, HERE)
        try:
            import build as _b  # oracle/build.py
        finally:
            sys.path.pop(0)
        path = _b.build()
        lib = C.CDLL(path)
        lib.oracle_run.argtypes = [C.POINTER(A.PmoProblem), C.POINTER(OracleTallies), C.c_int]
        lib.oracle_run.restype = C.c_int
        lib.oracle_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        lib.oracle_philox.restype = None
        lib.oracle_tallies_size.restype = C.c_size_t
        assert lib.oracle_tallies_size() == C.sizeof(OracleTallies)
        _LIB = lib
    return _LIB


def philox(ctr: np.ndarray, key) -> np.ndarray:
    """Philox4x32-10 words for counters ``ctr`` (n, 4) uint32 and a 2-word key."""
    lib = load()
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    k = np.ascontiguousarray(np.asarray(key, np.uint32).reshape(2))
    out = np.zeros_like(ctr)
    lib.oracle_philox(ctr.ctypes.data, k.ctypes.data, out.ctypes.data, ctr.shape[0])
    return out


def _ptr(a):
    return None if a is None else a.ctypes.data


def run(prob, n_photons: int, seed: int, *, begin: int = 0, precision: int = A.PMO_FP64,
        nr: int = 0, dr: float = 0.1, fluence: bool = False, per_photon: bool = False,
        threads: int = 0, max_events: int = 0, validate: bool = True,
        grad_coef=None) -> dict:
    """Trace photons ``[begin, begin + n_photons)`` of ``prob`` on the CPU.

    ``grad_coef`` ([PMO_RR_CATS, nr] dLoss/d(bin weight sum)) also returns the
    perturbation Monte Carlo derivatives per voxel and per label
    (``g_ma_voxel``, ``g_ms_voxel``, ``g_ma_label``, ``g_ms_label``)."""
    lib = load()
    if validate:
        prob.validate()
    s = A.PmoProblem()
    prob.fill_struct(s)
    keep = [prob.labels, prob.ma, prob.ms, prob.g, prob.n]
    s.labels = prob.labels.ctypes.data
    s.ma, s.ms, s.g, s.n = (a.ctypes.data for a in (prob.ma, prob.ms, prob.g, prob.n))
    if prob.vox_ma is not None:
        s.vox_ma, s.vox_ms = prob.vox_ma.ctypes.data, prob.vox_ms.ctypes.data
        keep += [prob.vox_ma, prob.vox_ms]
    if prob.source == A.PMO_SRC_STATE:
        st = [np.ascontiguousarray(prob.state_add, np.int32),
              np.ascontiguousarray(prob.state_p, np.float32),
              np.ascontiguousarray(prob.state_v, np.float32),
              np.ascontiguousarray(prob.state_w, np.float32)]
        keep += st
        s.state_add, s.state_p, s.state_v, s.state_w = (a.ctypes.data for a in st)
    s.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    s.photon_begin = int(begin)
    s.photon_count = int(n_photons)
    s.max_events = int(max_events)
    s.precision = int(precision)

    t = OracleTallies()
    rr = np.zeros((A.PMO_RR_CATS, nr), np.float64) if nr > 0 else None
    absorbed = np.zeros(prob.labels.shape, np.float64) if fluence else None
    ph_state = np.zeros((n_photons, 10), np.float64) if per_photon else None
    ph_counts = np.zeros((n_photons, 4), np.uint32) if per_photon else None
    t.rr, t.nr, t.dr = _ptr(rr), int(nr), float(dr)
    t.absorbed = _ptr(absorbed)
    t.ph_state, t.ph_counts = _ptr(ph_state), _ptr(ph_counts)
    grads = {}
    if grad_coef is not None:
        if nr <= 0:
            raise ValueError("gradients need R(r) bins (nr > 0)")
        gc = np.ascontiguousarray(np.asarray(grad_coef, np.float64).reshape(A.PMO_RR_CATS, nr))
        keep.append(gc)
        grads = {"g_ma_voxel": np.zeros(prob.labels.shape), "g_ms_voxel": np.zeros(prob.labels.shape),
                 "g_ma_label": np.zeros(prob.n_labels), "g_ms_label": np.zeros(prob.n_labels)}
        t.grad_coef = gc.ctypes.data
        for k, v in grads.items():
            setattr(t, k, v.ctypes.data)
    if threads <= 0:
        threads = os.cpu_count() or 1
    status = lib.oracle_run(C.byref(s), C.byref(t), int(threads))
    del keep
    return {
        "status": int(status),
        "ledger": np.array(t.ledger[:], np.float64),
        "counters": np.array(t.counters[:], np.uint64),
        "rr": rr,
        "absorbed": absorbed,
        "ph_state": ph_state,
        "ph_counts": ph_counts,
        "threads": threads,
        **grads,
    }
