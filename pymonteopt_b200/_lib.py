"""Loader for the CUDA shared library (``_lib/libpmo_b200.so``).

The library is the only compute path: if it is missing or cannot be loaded,
every transport call raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import _abi as A

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libpmo_b200.so")

_lock = threading.Lock()
_lib = None

# Every symbol the C header declares, with (restype, argtypes).
SIGNATURES = {
    "pmo_run_obd": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                              C.c_void_p, C.c_void_p]),
    "pmo_abi_version": (C.c_int, []),
    "pmo_status_string": (C.c_char_p, [C.c_int]),
    "pmo_device_info": (C.c_int, [C.POINTER(C.c_int)] * 3),
    "pmo_workspace_bytes": (C.c_size_t, []),
    "pmo_run_plain": (C.c_int, [C.POINTER(A.PmoProblem), C.POINTER(A.PmoTallies),
                                C.POINTER(A.PmoLaunch), C.c_void_p, C.c_size_t, C.c_void_p]),
    "pmo_run_grad": (C.c_int, [C.POINTER(A.PmoProblem), C.POINTER(A.PmoGrad),
                               C.POINTER(A.PmoLaunch), C.c_void_p, C.c_size_t, C.c_void_p]),
    "pmo_run_batched": (C.c_int, [C.POINTER(A.PmoBatch), C.POINTER(A.PmoLaunch), C.c_void_p,
                                  C.c_size_t, C.c_void_p]),
    "pmo_batch_finalize": (C.c_int, [C.POINTER(A.PmoBatch), C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "pmo_run_stack_batch": (C.c_int, [C.POINTER(A.PmoStackBatch), C.POINTER(A.PmoLaunch),
                                      C.c_void_p, C.c_size_t, C.c_void_p]),
    "pmo_stack_batch_finalize": (C.c_int, [C.POINTER(A.PmoStackBatch), C.c_void_p, C.c_void_p,
                                           C.c_void_p]),
    "pmo_run_plain_static": (C.c_int, [C.POINTER(A.PmoProblem), C.POINTER(A.PmoTallies),
                                       C.POINTER(A.PmoLaunch), C.c_void_p]),
    "pmo_cuvmc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_float, C.c_int32, C.c_int32, C.c_int32,
                            C.c_int8, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t,
                            C.c_void_p]),
    "pmo_normalize_fluence": (C.c_int, [C.POINTER(A.PmoProblem), C.c_void_p, C.c_double,
                                        C.c_void_p, C.c_void_p]),
    "pmo_check_counters": (C.c_int, [C.c_void_p]),
    "pmo_philox_words": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_int,
                                   C.c_void_p]),
    "pmo_build_voxel_words": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "pmo_fp32_probe": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "pmo_philox_words_curand": (C.c_int, [C.c_ulonglong, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_int, C.c_void_p]),
}


class ExtensionMissing(RuntimeError):
    pass


def load():
    """Load the CUDA library once; raise :class:`ExtensionMissing` if absent."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ExtensionMissing(
                    f"{LIB_PATH} is missing: build it with "
                    "`python -m pymonteopt_b200._build` (needs nvcc); there is no CPU fallback")
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            if lib.pmo_abi_version() != A.PMO_ABI_VERSION:
                raise ExtensionMissing("libpmo_b200.so ABI version mismatch; rebuild it")
            _lib = lib
        return _lib


class PmoError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        self.status = int(status)
        msg = A.STATUS_NAMES.get(self.status, f"status {status}")
        super().__init__(f"{where}: {msg}" if where else msg)


def check(status: int, where: str = "") -> None:
    if status != A.PMO_OK:
        raise PmoError(status, where)
