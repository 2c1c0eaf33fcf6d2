"""The C ABI without a GPU: header constants, struct layouts, exported symbols."""
import ctypes as C
import os
import re
import subprocess

import pytest

from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "pmo_b200.h")


def _header():
    with open(HEADER) as f:
        return f.read()


def test_header_defines_match_python():
    defs = dict(re.findall(r"#define\s+(PMO_\w+)\s+(\d+)u?\b", _header()))
    assert defs, "no #defines parsed"
    for name, val in defs.items():
        assert hasattr(A, name), f"{name} missing from _abi.py"
        assert getattr(A, name) == int(val), name


def _declared_functions():
    return set(re.findall(r"^\s*(?:int|size_t|const char \*)\s*(pmo_\w+)\(", _header(), re.M))


@pytest.fixture(scope="module")
def built_lib():
    from pymonteopt_b200 import _build
    _build.build()
    return _lib.load()


def test_library_loads_and_exports_every_declared_symbol(built_lib):
    names = _declared_functions()
    assert {"pmo_run_plain", "pmo_cuvmc", "pmo_status_string"} <= names
    for n in names:
        assert hasattr(built_lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"
    # entry points that need no GPU
    assert built_lib.pmo_abi_version() == A.PMO_ABI_VERSION
    assert built_lib.pmo_workspace_bytes() >= 512
    assert built_lib.pmo_status_string(A.PMO_ERR_LABEL).decode().startswith("photon")
    c = (C.c_ulonglong * A.PMO_COUNTERS_N)()
    assert built_lib.pmo_check_counters(c) == A.PMO_OK
    c[A.PMO_C_ERR_CAP] = 1
    assert built_lib.pmo_check_counters(c) == A.PMO_ERR_STEP_CAP


def test_argument_validation_rejects_before_any_device_call(built_lib):
    # null problem / tallies are refused on the host, no CUDA call is made
    assert built_lib.pmo_run_plain(None, None, None, None, 0, None) == A.PMO_ERR_ARG
    p = A.PmoProblem()
    assert built_lib.pmo_run_plain(C.byref(p), None, None, None, 0, None) == A.PMO_ERR_ARG
    assert built_lib.pmo_run_grad(None, None, None, None, 0, None) == A.PMO_ERR_ARG
    # the entry point without a workspace argument: problem, tallies, launch, stream
    sig = _lib.SIGNATURES["pmo_run_plain_static"]
    assert sig == (C.c_int, [C.POINTER(A.PmoProblem), C.POINTER(A.PmoTallies),
                             C.POINTER(A.PmoLaunch), C.c_void_p])
    assert built_lib.pmo_run_plain_static(None, None, None, None) == A.PMO_ERR_ARG
    assert built_lib.pmo_workspace_bytes() <= A.PMO_STATIC_WORKSPACE_BYTES
    # batched slabs: the pointers are only checked for null on the host, so
    # stand-in addresses reach the checks of the other fields
    fake = 256
    b = A.PmoBatch()
    b.slabs, b.items, b.sums, b.bins = fake, fake, fake, fake
    b.n_problems, b.n_items, b.nr, b.precision = 1, 1, 4, A.PMO_FP32
    b.tally_mode = 7
    assert built_lib.pmo_run_batched(C.byref(b), None, C.c_void_p(fake), 512, None) == A.PMO_ERR_ARG
    b.tally_mode, b.precision = A.PMO_BT_GLOBAL, 5
    assert built_lib.pmo_run_batched(C.byref(b), None, C.c_void_p(fake), 512, None) == A.PMO_ERR_ARG
    b.precision = A.PMO_FP32
    assert built_lib.pmo_run_batched(C.byref(b), None, None, 0, None) == A.PMO_ERR_WORKSPACE
    # optical bench: an empty or oversized scan and a fixed draw outside [0, 1)
    o = A.PmoObdParams()
    o.z, o.n_z, o.fixed_u = fake, 0, -1.0
    out = C.c_void_p(fake)
    args = (C.c_void_p(fake), C.c_void_p(fake), C.c_void_p(fake), 10, out, None)
    assert built_lib.pmo_run_obd(C.byref(o), *args) == A.PMO_ERR_ARG
    o.n_z = 4097
    assert built_lib.pmo_run_obd(C.byref(o), *args) == A.PMO_ERR_ARG
    o.n_z, o.fixed_u = 8, 1.0
    assert built_lib.pmo_run_obd(C.byref(o), *args) == A.PMO_ERR_ARG
    # no photons: nothing to do, and no device call
    o.fixed_u = -1.0
    assert built_lib.pmo_run_obd(C.byref(o), C.c_void_p(fake), C.c_void_p(fake),
                                 C.c_void_p(fake), 0, out, None) == A.PMO_OK


def _c_offsets(struct_name, fields):
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
           f'printf("%zu\\n", sizeof({struct_name}));']
    for f in fields:
        src.append(f'printf("%zu\\n", offsetof({struct_name}, {f}));')
    src.append("return 0;}")
    d = os.path.join(REPO, "oracle", "_build")
    os.makedirs(d, exist_ok=True)
    c_path = os.path.join(d, f"layout_{struct_name}.c")
    exe = c_path[:-2]
    with open(c_path, "w") as fh:
        fh.write("\n".join(src))
    subprocess.run(["gcc", "-o", exe, c_path], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return [int(x) for x in out]


@pytest.mark.parametrize("cls,name", [(A.PmoProblem, "pmo_problem"), (A.PmoTallies, "pmo_tallies"),
                                      (A.PmoLaunch, "pmo_launch"), (A.PmoGrad, "pmo_grad"),
                                      (A.PmoSlab, "pmo_slab"), (A.PmoBatchItem, "pmo_batch_item"),
                                      (A.PmoBatch, "pmo_batch"),
                                      (A.PmoLayer, "pmo_layer"), (A.PmoStack, "pmo_stack"),
                                      (A.PmoStackBatch, "pmo_stack_batch"),
                                      (A.PmoObdParams, "pmo_obd_params")])
def test_struct_layout_matches_header(cls, name):
    fields = [f[0] for f in cls._fields_]
    got = _c_offsets(name, fields)
    assert got[0] == C.sizeof(cls)
    for f, off in zip(fields, got[1:]):
        assert getattr(cls, f).offset == off, f
