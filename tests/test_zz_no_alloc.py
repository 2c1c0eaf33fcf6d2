"""pmo_run_plain_static: the transport entry point that allocates nothing.

It serves callers that cannot allocate device memory themselves (a plugin
whose host application owns all device memory through its own pool, or a
path where cudaMalloc may not run because it can synchronise the device).
Its scratch is a file-scope device array inside the library instead of a
caller-allocated workspace; its results must equal those of pmo_run_plain on
the same photons, on consecutive calls (the array keeps the previous call's
contents, so this also checks that the photon counter is cleared each time).
Both entry points are called through the C ABI.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import engine as E
from pymonteopt_b200 import volumes as V
from pymonteopt_b200._lib import load

pytestmark = pytest.mark.gpu


def _run(static: bool, dp, spec, n, seed, t=None):
    lib = load()
    t = E.Tallies(dp, spec, n) if t is None else t.zero_()
    s = dp.struct(seed, 0, n, A.PMO_FP32, flags=A.PMO_FLAG_EXPORT_EXITS)
    ts = t.struct()
    launch = A.PmoLaunch(0, 0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if static:
        st = lib.pmo_run_plain_static(C.byref(s), C.byref(ts), C.byref(launch), stream)
    else:
        st = lib.pmo_run_plain(C.byref(s), C.byref(ts), C.byref(launch),
                               C.c_void_p(dp.workspace.data_ptr()), dp.workspace.numel(), stream)
    assert st == A.PMO_OK, lib.pmo_status_string(st)
    torch.cuda.synchronize()
    t.check()
    return t


def test_static_workspace_entry_matches_allocating_entry(cuda):
    assert load().pmo_workspace_bytes() <= A.PMO_STATIC_WORKSPACE_BYTES
    prob = V.c1_slab()
    dp = E.DeviceProblem(prob, cuda)
    n, seed = 200000, 21
    spec = E.TallySpec(nr=100, dr=0.1, fluence=A.PMO_FLU_GLOBAL, export_exits=True)
    ref = _run(False, dp, spec, n, seed)
    got = E.Tallies(dp, spec, n)        # the caller's tally buffers, allocated up front
    _run(True, dp, spec, n, seed, got)  # the first call on the device looks up the scratch

    def used():
        torch.cuda.synchronize()
        return torch.cuda.memory_allocated(cuda), torch.cuda.mem_get_info(cuda)[0]

    for _ in range(2):   # two calls in a row share the static scratch
        before = used()
        _run(True, dp, spec, n, seed, got)
        # the call allocated nothing: neither through torch nor on the device
        assert used() == before
        # integer counters and per-photon exit states are exact; sums of
        # float atomics differ only by the order of additions
        assert np.array_equal(got.host_counters(), ref.host_counters())
        for a, b in ((got.exit_add, ref.exit_add), (got.exit_p, ref.exit_p),
                     (got.exit_v, ref.exit_v), (got.exit_w, ref.exit_w)):
            assert torch.equal(a, b)
        np.testing.assert_allclose(got.ledger.cpu().numpy(), ref.ledger.cpu().numpy(),
                                   rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(got.rr.cpu().numpy(), ref.rr.cpu().numpy(),
                                   rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(got.absorbed.cpu().numpy(), ref.absorbed.cpu().numpy(),
                                   rtol=1e-4, atol=1e-6)
