"""The multi-rank replica path on CPU (gloo, world size 2).

Each rank traces its share of one run's photon ids with the CPU oracle (the
device kernel uses the same Philox streams, and ``tests/test_gpu_transport``
checks it against the oracle per photon). The ranks sum their tallies with
``replicas.reduce_tallies``, which reproduces the single-process run.
``max_over_ranks`` gives the benchmark's timing reduction.
"""
import multiprocessing as mp
import os
import socket
import sys
import traceback
from datetime import timedelta

import numpy as np
import pytest

from pymonteopt_b200 import _abi as A
from pymonteopt_b200 import replicas
from pymonteopt_b200 import volumes as V
from pymonteopt_b200.problem import pencil_problem

HERE = os.path.dirname(os.path.abspath(__file__))
N_PHOTONS, SEED, NR, DR = 3001, 11, 20, 0.1


def _problem():
    vol, end = V.plate_volume(2.0, 2.0, 0.1, [0.5, 0.5])
    return pencil_problem(vol, 0.1, end, [0.2, 0.1], [10.0, 20.0], [0.9, 0.8],
                          [1.4, 1.5, 1.0])


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, queue):
    try:
        sys.path.insert(0, HERE)
        sys.path.insert(0, os.path.dirname(HERE))
        import torch
        import torch.distributed as dist
        import oracle
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=timedelta(seconds=60))
        begin, count = replicas.photon_range(rank, world, N_PHOTONS)
        r = oracle.run(_problem(), count, SEED, begin=begin, precision=A.PMO_FP64, nr=NR,
                       dr=DR, fluence=True, threads=1)
        ledger = torch.from_numpy(r["ledger"].copy())
        counters = torch.from_numpy(r["counters"].astype(np.int64))
        rr = torch.from_numpy(r["rr"].copy())
        absorbed = torch.from_numpy(r["absorbed"].copy())
        replicas.reduce_tallies([ledger, counters, rr, None, absorbed])
        t_max = replicas.max_over_ranks(1.5 + rank)
        spans = [None] * world
        dist.all_gather_object(spans, (begin, count))
        if rank == 0:
            queue.put(("ok", ledger.numpy(), counters.numpy(), rr.numpy(), absorbed.numpy(),
                       t_max, spans))
        dist.barrier()
        dist.destroy_process_group()
    except Exception:  # report to the parent instead of hanging it
        queue.put(("error", traceback.format_exc()))


def test_photon_ranges_partition():
    for n in (0, 1, 7, 3001, 10**9 + 3):
        for world in (1, 2, 3, 8):
            spans = [replicas.photon_range(r, world, n) for r in range(world)]
            assert spans[0][0] == 0
            assert all(spans[i][0] + spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            assert sum(c for _, c in spans) == n
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1
    assert replicas.rank_offset(3, 100, 7) == 2100
    with pytest.raises(ValueError):
        replicas.photon_range(2, 2, 10)


def test_two_gloo_ranks_reproduce_single_run():
    import oracle
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        msg = queue.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert msg[0] == "ok", msg[1]
    _, ledger, counters, rr, absorbed, t_max, spans = msg
    assert spans == [replicas.photon_range(r, 2, N_PHOTONS) for r in range(2)]
    assert t_max == 2.5
    ref = oracle.run(_problem(), N_PHOTONS, SEED, begin=0, precision=A.PMO_FP64, nr=NR, dr=DR,
                     fluence=True, threads=1)
    np.testing.assert_array_equal(counters.astype(np.uint64), ref["counters"])
    np.testing.assert_allclose(ledger, ref["ledger"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(rr, ref["rr"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(absorbed, ref["absorbed"], rtol=1e-12, atol=1e-15)
    assert counters[A.PMO_C_PHOTONS] == N_PHOTONS
