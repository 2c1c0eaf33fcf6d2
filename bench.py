#!/usr/bin/env python3
"""Photon-transport benchmark on one B200 (or N replicas).

Workload (one step): 1e8 photons of the three-layer skin slab — 400x400x400
voxels at 0.05 mm (padded 402^3 uint8 labels), epidermis 0.1 mm / dermis 2 mm
/ subcutis, collimated Gaussian beam of 1 mm 1/e^2 radius, FP32 transport,
FP64 ledger, R(r)/T(r) with 100 bins of 0.1 mm.  Synthetic and seeded; no
dataset is involved.

``value`` is photons/s with the volume resident in HBM, timed with CUDA events
on the launching stream, L2 flushed between steps; ``e2e`` is the same metric
through the drop-in model API, every step: ``VoxelPlateModel.build`` on the
host, ``start`` (label and table upload, box map, transport, ledger read)
and the Rd/Tt and R(r) getters.  ``parity`` holds the timed run against the
reference's own runs of the workload (tests/golden/ref_c2_gaussian.json).
``--impl reference`` and ``cpu_baseline`` time the reference's own CPU path
(pymopt.voxel, Numba, unmodified, from baseline/_ref) on all host cores, on
bounded samples of the same workload.

Multi-GPU (``torchrun --nproc-per-node N``): photons are independent, so each
rank runs its own photon range of the same problem (weak scaling, no
collective on the data path); only the timing uses a barrier and a MAX
reduction.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "photons/s per B200 at R(r) within 3σ of ref"
UNIT = "photons/s"
WORKLOAD = "c2_three_layer_skin_400^3_gaussian_beam"
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--photons", type=float, default=1e8, help="photons per step per GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched+gradient vs plain comparison (4096 slabs)")
    ap.add_argument("--no-stacks", action="store_true",
                    help="skip the layered batch vs plain comparison (1024 skin stacks)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own cuVMC kernel on the 256^3 volume")
    ap.add_argument("--ref-gpu-photons", type=float, default=1e7)
    ap.add_argument("--no-gradient", action="store_true",
                    help="skip timing the differentiable form (64^3 per-voxel optics)")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the FP32-vs-FP64 error of the results (1e6 photons, C1 and C2)")
    ap.add_argument("--block-threads", type=int, default=0)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    return ap.parse_args()


def config_dict(photons: int, world: int) -> dict:
    from pymonteopt_b200 import volumes as V
    return {
        "workload": WORKLOAD,
        "voxels": [402, 402, 402],
        "voxel_space_mm": V.C2_PARAMS["voxel_space"],
        "layers_mm": V.C2_PARAMS["thickness"],
        "w_beam_mm": V.C2_W_BEAM,
        "photons_per_step_per_gpu": photons,
        "rr_bins": [100, 0.1],
        "fluence_tally": False,
        "l2": "flushed between timed steps (256 MiB write); uint16 voxel-word map 130 MB",
        "parallelism": f"replicas x{world} (photon ranges per GPU, no collectives)",
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": num(rows[0][2]), "reasons": reasons, "samples": len(rows),
                "power_w_max": max((num(r[3]) or 0.0) for r in rows)}


# ---------------------------------------------------------------------------
def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_oracle_rate(target_seconds: float, seed: int = 1234) -> dict:
    """Photons/s of the FP32 C restatement (oracle/vmc_oracle.c, OpenMP on
    all host threads) on a bounded sample of the benchmark workload: context
    for the reference's own CPU path, which runs one photon at a time."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # noqa: E402  (test infrastructure; CPU baseline only)
    from pymonteopt_b200 import _abi as A
    from pymonteopt_b200 import volumes as V
    prob = V.c2_skin()
    threads = host_threads()
    oracle.load()                      # build/load outside the timed calibration
    n = max(2000, 200 * threads)
    t0 = time.perf_counter()
    oracle.run(prob, n, seed, precision=A.PMO_FP32, nr=100, dr=0.1, threads=threads)
    dt = time.perf_counter() - t0
    n2 = int(max(n, min(5e8, n * target_seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    r = oracle.run(prob, n2, seed + 1, begin=n, precision=A.PMO_FP32, nr=100, dr=0.1,
                   threads=threads)
    dt = time.perf_counter() - t0
    return {"value": n2 / dt, "photons": n2, "seconds": dt, "threads": threads,
            "Rd": float(r["ledger"][A.PMO_L_RD] / n2)}


class ReferenceCPU:
    """The reference's own CPU path on this host: ``VoxelPlateModel(nPh,
    w_beam=1.0).build(**C2).start()`` (Numba ``vmc_kernel``,
    pymopt/voxel/_kernel.py:23-172, one photon after another), unmodified,
    imported from the copy in baseline/_ref (oracle/ref_cpu.py).  ``processes``
    independent spawned processes with distinct seeds; Numba's JIT runs before
    the first timed sample.  A step times every process's own start() on
    ``n_per`` photons; its rate is all photons over the slowest process."""

    def __init__(self, processes: int):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import ref_cpu  # noqa: E402  (reference baseline only)
        from pymonteopt_b200 import volumes as V
        self.ref_cpu = ref_cpu
        if not ref_cpu.available():
            raise RuntimeError("baseline/_ref holds no copy of the reference "
                               "(python oracle/ref_cpu.py <reference checkout>)")
        import numba  # noqa: F401  (the reference's kernel needs it)
        self.processes = processes
        self.pool = ref_cpu.RefPool(dict(V.C2_PARAMS), processes, {"w_beam": V.C2_W_BEAM})
        self.rate_per_process = None

    def calibrate(self, photons: int = 1000, seed: int = 50) -> dict:
        r = self.pool.step(photons, seed)
        self.rate_per_process = photons / max(r["seconds"], 1e-6)
        return r

    def timed(self, seconds: float, seed: int) -> dict:
        n_per = int(min(2e6, max(1000, self.rate_per_process * seconds)))
        return self.pool.step(n_per, seed)

    def close(self):
        self.pool.close()

    def describe(self) -> dict:
        return {"cpu": self.ref_cpu.host_cpu(), "processes": self.processes,
                "code": "reference pymopt.voxel VoxelPlateModel.start (Numba vmc_kernel), "
                        "unmodified copy in baseline/_ref, one photon at a time per process"}


def reference_cpu_baseline(target_seconds: float = 8.0) -> dict:
    """cpu_baseline of this arm: the reference's own CPU path on all host
    cores, one bounded sample of the workload, plus one process alone."""
    threads = host_threads()
    ref = ReferenceCPU(threads)
    try:
        ref.calibrate()
        r = ref.timed(target_seconds, seed=60)
        desc = ref.describe()
    finally:
        ref.close()
    one = ReferenceCPU(1)
    try:
        one.calibrate()
        r1 = one.timed(target_seconds / 2, seed=70)
    finally:
        one.close()
    return {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{r['photons']} photons of the workload ({r['photons'] // threads} per "
                      f"process) in {r['seconds']:.1f} s on {threads} processes; "
                      f"one process alone: {r1['value']:.4g} photons/s "
                      f"({r1['photons']} photons in {r1['seconds']:.1f} s)",
            "single_process_value": r1["value"], **desc}


def run_reference(args, rank: int, world: int) -> None:
    """Reference arm: the reference's own CPU path (ReferenceCPU) on all host
    cores; each step is a bounded sample of the workload (its photons and
    seconds are the step's own).  Falls back to the C restatement, marked
    kind "port", only if the reference copy or Numba is missing.  Under
    torchrun only rank 0 runs."""
    if rank != 0:
        return
    photons = int(args.photons)
    threads = host_threads()
    per_step = max(1.0, min(8.0, 120.0 / max(args.steps, 1)))
    vals, secs, sample = [], [], 0
    try:
        ref = ReferenceCPU(threads)
    except (RuntimeError, ImportError) as e:
        ref, why = None, str(e)
    if ref is not None:
        try:
            for k in range(max(args.warmup, 1)):
                ref.calibrate(seed=80 + k)
            for k in range(args.steps):
                r = ref.timed(per_step, seed=100 + k)
                vals.append(r["value"])
                secs.append(r["seconds"])
                sample += r["photons"]
            desc = ref.describe()
        finally:
            ref.close()
        kind = "reference"
        what = (f"{sample} photons of the workload over {args.steps} steps "
                f"({sum(secs):.1f} s of start() time, {threads} processes)")
    else:
        for _ in range(args.warmup):
            cpu_oracle_rate(per_step / 4)
        for k in range(args.steps):
            r = cpu_oracle_rate(per_step, seed=100 + k)
            vals.append(r["value"])
            secs.append(r["seconds"])
            sample += r["photons"]
        kind, desc = "port", {"reference_unavailable": why}
        what = (f"{sample} photons of the workload over {args.steps} steps "
                f"({sum(secs):.1f} s), oracle/vmc_oracle.c FP32, OpenMP")
    value = float(sample / sum(secs))
    line = {
        "impl": "reference",
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(secs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": config_dict(photons, world),
        "step_sample": {"photons_per_step": sample // max(args.steps, 1),
                        "note": "each step runs this many photons of the workload; "
                                "ms_per_step is that sample's own time"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": what, **desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_gpu_leg(torch, dev, photons: int) -> dict:
    """The reference's own GPU kernel cuVMC (pymopt/voxel_gpu/_cukernel.py,
    compiled unchanged into oracle/_ref) against this kernel on the 256^3
    CT-like volume with a pencil beam, the same photon count on each side.

    * kernel: state (reference) or volume (ours) resident on the device,
      CUDA events around the launch;
    * e2e: the reference's start() traffic, i.e. 40 B/photon of state copied
      from pinned host memory and back; ours copies the label volume in and
      the tallies out.
    """
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref_gpu  # noqa: E402  (reference kernel: baseline only)
    from pymonteopt_b200 import _abi as A
    from pymonteopt_b200 import engine as E
    from pymonteopt_b200 import volumes as V
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/libcuvmc_ref.so was not built (reference tree absent)"}
    prob = V.c3_ct_like(0)
    stream = torch.cuda.current_stream()

    def timed(fn, reps=3):
        best = float("inf")
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b) / 1e3)
        return best

    ref = ref_gpu.RefVolume(prob, dev)
    warm = ref.initial_state(100000)
    ref.launch(*warm, seed=1)
    state = ref.initial_state(photons)
    fresh = [t.clone() for t in state]

    def ref_kernel():
        for d, s0 in zip(state, fresh):
            d.copy_(s0)
        ref.launch(*state, seed=7)
    # the state reset is a device copy of 40 B/photon, timed apart and removed
    t_reset = timed(lambda: [d.copy_(s0) for d, s0 in zip(state, fresh)])
    t_ref = max(timed(ref_kernel) - t_reset, 1e-9)
    ref_res = ref.results(*state, nr=100, dr=0.2)

    host = [t.cpu().pin_memory() for t in fresh]
    back = [torch.empty_like(h).pin_memory() for h in host]

    def ref_e2e():
        for d, h in zip(state, host):
            d.copy_(h, non_blocking=True)
        ref.launch(*state, seed=8)
        for h, d in zip(back, state):
            h.copy_(d, non_blocking=True)
    t_ref_e2e = timed(ref_e2e)

    out = {"workload": "c3_ct_like_256^3_pencil", "photons": photons,
           "reference": {"kernel_photons_per_s": photons / t_ref,
                         "e2e_photons_per_s": photons / t_ref_e2e,
                         "Rd": ref_res["Rd"], "Tt": ref_res["Tt"],
                         "source": "pymopt/voxel_gpu/_cukernel.py cuVMC, nvcc sm_100a, "
                                   "128 threads/block, one thread per photon"}}
    dp = E.DeviceProblem(prob, dev)
    pinned_labels = torch.from_numpy(prob.labels).pin_memory()
    for name, flu in (("ours", A.PMO_FLU_NONE), ("ours_with_fluence", A.PMO_FLU_GLOBAL)):
        spec = E.TallySpec(nr=100, dr=0.2, fluence=flu)
        t = E.run_plain(dp, 100000, 1, spec=spec)
        tal = E.Tallies(dp, spec, photons)

        def ours_kernel():
            tal.zero_()
            E.run_plain(dp, photons, 7, tallies=tal)
        t_zero = timed(tal.zero_)
        t_ours = max(timed(ours_kernel) - t_zero, 1e-9)
        tal.check()
        led = tal.ledger.cpu().numpy()
        host_led = torch.empty_like(tal.ledger, device="cpu").pin_memory()
        host_rr = torch.empty_like(tal.rr, device="cpu").pin_memory()
        host_abs = (torch.empty_like(tal.absorbed, device="cpu").pin_memory()
                    if tal.absorbed is not None else None)

        def ours_e2e():
            dp.labels.copy_(pinned_labels, non_blocking=True)
            tal.zero_()
            E.run_plain(dp, photons, 8, tallies=tal)
            host_led.copy_(tal.ledger, non_blocking=True)
            host_rr.copy_(tal.rr, non_blocking=True)
            if host_abs is not None:
                host_abs.copy_(tal.absorbed, non_blocking=True)
        t_ours_e2e = timed(ours_e2e)
        out[name] = {"kernel_photons_per_s": photons / t_ours,
                     "e2e_photons_per_s": photons / t_ours_e2e,
                     "Rd": float(led[A.PMO_L_RD] / photons),
                     "Tt": float(led[A.PMO_L_TT] / photons)}
    # the drop-in entry point with the reference's own arguments and in-place
    # state arrays (pmo_cuvmc: voxel-by-voxel stepping, no box map), timed
    # and copied exactly as the reference kernel is above
    ws = torch.empty(int(E.load().pmo_workspace_bytes()), dtype=torch.uint8, device=dev)

    def dropin(seed):
        E.cuvmc(*state, ref.ma, ref.ms, ref.n, ref.g, ref.model,
                float(np.float32(prob.voxel_space)), photons, int(prob.end_label), seed, ws)

    def dropin_kernel():
        for d, s0 in zip(state, fresh):
            d.copy_(s0)
        dropin(7)
    t_drop = max(timed(dropin_kernel) - t_reset, 1e-9)
    drop_res = ref.results(*state, nr=100, dr=0.2)

    def dropin_e2e():
        for d, h in zip(state, host):
            d.copy_(h, non_blocking=True)
        dropin(8)
        for h, d in zip(back, state):
            h.copy_(d, non_blocking=True)
    t_drop_e2e = timed(dropin_e2e)
    out["ours_dropin_cuvmc"] = {"kernel_photons_per_s": photons / t_drop,
                                "e2e_photons_per_s": photons / t_drop_e2e,
                                "Rd": drop_res["Rd"], "Tt": drop_res["Tt"],
                                "path": "pmo_cuvmc: the reference's argument list and state "
                                        "arrays, voxel-by-voxel stepping"}
    out["speedup_kernel"] = out["ours"]["kernel_photons_per_s"] / out["reference"]["kernel_photons_per_s"]
    out["speedup_e2e"] = out["ours"]["e2e_photons_per_s"] / out["reference"]["e2e_photons_per_s"]
    return out


def gradient_leg(torch, dev, photons: int = 10_000_000, evals: int = 3) -> dict:
    """The differentiable form on its workload: 64^3 voxels at 0.25 mm with
    per-voxel optics, 1e7 photons, loss = squared error of the 50-bin R(r)
    against a seeded target, backward = Philox replay giving dL/dmu_a and
    dL/dmu_s per voxel.  Times forward and backward with CUDA events."""
    from pymonteopt_b200 import grad as G
    from pymonteopt_b200 import volumes as V
    model = G.DifferentiableRr(V.c4_voxel_props(0), n_photons=photons, seed=3, nr=50, dr=0.1,
                               props="voxel", device=dev)
    ma, ms = model.initial_params()
    target = model(ma * 1.1, ms * 0.95).detach()      # a seeded, different target
    stream = torch.cuda.current_stream()
    fw, bw = [], []
    for k in range(evals + 1):
        ma_, ms_ = ma.clone().requires_grad_(True), ms.clone().requires_grad_(True)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(stream)
        R = model(ma_, ms_)
        loss = ((R - target) ** 2).sum()
        e1.record(stream)
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
        if k:                                          # the first evaluation warms up
            fw.append(e0.elapsed_time(e1) / 1e3)
            bw.append(e1.elapsed_time(e2) / 1e3)
    rep = model.last_replay
    t_f, t_b = float(np.median(fw)), float(np.median(bw))
    return {"workload": "c4_voxel_props_64^3_per_voxel_optics", "photons": photons,
            "forward_s": t_f, "backward_s": t_b, "evals_per_s": 1.0 / (t_f + t_b),
            "forward_photons_per_s": photons / t_f,
            "replayed_photons": int(rep.replayed), "replay_mismatches": int(rep.mismatches),
            "backward_replayed_photons_per_s": rep.replayed / t_b,
            "grad_finite": bool(torch.isfinite(ma_.grad).all() and torch.isfinite(ms_.grad).all())}


def precision_leg(torch, dev, photons: int = 1_000_000) -> dict:
    """Error of the FP32 product against the FP64 build of the same kernel on
    identical Philox streams (the per-photon oracle): Rd, Tt, A, R(r) and the
    absorbed grid, on C1 and on the CT-like volume (both with the fluence
    tally; the CT-like volume has the most Fresnel events per photon) and on
    this workload (C2)."""
    from pymonteopt_b200 import _abi as A
    from pymonteopt_b200 import engine as E
    from pymonteopt_b200 import volumes as V
    out = {"photons": photons}
    for name, prob, flu in (("c1_slab", V.c1_slab(), A.PMO_FLU_GLOBAL),
                            ("c3_ct_like", V.c3_ct_like(0), A.PMO_FLU_GLOBAL),
                            ("c2_skin", V.c2_skin(), A.PMO_FLU_NONE)):
        dp = E.DeviceProblem(prob, dev)
        runs = {}
        for prec in (A.PMO_FP32, A.PMO_FP64):
            spec = E.TallySpec(nr=100, dr=0.1, fluence=flu, photon_stats=True)
            t = E.run_plain(dp, photons, 4242, spec=spec, precision=prec)
            torch.cuda.synchronize()
            t.check()
            runs[prec] = t
        t32, t64 = runs[A.PMO_FP32], runs[A.PMO_FP64]
        s32, s64 = t32.summary(), t64.summary()
        r = {}
        for key in ("Rd", "Tt", "A"):
            r[key] = {"fp32": float(s32[key]), "fp64": float(s64[key]),
                      "abs_err": float(abs(s32[key] - s64[key]))}
        # Rd's standard error from the run itself, for scale
        r["Rd"]["binomial_se"] = float(np.sqrt(max(s64["Rd"] * (1 - s64["Rd"]), 0.0) / photons))
        rr32 = t32.rr.double()[A.PMO_RR_TOP]
        rr64 = t64.rr.double()[A.PMO_RR_TOP]
        r["Rr_top"] = {"rel_l1_err": float((rr32 - rr64).abs().sum() / rr64.abs().sum()),
                       "max_abs_err_of_max": float((rr32 - rr64).abs().max() / rr64.abs().max())}
        same = (t32.ph[0] == t64.ph[0]) & (t32.ph[2] == t64.ph[2])
        r["same_event_counts_share"] = float(same.double().mean())
        if flu != A.PMO_FLU_NONE:
            g32, g64 = E.absorbed_weight(t32), E.absorbed_weight(t64)
            hot = g64 >= 0.01 * g64.max()
            r["absorbed"] = {
                "rel_l2_err": float((g32 - g64).norm() / g64.norm()),
                "max_rel_err_hot_voxels": float(((g32 - g64).abs()[hot] / g64[hot]).max()),
                "hot_voxels": int(hot.sum())}
        out[name] = r
    return out


def parity_vs_reference(tallies, photons: int) -> dict:
    """The timed run against the reference's own VoxelPlateModel(w_beam=1.0)
    runs of the same workload (tests/golden/ref_c2_gaussian.json, made by
    tests/golden/make_golden.py): z-scores of Rd and Tt and per-bin z of R(r)
    and T(r), each timed step one sample.  The fixture's standard error
    dominates (1.6e6 reference photons against 1e8 per step)."""
    from scipy import stats as st
    from pymonteopt_b200 import _abi as A
    if len(tallies) < 2:
        return {"unavailable": "the z-scores need the spread of at least 2 timed steps"}
    path = os.path.join(REPO, "tests", "golden", "ref_c2_gaussian.json")
    with open(path) as f:
        g = json.load(f)
    nr, dr = g["nr"], g["dr"]
    area = np.array([2 * np.pi * (i + 0.5) * dr ** 2 for i in range(nr)])
    Rd, Tt, Rr, Tr = [], [], [], []
    for t in tallies:
        L = t.ledger.cpu().numpy()
        rr = t.rr.cpu().numpy().astype(np.float64)
        if rr.shape[1] != nr:
            raise ValueError("the timed run's R(r) bins differ from the fixture's")
        Rd.append(L[A.PMO_L_RD] / photons)
        Tt.append(L[A.PMO_L_TT] / photons)
        Rr.append((rr[A.PMO_RR_TOP] + rr[A.PMO_RR_LAT_NEG]) / (area * photons))
        Tr.append((rr[A.PMO_RR_BOTTOM] + rr[A.PMO_RR_LAT_POS]) / (area * photons))

    def mse(x):
        x = np.asarray(x, np.float64)
        se = x.std(axis=0, ddof=1) / np.sqrt(len(x)) if len(x) > 1 else np.zeros_like(x[0])
        return x.mean(axis=0), se

    out = {"fixture": "tests/golden/ref_c2_gaussian.json",
           "reference_photons": int(g["nPh"]) * len(g["seeds"]),
           "reference_code": "pymopt.voxel VoxelPlateModel(w_beam=1.0) (Numba), unmodified"}
    zmax = 0.0
    for key, mine in (("Rd", Rd), ("Tt", Tt)):
        m, s_ = mse(mine)
        rm, rs = mse(g[key])
        z = float((m - rm) / np.hypot(s_, rs))
        out[key] = {"ours": float(m), "reference": float(rm), "reference_se": float(rs),
                    "z": z}
        zmax = max(zmax, abs(z))
    for key, mine in (("Rr", Rr), ("Tr", Tr)):
        m, s_ = mse(mine)
        ref = np.asarray(g[key], np.float64)
        rm, rs = mse(ref)
        keep = (np.count_nonzero(ref, axis=0) >= 5) & (rs > 0)
        z = (m[keep] - rm[keep]) / np.hypot(s_[keep], rs[keep])
        chi2 = float(np.sum(z ** 2))
        out[key] = {"bins": int(keep.sum()), "chi2": chi2,
                    "p": float(st.chi2.sf(chi2, int(keep.sum()))) if keep.any() else None,
                    "zmax": float(np.max(np.abs(z))) if keep.any() else 0.0}
        zmax = max(zmax, out[key]["zmax"])
    out["zmax"] = zmax
    out["within_3sigma"] = bool(abs(out["Rd"]["z"]) < 3 and abs(out["Tt"]["z"]) < 3 and
                                all(out[k]["p"] is None or out[k]["p"] > 1e-3
                                    for k in ("Rr", "Tr")))
    return out


# ---------------------------------------------------------------------------
def fp32_probe(torch, lib) -> float:
    """Measured FP32 issue rate (FFMA thread-instructions per second)."""
    import ctypes as C
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    blocks, threads = props.multi_processor_count * 8, 256
    out = torch.zeros(blocks, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream()
    iters = 2000
    best = 0.0
    for rep in range(4):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        st = lib.pmo_fp32_probe(C.c_void_p(out.data_ptr()), blocks, threads, iters,
                                C.c_void_p(s.cuda_stream))
        e1.record(s)
        torch.cuda.synchronize()
        assert st == 0
        if rep == 0:
            continue
        t = e0.elapsed_time(e1) / 1e3
        best = max(best, blocks * threads * iters * 128 / t)
    return best


# the sources that define the plain transport kernel's instructions; the ncu
# summary records their digest, and figures captured from other sources are
# not used
KERNEL_SOURCES = ("vmc_transport.cuh", "philox.cuh", "pmo_internal.h")


def kernel_source_digest() -> str:
    import hashlib
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        with open(os.path.join(REPO, "pymonteopt_b200", "csrc", name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def read_traffic():
    """DRAM bytes and instructions per photon of the transport kernel from the
    committed ncu summary, if present and captured from the current kernel
    sources; else None (the line then carries no traffic)."""
    path = os.path.join(REPO, "profiles", "vmc_plain_c2_ncu.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    if d.get("kernel_source_sha256") != kernel_source_digest():
        return None
    return d


def summary_dict(value, e2e, parity, batched, gradient, reference_gpu, cpu, roofline,
                 stacks=None) -> dict:
    """The headline figures of the run, one level deep."""
    def get(d, *keys):
        for k in keys:
            if not isinstance(d, dict) or d.get(k) is None:
                return None
            d = d[k]
        return d
    return {
        "photons_per_s": value,
        "e2e_photons_per_s": get(e2e, "value"),
        "fp32_issue_frac": get(roofline, "frac"),
        "parity_zmax_vs_reference": get(parity, "zmax"),
        "parity_within_3sigma": get(parity, "within_3sigma"),
        "reference_cpu_photons_per_s": get(cpu, "value"),
        "reference_cpu_single_process_photons_per_s": get(cpu, "single_process_value"),
        "reference_cuvmc_on_b200_kernel_speedup": get(reference_gpu, "speedup_kernel"),
        "batched_evals_per_s": get(batched, "batched_evals_per_s"),
        "batched_ratio_vs_plain_reused": get(batched, "ratio"),
        "batched_ratio_vs_single_launches": get(batched, "ratio_vs_single_launches"),
        "gradient_c4_evals_per_s": get(gradient, "evals_per_s"),
        "stacks_evals_per_s": get(stacks, "batched_evals_per_s"),
        "stacks_ratio_vs_plain_reused": get(stacks, "ratio"),
    }


def main() -> int:
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return 0

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from pymonteopt_b200 import _abi as A
    from pymonteopt_b200 import engine as E
    from pymonteopt_b200 import opcount
    from pymonteopt_b200 import replicas
    from pymonteopt_b200 import volumes as V
    from pymonteopt_b200._lib import load

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    lib = load()
    photons = int(args.photons)
    stream = torch.cuda.current_stream()

    prob = V.c2_skin()
    dp = E.DeviceProblem(prob, dev)
    spec = E.TallySpec(nr=100, dr=0.1)
    # disjoint photon ids for every rank and launch (replicas of one problem)
    begin0 = replicas.rank_offset(rank, photons, args.steps + args.warmup + 1)

    def step(k: int, tallies):
        return E.run_plain(dp, photons, seed=1000 + k, tallies=tallies,
                           begin=begin0 + k * photons,
                           block_threads=args.block_threads, blocks_per_sm=args.blocks_per_sm)

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    for k in range(args.warmup):
        t = step(k, E.Tallies(dp, spec, photons))
    torch.cuda.synchronize()
    t.check()

    peak = fp32_probe(torch, lib)

    # ---- timed region: value -------------------------------------------
    tallies = [E.Tallies(dp, spec, photons) for _ in range(args.steps)]
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    w0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()                       # L2 flush between timed steps
        evs[k][0].record(stream)
        step(args.warmup + k, tallies[k])
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    wall = time.perf_counter() - w0
    clk = clocks.stop()
    dev_s = sum(a.elapsed_time(b) for a, b in evs) / 1e3
    for t in tallies:
        t.check()
    dev_s_max = replicas.max_over_ranks(dev_s, dev)
    total_photons = photons * args.steps * world
    value = total_photons / dev_s_max

    counters = sum(t.host_counters().astype(np.float64) for t in tallies)
    ledger = sum(t.ledger.cpu().numpy() for t in tallies)
    fp32_per_launch = opcount.fp32_ops(counters.astype(np.uint64)) / args.steps
    launch_s = dev_s / args.steps
    achieved = fp32_per_launch / launch_s
    traffic = read_traffic()
    roofline = {
        "bound": "fp32-issue",
        "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "G FP32 inst/s",
        "frac": achieved / peak,
        "peak_source": "measured in this run: FFMA-throughput probe (pmo_fp32_probe)",
        "traffic": (traffic["dram_bytes_per_photon"] * photons) if traffic else None,
        "traffic_note": None if traffic else
            "no ncu summary captured from the current kernel sources",
        "traffic_unit": "bytes per launch (ncu dram__bytes_read+write, scaled per photon)",
        "algorithmic_fp32_per_photon": fp32_per_launch / photons,
        "mufu_per_photon": opcount.mufu_ops(counters.astype(np.uint64)) / (photons * args.steps),
        "philox_draws_per_photon": opcount.philox_draws(counters.astype(np.uint64)) / (photons * args.steps),
    }
    if traffic and "warp_inst_per_photon" in traffic:
        # the instruction-issue ceiling: warp instructions per photon (ncu, same
        # workload) x photons/s against 4 schedulers x SMs x the sampled clock
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        clk_hz = (clk.get("sm_mhz") or clk.get("sm_max_mhz") or 0) * 1e6
        ach = traffic["warp_inst_per_photon"] * photons / launch_s
        pk = 4 * sms * clk_hz
        roofline["issue"] = {
            "achieved": ach / 1e9, "peak": pk / 1e9 if pk else None,
            "unit": "G warp inst/s", "frac": ach / pk if pk else None,
            "warp_inst_per_photon": traffic["warp_inst_per_photon"],
            "lanes_per_warp_inst": traffic["thread_inst_per_photon"] / traffic["warp_inst_per_photon"],
            "source": "instruction counts from ncu on the same workload (profiles/vmc_plain_c2_ncu.json); "
                      "peak = 4 issue slots x SMs x median sampled SM clock",
        }
    if traffic:
        # the HBM side, for scale: DRAM bytes per launch (ncu, same workload)
        # over the launch time, against the measured copy bandwidth
        hbm_peak, hbm_src = 6650.0, "fallback (no MEASURED_PEAKS.json): 6.65 TB/s copy"
        try:
            with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
                mp = json.load(f)
            if mp.get("hbm_gbs"):
                hbm_peak, hbm_src = float(mp["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
        except (OSError, ValueError):
            pass
        gbs = traffic["dram_bytes_per_photon"] * photons / launch_s / 1e9
        roofline["hbm"] = {"achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                           "frac": gbs / hbm_peak, "peak_source": hbm_src}
    inflow = ledger[A.PMO_L_WINIT] + ledger[A.PMO_L_RGAIN]
    outflow = (ledger[A.PMO_L_RD] + ledger[A.PMO_L_TT] + ledger[A.PMO_L_EXIT0] +
               ledger[A.PMO_L_ABS] + ledger[A.PMO_L_RLOSS] + ledger[A.PMO_L_ERRW])
    nsteps_ph = photons * args.steps
    results = {"Rd": ledger[A.PMO_L_RD] / nsteps_ph, "Tt": ledger[A.PMO_L_TT] / nsteps_ph,
               "A": ledger[A.PMO_L_ABS] / nsteps_ph,
               "energy_balance_rel": (inflow - outflow) / inflow,
               "interactions_per_photon": counters[A.PMO_C_INTERACT] / nsteps_ph,
               "crossings_per_photon": counters[A.PMO_C_CROSS] / nsteps_ph,
               "extra_philox_draws_per_photon": counters[A.PMO_C_XDRAWS] / nsteps_ph}
    parity = parity_vs_reference(tallies, photons) if rank == 0 else None

    # ---- e2e: engine API with host buffers --------------------------------
    e2e = None
    if not args.no_e2e:
        # the plugin call a pymopt user makes, every step: build the model's
        # volume on the host, start() (uploads the labels and optical tables,
        # rebuilds the uniform-box map on the device, runs the transport,
        # reads back the ledger and counters) and read Rd/Tt and R(r)
        from pymonteopt_b200 import VoxelPlateModel
        model = VoxelPlateModel(nPh=photons, w_beam=V.C2_W_BEAM, keep_exits=False,
                                verbose=False, nr=100, dr=0.1, device=dev,
                                threadnum=args.block_threads or None)
        # W untimed steps of the same path (the caching allocators, device and
        # page-locked host, reach their steady state here)
        for w_ in range(max(1, args.warmup)):
            model.build(**V.C2_PARAMS)
            model.start(4999 - w_ + 7919 * rank)
            model.getRdTtValues()
            model.get_Rr()
        e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(args.steps)]
        e_wall = []
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            w0_ = time.perf_counter()
            e_ev[k][0].record(stream)
            model.build(**V.C2_PARAMS)
            model.start(5000 + k + 7919 * rank)
            vals = model.getRdTtValues()
            _, rr_host = model.get_Rr()
            e_ev[k][1].record(stream)
            torch.cuda.synchronize()
            e_wall.append(time.perf_counter() - w0_)
        e_s = replicas.max_over_ranks(sum(a.elapsed_time(b) for a, b in e_ev) / 1e3, dev)
        tal = model._tallies
        h2d = model.model.voxel_model.nbytes + sum(
            np.asarray(a, np.float32).nbytes for a in (model.model.ma, model.model.ms,
                                                       model.model.g, model.model.n))
        # start(): counters (check), ledger and counters (results); get_Rr: R(r)
        d2h = 2 * tal.counters.numel() * 8 + tal.ledger.numel() * 8 + tal.rr.numel() * 4
        e2e = {"value": total_photons / e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "path": "VoxelPlateModel(nPh, w_beam=1.0).build(**C2); start(seed); "
                       "getRdTtValues(); get_Rr() -- every step",
               "wall_s_per_step": float(np.mean(e_wall)), "Rd_last_step": vals["Rd"]}
        del model

    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        # second half of the metric: 4096 slab problems, forward + gradient in
        # one graph-captured persistent launch vs per-problem plain evaluations
        from pymonteopt_b200 import batched as B
        batched = B.batched_vs_plain(count=4096, device=dev)

    stacks = None
    if rank == 0 and world == 1 and not args.no_stacks:
        # layered problems: a sweep of three-layer skin stacks in one launch
        from pymonteopt_b200 import batched as B
        stacks = B.stacks_vs_plain(count=1024, device=dev)

    reference_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        reference_gpu = reference_gpu_leg(torch, dev, int(args.ref_gpu_photons))

    gradient = None
    if rank == 0 and world == 1 and not args.no_gradient:
        gradient = gradient_leg(torch, dev)

    precision = None
    if rank == 0 and world == 1 and not args.no_precision:
        precision = precision_leg(torch, dev)

    cpu = cpu_port = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = reference_cpu_baseline(8.0)
        except (RuntimeError, ImportError) as e:
            cpu = {"value": None, "unit": UNIT, "cores": host_threads(), "kind": "reference",
                   "sample": None, "unavailable": str(e)}
        r = cpu_oracle_rate(4.0)
        cpu_port = {"value": r["value"], "unit": UNIT, "cores": r["threads"], "kind": "port",
                    "sample": f"{r['photons']} photons of the workload in {r['seconds']:.1f} s "
                              f"(oracle/vmc_oracle.c FP32, OpenMP, {r['threads']} threads)"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # the long detail blocks come first and the compact summary last, so a
    # record that keeps only the end of the line keeps the headline figures
    line = {
        "fp32_vs_fp64": precision,
        "reference_gpu": reference_gpu,
        "gradient": gradient,
        "batched": batched,
        "stacks": stacks,
        "cpu_port": cpu_port,
        "results": results,
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dev_s_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": config_dict(photons, world),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": args.steps,
        "clocks": clk,
        "wall_s_timed_region": wall,
        "parity": parity,
        "summary": summary_dict(value, e2e, parity, batched, gradient, reference_gpu, cpu,
                                roofline, stacks),
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
