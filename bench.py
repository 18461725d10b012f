#!/usr/bin/env python
"""Benchmark of the 3dmhd time step on B200: Mcell-RK3-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the FP64-plain fine run of the learned-closure case, 512x512x256,
rotating MHD polytrope (Ra=1e6, Ta=1e6, Pr=1, Pm=4, density contrast 10,
beta=1e4, tanh z stretch 1.5), set up by the host mirror of the reference
driver (STATIC + TUBE model 4 + RAN2 perturbation).  One "step" is one
full RK3 step (one CALL STEP).

value  : cells x steps / device time, time from CUDA events on the stream
         the kernels run on, max over ranks; N>1 runs independent replicas
         (the single-GPU path does not shard across GPUs).
e2e    : the same metric through the public C-ABI with host buffers:
         mhd3d_upload from pinned host memory, K x mhd3d_step(1) (each reads
         DT/TIMC/TIMT/UMACH/NIT back, as the driver's DT check needs), and
         mhd3d_download to pinned host memory, all inside the timed region.
roofline: the fused stage kernel, algorithmic bytes 10*nf*8 per cell and
         step (compulsory U/Z traffic), against the measured HBM copy peak.
cpu_baseline: the reference's own step (translated build in oracle/_ref)
         on a bounded 512x512x32 slab of the same physics, all host cores.
--impl reference: the reference's CPU step timed on the host cores for the
         same metric (rank 0 only).
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rast-3dmhd_b200"))

METRIC = "Mcell-RK3-steps/s at 512²×256: FP32+closure vs FP64 plain, same flux error"
UNIT = "Mcell-RK3-steps/s"
WORKLOAD = dict(npx=512, npy=512, npz=256, ra=1e6, ta=1e6, pr=1.0, pm=4.0, contrast=10.0, m=1.0, beta=1e4,
                stretch=1.5, ampt=2e-4)
WORKLOAD_NAME = ("FP64-plain fine run of the closure case: 512x512x256 rotating MHD polytrope, "
                 "Ra=1e6 Ta=1e6 Pr=1 Pm=4 contrast 10 beta=1e4 tanh stretch 1.5")
SAMPLE_NPZ = 32  # CPU baseline slab
# the other named cases, at their own sizes and physics (--case); they print
# the same line for the results table and are not the headline workload
CASES = {
    "c1": dict(npx=64, npy=64, npz=48, ra=1e5, ta=1e4, pr=1.0, pm=4.0, contrast=10.0, m=1.0, beta=1e4,
               stretch=1.5, ampt=2e-4, mode="fast",
               name="c1: 64x64x48 rotating MHD, Ra=1e5 Ta=1e4 contrast 10, FP64 (state fits in L2)"),
    "c2": dict(npx=256, npy=256, npz=128, ra=1e6, ta=1e6, pr=1.0, pm=4.0, contrast=10.0, m=1.0, beta=1e4,
               stretch=1.5, ampt=2e-4, mode="fast", name="c2: 256x256x128 rotating MHD, Ra=1e6 Ta=1e6, FP64"),
    "c5": dict(npx=1024, npy=1024, npz=512, ra=1e7, ta=1e7, pr=1.0, pm=4.0, contrast=30.0, m=1.0, beta=1e4,
               stretch=2.0, ampt=2e-4, mode="fp32",
               name="c5: 1024x1024x512 rotating MHD, Ra=1e7 Ta=1e7 contrast 30 stretch 2, FP32 form"),
    "c5fp64": dict(npx=768, npy=768, npz=384, ra=1e7, ta=1e7, pr=1.0, pm=4.0, contrast=30.0, m=1.0, beta=1e4,
                   stretch=2.0, ampt=2e-4, mode="fast",
                   name="c5 FP64 variant: 768x768x384, Ra=1e7 Ta=1e7 contrast 30 stretch 2, FP64 FMA mode"),
}


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        self.tmp.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.tmp.read().strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.tmp.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(ms: float, dist) -> float:
    """The slowest rank's time (every rank takes the same collective)."""
    if dist is None:
        return ms
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(cells_per_rank: int, steps: int, ms: float, world: int) -> float:
    """Whole-job Mcell-RK3-steps/s: all ranks' cells x steps over the slowest rank's time."""
    return world * cells_per_rank * steps / (ms / 1e3) / 1e6


def pow2_floor(n):
    p = 1
    while p * 2 <= n:
        p *= 2
    return p


def decomposition(cores, npy, npz):
    """NPEY x NPEZ for the reference's own MPI layout: powers of two, >=4 z planes per rank."""
    p = pow2_floor(max(1, cores))
    npez = 1
    while npez * 2 <= p and npz // (npez * 2) >= 4 and npz % (npez * 2) == 0:
        npez *= 2
    npey = p // npez
    while npey > 1 and npy % npey:
        npey //= 2
    return npey, npez


def cpu_reference_run(steps: int, warmup: int, npz: int = SAMPLE_NPZ, work: dict | None = None):
    """Time the reference's own step (translated build) on an npx x npy x npz slab
    of the workload (the bench workload unless work is given), all cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mhd3d
    import oracle_py
    w = dict(work or WORKLOAD, npz=npz)
    cfg = mhd3d.convection_config(w["npx"], w["npy"], w["npz"], w["ra"], w["ta"], w["pr"], w["pm"], w["contrast"],
                                  w["m"], w["beta"], w["stretch"], w["ampt"])
    setup = mhd3d.make_setup(cfg)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    cells = w["npx"] * w["npy"] * w["npz"]
    if oracle_py.reference_available():
        npey, npez = decomposition(cores, w["npy"], w["npz"])
        r = oracle_py.run_reference(setup.params, setup.grid, setup.state, steps, npey=npey, npez=npez,
                                    warmup=warmup)
        secs = r["seconds"]
        kind, used = "reference", npey * npez
        how = f"translated reference STEP, {npey}x{npez} MPI ranks (emulated)"
    else:
        oracle_py.set_threads(cores)
        o = oracle_py.Oracle(setup.params, setup.grid, setup.state)
        o.step(warmup)
        t0 = time.perf_counter()
        o.step(steps)
        secs = time.perf_counter() - t0
        kind, used = "port", oracle_py.oracle_lib().oracle_get_threads()
        how = "C restatement (oracle), OpenMP"
    value = cells * steps / secs / 1e6
    return {"value": value, "unit": UNIT, "cores": used, "kind": kind,
            "sample": f"{w['npx']}x{w['npy']}x{w['npz']} slab of the same physics, {warmup} warm-up + {steps} timed "
                      f"RK3 steps, {how}; {secs:.2f} s"}


def cpu_compare(steps: int, npz: int = SAMPLE_NPZ):
    """The CPU baselines side by side on the bench workload's slab: the C
    restatement (oracle, OpenMP) at 1 thread and at all host cores, and the
    translated reference STEP with its MPI decomposition; one JSON line."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mhd3d
    import oracle_py
    w = dict(WORKLOAD, npz=npz)
    cfg = mhd3d.convection_config(w["npx"], w["npy"], w["npz"], w["ra"], w["ta"], w["pr"], w["pm"], w["contrast"],
                                  w["m"], w["beta"], w["stretch"], w["ampt"])
    setup = mhd3d.make_setup(cfg)
    cells = w["npx"] * w["npy"] * w["npz"]
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    out = {"cpu_compare": True, "unit": UNIT, "slab": [w["npx"], w["npy"], w["npz"]], "steps": steps,
           "host_cores": cores}
    for threads in (1, cores):
        oracle_py.set_threads(threads)
        o = oracle_py.Oracle(setup.params, setup.grid, setup.state)
        o.step(1)
        t0 = time.perf_counter()
        o.step(steps)
        out[f"oracle_{threads}_threads"] = cells * steps / (time.perf_counter() - t0) / 1e6
    if oracle_py.reference_available():
        out["reference_mpi"] = cpu_reference_run(steps, 1, npz=npz)
    print(json.dumps(out), flush=True)


def run_reference_arm(args, rank, world):
    """The reference's own CPU step on the host cores.  A full 512x512x256
    step takes seconds on a CPU, so each step is timed on a slab of the same
    physics (512x512xREF_NPZ): the line's config.grid is that slab,
    ms_per_step is the slab's, and extrapolated_to names the workload whose
    per-cell rate the value stands for (the metric is per cell)."""
    if rank != 0:
        return None
    npz = args.ref_npz
    slab = [WORKLOAD["npx"], WORKLOAD["npy"], npz]
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (host set-up of the reference's STATIC/TUBE/RAN2)",
            "config": {"workload": f"{slab[0]}x{slab[1]}x{slab[2]} slab of the {WORKLOAD_NAME}",
                       "grid": slab,
                       "extrapolated_to": [WORKLOAD["npx"], WORKLOAD["npy"], WORKLOAD["npz"]],
                       "parallelism": "reference MPI decomposition on the host cores"}}
    try:
        cb = cpu_reference_run(args.steps, args.warmup, npz=npz)
    except Exception as e:  # noqa: BLE001
        return {"impl": "reference", "unavailable": f"reference CPU step failed: {e}"[:300]}
    line["value"] = cb["value"]
    line["ms_per_step"] = slab[0] * slab[1] * slab[2] / (cb["value"] * 1e6) * 1e3
    line["cpu_baseline"] = cb
    line["e2e"] = {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    return line


ENSEMBLE_NAME = ("batched FP32 ensemble: 48 rotating MHD members, grids drawn from {64x64x48, 96x96x64, "
                 "128x128x96}, Ra log-uniform 1e4-1e6, Ta log-uniform 1e3-1e6, contrast uniform 3-30, "
                 "perturbation 2e-4, master seed 20261203")


def ensemble_setups(mhd3d, seed=20261203, n=48):
    import numpy as np
    rng = np.random.default_rng(seed)
    grids = [(64, 64, 48), (96, 96, 64), (128, 128, 96)]
    out = []
    for i in range(n):
        g = grids[rng.integers(3)]
        ra, ta, con = 10 ** rng.uniform(4, 6), 10 ** rng.uniform(3, 6), rng.uniform(3, 30)
        cfg = mhd3d.convection_config(*g, ra=ra, ta=ta, contrast=con, ampt=2e-4, seed=i + 1)
        out.append(mhd3d.make_setup(cfg))
    return out


def run_ensemble(args, rank, world, local):
    """The batched ensemble: every member's stages in one persistent launch
    per stage, a step as a CUDA graph, tiles autotuned; value = all members'
    cells x steps / device time."""
    import numpy as np
    import torch
    import mhd3d

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    setups = ensemble_setups(mhd3d)
    cells = sum(su.params.npx * su.params.npy * su.params.npz for su in setups)
    ens = mhd3d.Ensemble(setups)
    stream = torch.cuda.Stream()
    ens.set_stream(stream.cuda_stream)
    for m, su in zip(ens.members, setups):
        m.upload(su.state)
    ens.step(1)
    tuned = ens.tune(steps=3)
    ens.step(args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local) if rank == 0 else None
    barrier()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.step_async(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    res = ens.sync()
    barrier()
    clk = clocks.stop() if clocks else None
    ms = max_over_ranks(ms, dist)
    value = world * cells * args.steps / (ms / 1e3) / 1e6
    peaks, peak_src = measured_peaks()
    achieved = cells * 320.0 * args.steps / (ms / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": None,
            "kernel": "k_stage32_multi (3 persistent launches per step) + k_finalize_multi, whole step",
            "algorithmic_bytes_per_step": cells * 320.0,
            "peak_source": f"{peak_src} MEASURED_PEAKS.json hbm_gbs" if peak_src == "measured" else "fallback 6650 GB/s"}
    # e2e: upload every member from pinned memory, K steps, download every member
    pins = []
    for su in setups:
        nf = 8
        sh = su.shape
        n = sh[0] * sh[1] * sh[2]
        pin_in = torch.empty((nf, n), dtype=torch.float64, pin_memory=True)
        pin_out = torch.empty((nf, n), dtype=torch.float64, pin_memory=True)
        hin = {f: pin_in[i].numpy().reshape(sh, order="F") for i, f in enumerate(mhd3d.FIELDS)}
        hout = {f: pin_out[i].numpy().reshape(sh, order="F") for i, f in enumerate(mhd3d.FIELDS)}
        for f in mhd3d.FIELDS:
            hin[f][...] = su.state[f]
        pins.append((hin, hout, pin_in, pin_out))
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    wt0 = time.perf_counter()
    f0.record(stream)
    for m, (hin, hout, _, _) in zip(ens.members, pins):
        assert m.lib.mhd3d_upload(m.h, *[mhd3d._ptr(hin[f]) for f in mhd3d.FIELDS]) == 0
    ens.step_async(args.steps)
    r2 = ens.sync()
    for m, (hin, hout, _, _) in zip(ens.members, pins):
        assert m.lib.mhd3d_download(m.h, *[mhd3d._ptr(hout[f]) for f in mhd3d.FIELDS]) == 0
    f1.record(stream)
    f1.synchronize()
    ms_e2e = max(f0.elapsed_time(f1), (time.perf_counter() - wt0) * 1e3)
    state_bytes = sum(8 * 8 * su.shape[0] * su.shape[1] * su.shape[2] for su in setups)
    e2e = {"value": world * cells * args.steps / (ms_e2e / 1e3) / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": state_bytes / args.steps,
           "sequence": f"48 x mhd3d_upload (pinned) + mhd3d_ensemble_step({args.steps}) + mhd3d_ensemble_sync "
                       f"+ 48 x mhd3d_download (pinned)", "ms": ms_e2e}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: members set up by the host mirror of STATIC/TUBE model 4/RAN2",
                "config": {"workload": ENSEMBLE_NAME, "members": len(setups), "cells": cells,
                           "tuned": tuned, "l2": "state 1.5 GB in HBM >> 126 MB L2, no flush needed",
                           "parallelism": f"{world} independent ensemble replica(s), one per GPU, no collectives",
                           "nit": [int(x) for x in res["nit"][:4]], "status_nonzero": int((res["status"] != 0).sum())},
                "roofline": roof, "cpu_baseline": None, "e2e": e2e,
                "gpu_launches": 4 * args.steps, "clocks": clk}
        print(json.dumps(line), flush=True)
    ens.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def closure_measure(args, rank, world, local, dt_fine=None):
    """The coarse side of the headline comparison: 128x128x64 FP32 with the
    learned closure attached (evaluated every step: features, three tcgen05
    convolutions, tendencies), same physics as the fine workload, timed with
    CUDA events on its stream; the fine-equivalent rate 512^2*256 *
    (DT_coarse/DT_fine) / wall; and the tensor roofline of the three
    convolutions of one evaluation timed alone.  Returns the pieces for a
    bench line (the handle stays open for the e2e pass of run_closure)."""
    import torch
    import mhd3d
    import closure

    w = dict(WORKLOAD)
    cfg = mhd3d.convection_config(128, 128, 64, w["ra"], w["ta"], w["pr"], w["pm"], w["contrast"], w["m"],
                                  w["beta"], w["stretch"], w["ampt"], seed=62659 + rank)
    setup = mhd3d.make_setup(cfg)
    cells = 128 * 128 * 64
    sim = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.upload(setup.state)
    net = closure.ClosureNet(seed=0)
    net.attach(sim, trip=1e30)
    sim.step(args.warmup)
    clocks = ClockSampler(local) if rank == 0 else None
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step_async(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    res = sim.sync()
    clk = clocks.stop() if clocks else None
    status = sim.closure_status()
    value = world * cells * args.steps / (ms / 1e3) / 1e6
    if dt_fine is None:
        # DT of the fine 512x512x256 run from the same initial physics (one CFL pass)
        fcfg = mhd3d.convection_config(w["npx"], w["npy"], w["npz"], w["ra"], w["ta"], w["pr"], w["pm"],
                                       w["contrast"], w["m"], w["beta"], w["stretch"], w["ampt"], seed=62659 + rank)
        fsetup = mhd3d.make_setup(fcfg)
        fine = mhd3d.GpuSim(fsetup, mode=mhd3d.MODE_FAST)
        fine.upload(fsetup.state)
        dt_fine, _ = fine.cfl()
        fine.close()
    dt_coarse = res["dt"]
    fine_cells = w["npx"] * w["npy"] * w["npz"]
    fine_equiv = fine_cells * (dt_coarse / dt_fine) * args.steps / (ms / 1e3) / 1e6

    # the closure as a per-plane bias tendency alone (no network attached, so
    # none is evaluated): same grid, physics and step count, its own handle
    import numpy as np
    bsim = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    bsim.set_stream(stream.cuda_stream)
    bsim.upload(setup.state)
    bias = np.zeros((7, setup.params.npz), dtype=np.float32)
    bias[:, 1:-1] = 1e-6   # values do not change the cost
    bsim.closure_set_bias(bias)
    bsim.step(args.warmup)
    torch.cuda.synchronize()
    e0.record(stream)
    bsim.step_async(args.steps)
    e1.record(stream)
    e1.synchronize()
    bms = e0.elapsed_time(e1)
    bres = bsim.sync()
    bsim.close()
    bias_only = {"value": world * cells * args.steps / (bms / 1e3) / 1e6, "ms_per_step": bms / args.steps,
                 "dt_coarse": bres["dt"], "status": bres["status"],
                 "fine_equivalent_value": fine_cells * (bres["dt"] / dt_fine) * args.steps / (bms / 1e3) / 1e6}

    # tensor roofline of the convolutions: the three layers of one evaluation,
    # timed alone (CUDA events on the launching stream), against the burst
    # BF16 peak; algorithmic FLOPs 2*27*(8*32 + 32*32 + 32*12) per voxel (the
    # 8 real input channels and 12 real outputs)
    lib = mhd3d.gpu_lib()
    nz, ny, nx = 64, 128, 128
    nvox = nx * ny * nz
    P = lambda t: mhd3d.C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    with torch.cuda.stream(stream):
        feat = (torch.randn((nz, ny, nx, 16), device="cuda") * 0.5).to(torch.bfloat16)
        a1 = torch.empty((nz, ny, nx, 32), dtype=torch.bfloat16, device="cuda")
        a2 = torch.empty_like(a1)
        pred = torch.empty((nz, ny, nx, 16), dtype=torch.float32, device="cuda")
    cerr = torch.zeros(1, dtype=torch.int32, device="cuda")
    sh = mhd3d.C.c_void_p(stream.cuda_stream)

    def evaluation():
        for cin, cout, src, dst, dstf, li, relu in ((16, 32, feat, a1, None, 0, 1), (32, 32, a1, a2, None, 1, 1),
                                                    (32, 16, a2, None, pred, 2, 0)):
            st = lib.mhd3d_conv3d(cin, cout, P(src), P(net.w16[li]), P(net.b[li]), None, relu, P(dst), P(dstf),
                                  nx, ny, nz, P(cerr), sh)
            assert st == 0, st
    for _ in range(3):
        evaluation()
    reps = 20
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    c0.record(stream)
    for _ in range(reps):
        evaluation()
    c1.record(stream)
    c1.synchronize()
    conv_ms = c0.elapsed_time(c1) / reps
    alg_flop = 2.0 * 27 * (8 * 32 + 32 * 32 + 32 * 12) * nvox
    peaks, peak_kind = measured_peaks()
    peak_tf = peaks.get("bf16_tflops", 1590.0)
    achieved_tf = alg_flop / (conv_ms / 1e3) / 1e12
    roof = {"bound": "tensor", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
            "frac": achieved_tf / peak_tf, "traffic": None,
            "kernel": "k_conv3d (three layers of one closure evaluation, timed alone)",
            "algorithmic_flop_per_evaluation": alg_flop, "ms_per_evaluation": conv_ms,
            "peak_source": "measured MEASURED_PEAKS.json bf16_tflops (burst)" if peak_kind == "measured"
            else "fallback 1.59 PFLOP/s"}
    return {"sim": sim, "setup": setup, "cfg": cfg, "stream": stream, "cells": cells, "ms": ms, "value": value,
            "status": status, "dt_coarse": dt_coarse, "dt_fine": dt_fine, "fine_equiv": fine_equiv, "roof": roof,
            "clocks": clk, "bias_only": bias_only}


def closure_profile_record():
    """The a-posteriori profile errors of the closure case as last measured by
    rast-3dmhd_b200/closure_case.py (grid sizes named in the record), read
    from its committed summary; None when the summary is absent."""
    path = os.path.join(ROOT, "profiles", "closure_case_profile_errors.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def closure_summary(args, rank, world, local, dt_fine):
    """The closure object of the default line: the coarse FP32+closure rate
    measured here, its fine-equivalent rate, the convolutions' tensor
    roofline, and the recorded profile errors of the closure case."""
    cm = closure_measure(args, rank, world, local, dt_fine=dt_fine)
    cm["sim"].close()
    return {"workload": "FP32+closure coarse run, 128x128x64, same physics as the fine workload, closure evaluated "
                        "every step (network weights seeded, not trained: throughput does not depend on them)",
            "value": cm["value"], "unit": UNIT, "ms_per_step": cm["ms"] / args.steps, "steps": args.steps,
            "dt_coarse": cm["dt_coarse"], "dt_fine": cm["dt_fine"],
            "fine_equivalent_value": cm["fine_equiv"],
            "fine_equivalent_formula": "512^2*256 cells x (DT_coarse/DT_fine) x steps / coarse wall",
            "closure_status": cm["status"], "conv_roofline": cm["roof"],
            "bias_only": dict(cm["bias_only"], workload="the same coarse run with the closure's per-plane bias "
                              "tendency alone (no network attached), the closure chosen in the recorded case"),
            "profile_error": closure_profile_record()}


def run_closure(args, rank, world, local):
    """The FP32+closure coarse run as its own bench line (see closure_measure),
    with an e2e pass through the C-ABI."""
    import torch
    import mhd3d

    cm = closure_measure(args, rank, world, local)
    sim, setup, cfg, stream, cells = cm["sim"], cm["setup"], cm["cfg"], cm["stream"], cm["cells"]
    ms, value, status, roof, clk = cm["ms"], cm["value"], cm["status"], cm["roof"], cm["clocks"]
    dt_coarse, dt_fine, fine_equiv = cm["dt_coarse"], cm["dt_fine"], cm["fine_equiv"]

    # end to end through the C-ABI: upload from pinned memory, K steps with
    # the closure, download
    shape = setup.shape
    nfort = shape[0] * shape[1] * shape[2]
    nf = 8 if cfg.lmag else 5
    pin = [torch.empty(nfort, dtype=torch.float64, pin_memory=True) for _ in range(2 * nf)]
    hin, hout = {}, {}
    for i, f in enumerate(mhd3d.FIELDS[:nf]):
        a = pin[i].numpy().reshape(shape, order="F")
        a[...] = setup.state[f]
        hin[f] = a
        hout[f] = pin[nf + i].numpy().reshape(shape, order="F")
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    wt0 = time.perf_counter()
    f0.record(stream)
    assert sim.lib.mhd3d_upload(sim.h, *[mhd3d._ptr(hin.get(f)) for f in mhd3d.FIELDS]) == 0
    for _ in range(args.steps):
        sim.step(1)
    assert sim.lib.mhd3d_download(sim.h, *[mhd3d._ptr(hout.get(f)) for f in mhd3d.FIELDS]) == 0
    f1.record(stream)
    f1.synchronize()
    ms_e2e = max(f0.elapsed_time(f1), (time.perf_counter() - wt0) * 1e3)
    state_bytes = nf * nfort * 8
    e2e = {"value": world * cells * args.steps / (ms_e2e / 1e3) / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": state_bytes / args.steps + 40,
           "sequence": f"mhd3d_upload (pinned) + {args.steps} x mhd3d_step(1) with the closure + mhd3d_download",
           "ms": ms_e2e}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
                "data": "synthetic: rotating MHD polytrope from the host mirror of STATIC/TUBE model 4/RAN2; "
                        "network weights seeded, not trained (throughput does not depend on them)",
                "config": {"workload": "FP32+closure coarse run of the closure case: 128x128x64, same physics as "
                                       "the 512x512x256 fine workload",
                           "closure": {"evals": status["evals"], "trips": status["trips"], "err": status["err"]},
                           "dt_coarse": dt_coarse, "dt_fine_first_step": dt_fine,
                           "fine_equivalent_mcell_steps_per_s": fine_equiv,
                           "fine_equivalent_note": "512^2*256 cells x (DT_coarse/DT_fine) per coarse step",
                           "parallelism": f"{world} independent replica(s), one per GPU, no collectives"},
                "roofline": roof, "cpu_baseline": None,
                "e2e": e2e, "gpu_launches": 12 * args.steps, "clocks": clk}
        print(json.dumps(line), flush=True)
    sim.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["fast", "exact", "fp32"], default="fast",
                    help="fast: FP64 with FMA (default); exact: FP64 reference rounding; fp32: FP32 form")
    ap.add_argument("--grid", type=str, default=None, help="override NPXxNPYxNPZ (testing)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-compare", action="store_true",
                    help="only time the CPU baselines (oracle at 1 and all threads, translated reference)")
    ap.add_argument("--no-closure", action="store_true",
                    help="skip the FP32+closure coarse measurement of the default line")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end pass (it pins two host copies of the state)")
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--ref-npz", type=int, default=SAMPLE_NPZ)
    ap.add_argument("--case", choices=sorted(CASES), default=None,
                    help="time another named case at its own size and physics instead of the bench workload")
    ap.add_argument("--workload", choices=["fine", "ensemble", "closure"], default="fine",
                    help="fine: the 512x512x256 step (default); ensemble: the batched FP32 ensemble "
                         "of 48 uneven grids; closure: the FP32+closure coarse 128x128x64 run")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)

    if args.cpu_compare:
        cpu_compare(args.cpu_steps, args.ref_npz)
        return 0
    if args.impl == "reference":
        line = run_reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0

    import numpy as np
    import torch
    import mhd3d

    torch.cuda.set_device(local)
    if args.workload == "ensemble":
        return run_ensemble(args, rank, world, local)
    if args.workload == "closure":
        return run_closure(args, rank, world, local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    w = dict(WORKLOAD)
    wname = WORKLOAD_NAME
    if args.case:
        w = {k: v for k, v in CASES[args.case].items() if k not in ("mode", "name")}
        wname = CASES[args.case]["name"]
        args.mode = CASES[args.case]["mode"]
    if args.grid:
        w["npx"], w["npy"], w["npz"] = (int(v) for v in args.grid.lower().split("x"))
    cfg = mhd3d.convection_config(w["npx"], w["npy"], w["npz"], w["ra"], w["ta"], w["pr"], w["pm"], w["contrast"],
                                  w["m"], w["beta"], w["stretch"], w["ampt"], seed=62659 + rank)
    setup = mhd3d.make_setup(cfg)
    cells = w["npx"] * w["npy"] * w["npz"]
    nf = 8 if cfg.lmag else 5
    mode = {"fast": mhd3d.MODE_FAST, "exact": mhd3d.MODE_EXACT, "fp32": mhd3d.MODE_FP32}[args.mode]
    word = 4 if args.mode == "fp32" else 8
    sim = mhd3d.GpuSim(setup, mode=mode)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.upload(setup.state)

    # warm-up (also builds DT of the first timed step)
    sim.step(args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident throughput -------------------------------------
    clocks = ClockSampler(local) if rank == 0 else None
    sim.profile(True)
    sim.profile_read()
    barrier()
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step_async(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    res = sim.sync()
    barrier()
    clk = clocks.stop() if clocks else None
    stage_ms, stage_n = sim.profile_read()
    sim.profile(False)
    ms = max_over_ranks(ms, dist)
    value = aggregate_rate(cells, args.steps, ms, world)

    # roofline of the fused stage kernel
    peaks, peak_src = measured_peaks()
    launches = sum(stage_n)
    kernel_ms = sum(stage_ms) / max(launches, 1)
    bytes_per_launch = 10 * nf * word * cells / 3.0
    achieved = bytes_per_launch / (kernel_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        key = "mhd_fp32" if args.mode == "fp32" else "mhd_fp64_" + args.mode
        if key in tj:
            traffic = tj[key]["dram_bytes_per_cell_per_launch"] * cells
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
            "kernel": "k_stage (fused RHS+RK3+BCON+CFL), mean of the 3 stage launches",
            "algorithmic_bytes_per_launch": bytes_per_launch, "kernel_ms_per_launch": kernel_ms,
            "peak_source": f"{peak_src} MEASURED_PEAKS.json hbm_gbs" if peak_src == "measured" else "fallback 6650 GB/s",
            "stage_ms_per_launch": [m / max(n, 1) for m, n in zip(stage_ms, stage_n)]}

    # ---- end to end through the C-ABI with pinned host buffers ----------
    e2e = None
    if not args.no_e2e:
        shape = setup.shape
        nfort = shape[0] * shape[1] * shape[2]
        pinned_t = [torch.empty(nfort, dtype=torch.float64, pin_memory=True) for _ in range(2 * nf)]
        hin = {}
        hout = {}
        for i, f in enumerate(mhd3d.FIELDS[:nf]):
            a = pinned_t[i].numpy().reshape(shape, order="F")
            a[...] = setup.state[f]
            hin[f] = a
            hout[f] = pinned_t[nf + i].numpy().reshape(shape, order="F")
        e2e_steps = args.steps
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        wt0 = time.perf_counter()
        f0.record(stream)
        st = sim.lib.mhd3d_upload(sim.h, *[mhd3d._ptr(hin.get(f)) for f in mhd3d.FIELDS])
        assert st == 0, st
        for _ in range(e2e_steps):
            r = sim.step(1)
        st = sim.lib.mhd3d_download(sim.h, *[mhd3d._ptr(hout.get(f)) for f in mhd3d.FIELDS])
        assert st == 0, st
        f1.record(stream)
        f1.synchronize()
        wall_e2e = time.perf_counter() - wt0
        ms_e2e = max(f0.elapsed_time(f1), wall_e2e * 1e3)
        ms_e2e = max_over_ranks(ms_e2e, dist)
        state_bytes = nf * nfort * 8
        e2e = {"value": world * cells * e2e_steps / (ms_e2e / 1e3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": state_bytes / e2e_steps,
               "d2h_bytes_per_step": state_bytes / e2e_steps + 40,
               "sequence": f"mhd3d_upload (pinned) + {e2e_steps} x mhd3d_step(1) with DT/TIMC/TIMT/UMACH/NIT read back "
                           f"+ mhd3d_download (pinned)",
               "ms": ms_e2e}

    # ---- CPU baseline (rank 0, N=1) --------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            if args.case:
                # the whole grid when it is small (c1), else a slab of the case's physics
                cpu = cpu_reference_run(args.cpu_steps, 1, npz=min(w["npz"], args.ref_npz) if w["npz"] > 64
                                        else w["npz"], work=w)
            else:
                cpu = cpu_reference_run(args.cpu_steps, 1)
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"[:200]}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.mode == "fp32" else "f64",
                "data": "synthetic: rotating MHD polytrope from the host mirror of STATIC/TUBE model 4/RAN2",
                "config": {"workload": wname, "grid": [w["npx"], w["npy"], w["npz"]],
                           "mode": args.mode, "fields": nf,
                           "l2": (f"state {3 * nf * cells * word / 1e9:.1f} GB in HBM >> 126 MB L2, no flush needed"
                                  if 3 * nf * cells * word > 126e6 else
                                  f"state {3 * nf * cells * word / 1e6:.0f} MB fits in L2: a small, launch-bound case"),
                           "parallelism": f"{world} independent replica(s), one per GPU, no collectives",
                           "last_dt": res["dt"], "nit": res["nit"]},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": 4 * args.steps, "clocks": clk}
    sim.close()
    # the metric's other half: the FP32+closure coarse run (default workload only)
    if not args.case and not args.grid and not args.no_closure:
        summary = closure_summary(args, rank, world, local, dt_fine=res["dt"])
        if rank == 0:
            line["closure"] = summary
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
