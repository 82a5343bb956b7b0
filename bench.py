"""Benchmark of the two-component D3Q27 TSLB step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One "step" is one time step of the fused CUDA kernel over the whole
lattice.  The workload is the two-component colour-gradient channel
384x192x128 (x, y periodic, half-way bounce-back walls at z, body force
gx = 2.5e-6, nu = 0.0015, 40 droplets of radius 8), FP32 state resident in
HBM.  The state (830 MB) is larger than the 126 MB L2, so no flush is
needed between steps.

Under torchrun every rank advances its own independent copy of the channel
on its own GPU (replicas, weak scaling): the step has no inter-GPU
exchange on one domain, so there is no collective on the data path.
Timing: CUDA events on the library's stream around exactly K steps,
bracketed by a barrier and a device synchronize, max over ranks.

--impl reference times the CPU path of the reference algorithm on the
host cores: the C++ restatement under oracle/ (the reference is Fortran
and no Fortran compiler exists on these machines), all host threads, on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALG_BYTES_PER_NODE = 88  # 11 FP32 moments read + 11 written per lattice update
METRIC = "MLUPS"
UNIT = "MLUPS"
WORKLOAD = ("channel 384x192x128 two-component colour-gradient recursive-regularized D3Q27 TSLB, "
            "x/y periodic, z half-way bounce-back, gx=2.5e-6, nu=0.0015, 40 droplets R=8, sigma=0.005, beta=0.7")


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(ms: float, device: str = "cuda") -> float:
    """Device time of the slowest rank (every rank calls this, in the same order)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_mlups(ws: int, nodes: int, steps: int, ms_max: float) -> float:
    """Weak scaling: every rank advances its own replica of `nodes` nodes."""
    return ws * nodes * steps / (ms_max * 1e-3) / 1e6


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_node():
    """DRAM bytes per lattice update of the step kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "step_kernel_traffic.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["dram_bytes_per_node"]), d
    return None, None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        def rd():
            for line in self.proc.stdout:
                self.lines.append(line.strip())
        self.thread = threading.Thread(target=rd, daemon=True)
        self.thread.start()

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(max_seconds: float = 20.0):
    """Time the oracle (C++ restatement of the reference CPU path, OpenMP, FP32)
    on the channel workload: full size if a step fits the budget, else slabs of
    fewer x columns (the full wall-to-wall depth, droplets in proportion)."""
    import oracle
    from entropicthreadsafe_b200 import workloads
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    nx = 384
    while True:
        p, f = workloads.channel() if nx == 384 else workloads.channel(nx=nx, ndrops=max(1, 40 * nx // 384))
        nz, ny = f["rho"].shape[0], f["rho"].shape[1]
        o = oracle.Oracle(p, nx, ny, nz, fp64=False, fast=True)
        o.set_moments({k: v.astype(np.float64) for k, v in f.items()})
        t0 = time.perf_counter()
        o.step(1)
        t1 = time.perf_counter() - t0
        if t1 * 3 <= max_seconds or nx <= 24:
            break
        o.close()
        nx = max(24, nx // 2)
    steps = max(1, int(max_seconds / max(t1, 1e-6)) - 1)
    steps = min(steps, 50)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    o.close()
    nodes = nx * ny * nz
    return {"value": nodes * steps / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"oracle (C++ restatement of the reference CPU path, FP32, OpenMP) on the channel "
                      f"{nx}x{ny}x{nz}, {steps} steps after 1 warm-up step, {dt:.1f} s"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    base = cpu_baseline(max_seconds=max(5.0, min(60.0, 3.0 * (args.steps + args.warmup))))
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded channel initial state)",
        "config": {"workload": WORKLOAD, "nx": 384, "ny": 192, "nz": 128},
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def e2e_run(args, p, f, ws, steps=None):
    """The same metric through the public API with host buffers: create,
    upload from pinned host memory, K x (step + FP64 diagnostics of that step
    queued for the host, tslb_reduce_async), the queued diagnostics read back
    (tslb_reduce_collect), download to pinned host memory; wall clock, max
    over ranks."""
    steps = args.steps if steps is None else steps
    import torch
    from entropicthreadsafe_b200 import capi
    from entropicthreadsafe_b200.solver import Lattice
    nz, ny, nx = f["rho"].shape
    nodes = nx * ny * nz
    pinned = {k: torch.empty((nz, ny, nx), dtype=torch.float32, pin_memory=True) for k in capi.FIELDS}
    for k in capi.FIELDS:
        pinned[k].numpy()[...] = f[k]
    host_in = {k: pinned[k].numpy() for k in capi.FIELDS}
    out_pinned = {k: torch.empty((nz, ny, nx), dtype=torch.float32, pin_memory=True) for k in capi.FIELDS}
    host_out = {k: out_pinned[k].numpy() for k in capi.FIELDS}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lat2 = Lattice(p, nx, ny, nz)
    t1 = time.perf_counter()
    lat2.upload_moments(host_in)
    t2 = time.perf_counter()
    diags = []
    for k in range(steps):
        lat2.step(1)
        lat2.reduce_async()
        if (k + 1) % capi.REDUCE_QUEUE == 0:
            diags += lat2.reduce_collect()
    diags += lat2.reduce_collect()
    t3 = time.perf_counter()
    assert len(diags) == steps
    lat2.download(host_out)
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    e2e_s = t4 - t0
    lat2.close()
    parts = {"create_ms": (t1 - t0) * 1e3, "upload_ms": (t2 - t1) * 1e3,
             "step_and_reduce_ms_per_step": (t3 - t2) * 1e3 / steps, "download_ms": (t4 - t3) * 1e3}
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    state_bytes = 11 * 4 * nodes
    return {"value": ws * nodes * steps / e2e_s / 1e6, "unit": UNIT, "steps": steps,
            "h2d_bytes_per_step": state_bytes / steps,
            "d2h_bytes_per_step": state_bytes / steps + 8 * capi.NREDUCE,
            "what": "tslb_create + tslb_upload_moments (pinned host) + K x (tslb_step(1) + tslb_reduce_async) "
                    "+ tslb_reduce_collect + tslb_download_moments, wall clock, per step", "parts": parts}


def ensemble_leg(args, ndomains: int = 48):
    """Config 4: 48 droplet-in-Couette domains of uneven size advanced by one
    launch per step (K steps from a CUDA graph, tuned z chunk and grid),
    against the same domains launched one at a time."""
    import torch
    from entropicthreadsafe_b200 import ensemble
    from entropicthreadsafe_b200.solver import Lattice
    doms = ensemble.couette_droplets(n=ndomains, seed=2024)
    nodes = sum(a * b * c for a, b, c in (d["dims"] for d in doms))
    with ensemble.Ensemble([d["params"] for d in doms], [d["dims"] for d in doms]) as ens:
        for i, d in enumerate(doms):
            ens.upload_moments(i, d["fields"])
        zc, gr = ens.tune()
        rows = ens.tune_results()
        st = torch.cuda.ExternalStream(ens.stream)
        k = args.steps if args.steps % 2 == 0 else args.steps + 1
        ens.step_graph(k)  # capture + warm-up
        ens.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        ens.step_graph(k)
        e1.record(st)
        ens.synchronize()
        ms_graph = e0.elapsed_time(e1) / k
        e0.record(st)
        ens.step(k)
        e1.record(st)
        ens.synchronize()
        ms_plain = e0.elapsed_time(e1) / k
        # the non-persistent form for comparison: one block per work item, the tuned z chunk
        ens.set_launch(zc, 0)
        ens.step(2)
        e0.record(st)
        ens.step(k)
        e1.record(st)
        ens.synchronize()
        ms_per_item = e0.elapsed_time(e1) / k
    # the same domains, one lattice at a time
    lats = []
    for d in doms:
        nx, ny, nz = d["dims"]
        lat = Lattice(d["params"], nx, ny, nz)
        lat.upload_moments(d["fields"])
        lat.step(1)
        lat.synchronize()
        lats.append(lat)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for lat in lats:
        lat.step(k)
        lat.synchronize()
    ms_seq = (time.perf_counter() - t0) * 1e3 / k
    for lat in lats:
        lat.close()
    # the tuner's table (10 steps per candidate): best time of each resident grid
    tuner = {"candidates": len(rows),
             "best_per_grid": {str(g): min((r["ms"] for r in rows if r["grid"] == g)) for g in sorted({r["grid"] for r in rows})}}
    return {"domains": ndomains, "nodes": nodes, "steps": k, "tuned": {"zchunk": zc, "grid": gr}, "tuner": tuner,
            "value_graph": nodes / (ms_graph * 1e-3) / 1e6, "value_launch_per_step": nodes / (ms_plain * 1e-3) / 1e6,
            "value_one_block_per_item": nodes / (ms_per_item * 1e-3) / 1e6,
            "value_one_at_a_time": nodes / (ms_seq * 1e-3) / 1e6, "unit": UNIT,
            "speedup_vs_one_at_a_time": ms_seq / ms_graph}


def closure_leg(args):
    """Config 5 cost: the coarse round jet (192 x 192 x 384, sponge, pressure
    outlet) stepped plain and with the learned closure attached (refresh every
    step and every 2 steps).  The closure's cost does not depend on its
    weights, so a seeded initial network stands in for the trained one (the
    accuracy study is entropicthreadsafe_b200.closure_study)."""
    import numpy as np
    import torch
    from entropicthreadsafe_b200 import workloads
    from entropicthreadsafe_b200.closure import Closure, init_params, lattice_attach
    from entropicthreadsafe_b200.solver import Lattice
    p, f, spec = workloads.jet(1)
    nodes = spec["nx"] * spec["ny"] * spec["nz"]
    res = {"workload": "round jet 192x192x384, disc inlet d=16, nu 8e-4", "nodes": nodes, "steps": args.steps}
    with Lattice(p, spec["nx"], spec["ny"], spec["nz"]) as lat, Closure() as c:
        c.set_params(init_params(0), np.zeros(10), np.array([1e-4] * 6 + [1.0, 0.3, 0.05, 1e-4]), 0.02)
        lat.upload_moments(f)
        lat.set_tau_correction(workloads.jet_sponge(spec))
        step = [0]

        def advance(k):
            for _ in range(k):
                if step[0] % spec["refresh"] == 0:
                    workloads.jet_inlet(lat, spec, 13, step[0])
                lat.step(1)
                step[0] += 1

        advance(300)  # the jet leaves the inlet
        lat.synchronize()
        st = torch.cuda.ExternalStream(lat.stream)

        def timed():
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            advance(args.warmup)
            e0.record(st)
            advance(args.steps)
            e1.record(st)
            lat.synchronize()
            return e0.elapsed_time(e1) / args.steps

        ms = {"plain": timed()}
        for k in (1, 2):
            lattice_attach(lat, c, k)
            ms[f"closure_every_{k}"] = timed()
        lattice_attach(lat, None)
    for name, m in ms.items():
        res[name] = {"value": nodes / (m * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": m}
    kern = ms["closure_every_1"] - ms["plain"]
    # inference kernel: reads 10 moment fields + previous and static dtau, writes dtau (52 B/node);
    # two dense layers 16x64 and 64x64 on the tensor cores (2 * 5120 flop/node)
    res["closure_kernel"] = {"ms": kern, "bytes_per_node": 52, "tensor_flop_per_node": 10240,
                             "GB_per_s": 52 * nodes / (kern * 1e-3) / 1e9,
                             "tensor_TFLOP_per_s": 10240 * nodes / (kern * 1e-3) / 1e12}
    return res


def single_leg(args):
    """Single-component mode (the reference's fused_TSLB_force_1c) on the channel
    384 x 192 x 128 without droplets: force gx, bounce-back walls at z; 80 B per
    lattice update (10 moment fields read and written)."""
    import torch
    from entropicthreadsafe_b200 import capi, workloads
    from entropicthreadsafe_b200.solver import Lattice
    p, f = workloads.channel()
    p.mode = capi.MODE_SINGLE
    f["phi"][:] = 1.0
    nz, ny, nx = f["rho"].shape
    nodes = nx * ny * nz
    with Lattice(p, nx, ny, nz) as lat:
        st = torch.cuda.ExternalStream(lat.stream)
        lat.upload_moments(f)
        lat.step(args.warmup)
        lat.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        lat.step(args.steps)
        e1.record(st)
        lat.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
    peak, kind = peaks()
    gbs = 80 * nodes / (ms * 1e-3) / 1e9
    return {"workload": "channel 384x192x128, single component, gx 2.5e-6, bounce-back walls", "value": nodes / (ms * 1e-3) / 1e6,
            "unit": UNIT, "ms_per_step": ms, "bytes_per_lu": 80,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak}}


def phasefield_leg(args):
    """The reference program's own operator (phase field, D3Q7 + CSF shift,
    recursive_2c_TSLB3D.f90) on the channel 384 x 192 x 128: the same seeded
    flow and droplets with phi in [0, 1], sharpening 0.3 * 3; 88 B per
    lattice update in the step kernel (plus the interface-normal pass, timed
    with it: every launch of a step is inside the timed region)."""
    import torch
    from entropicthreadsafe_b200 import capi, workloads
    from entropicthreadsafe_b200.solver import Lattice
    p, f = workloads.channel()
    p.mode = capi.MODE_PHASEFIELD
    p.sharp_c = 0.9
    f["phi"] = (0.5 * (1.0 + f["phi"])).astype(np.float32)
    nz, ny, nx = f["rho"].shape
    nodes = nx * ny * nz
    with Lattice(p, nx, ny, nz) as lat:
        st = torch.cuda.ExternalStream(lat.stream)
        lat.upload_moments(f)
        lat.step(args.warmup)
        lat.synchronize()
        l0 = lat.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        lat.step(args.steps)
        e1.record(st)
        lat.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        launches = (lat.launches - l0) / args.steps
    peak, kind = peaks()
    gbs = ALG_BYTES_PER_NODE * nodes / (ms * 1e-3) / 1e9
    return {"workload": "channel 384x192x128, phase field (phi in [0,1], sharp_c 0.9), sigma 0.005, gx 2.5e-6",
            "value": nodes / (ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms, "launches_per_step": launches,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak}}


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    from entropicthreadsafe_b200 import capi, workloads
    from entropicthreadsafe_b200.solver import Lattice

    p, f = workloads.channel(nz=args.nz) if args.nz else workloads.channel()
    nz, ny, nx = f["rho"].shape
    nodes = nx * ny * nz

    def barrier_sync():
        torch.cuda.synchronize()
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    lat = Lattice(p, nx, ny, nz)
    stream = torch.cuda.ExternalStream(lat.stream)
    lat.upload_moments(f)
    lat.step(args.warmup)
    lat.synchronize()
    # ---- device-resident timing ----
    barrier_sync()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = lat.launches
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    lat.step(args.steps)
    ev1.record(stream)
    lat.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = lat.launches - l0
    clk = clocks.stop()
    barrier_sync()
    red = lat.reduce()
    ms_max = max_over_ranks(ms)
    value = whole_job_mlups(ws, nodes, args.steps, ms_max)
    ms_step = ms_max / args.steps
    lat.close()
    # ---- end to end through the public API with host buffers (the same workload,
    # right after the device-resident run: its lattice reuses that run's memory) ----
    barrier_sync()
    e2e = None if args.no_e2e else e2e_run(args, p, f, ws)
    # the same at 200 steps, where the state's upload and download weigh less
    e2e_200 = None if args.no_e2e else e2e_run(args, p, f, ws, steps=200)
    # ---- precision forms of the same workload (bf16, fp16 with per-field scale) ----
    forms = None
    if not args.no_precision_forms:
        forms = {}
        for name, prec in (("bf16", capi.PREC_BF16), ("fp16s", capi.PREC_FP16S)):
            p.precision = prec
            lp = Lattice(p, nx, ny, nz)
            sp = torch.cuda.ExternalStream(lp.stream)
            lp.upload_moments(f)
            lp.step(args.warmup)
            lp.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(sp)
            lp.step(args.steps)
            e1.record(sp)
            lp.synchronize()
            ms_p = e0.elapsed_time(e1) / args.steps
            forms[name] = {"value": ws * nodes / (ms_p * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms_p,
                           "speedup_vs_fp32": ms_step / ms_p, "bytes_per_lu": 44,
                           "rounding": "stochastic (hashed from node, field and step)"}
            lp.close()
        p.precision = capi.PREC_FP32
    ens = None if args.no_ensemble else ensemble_leg(args)
    clo = None if args.no_closure else closure_leg(args)
    sgl = None if args.no_single else single_leg(args)
    pfl = None if args.no_phasefield else phasefield_leg(args)
    barrier_sync()
    state_bytes = 11 * 4 * nodes
    # ---- roofline of the step kernel ----
    peak, peak_kind = peaks()
    alg_bytes = ALG_BYTES_PER_NODE * nodes
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    tpn, tinfo = traffic_per_node()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tpn * nodes if tpn else None, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": alg_bytes, "kernel": "tslb::step_kernel<colour>"}
    # second ceiling: instruction issue.  The kernel executes `ipn` thread
    # instructions per lattice update (ncu counter smsp__thread_inst_executed.sum
    # of one launch / its nodes, committed with the traffic figure); an SM
    # issues at most 4 warp instructions (128 thread instructions) per cycle.
    ipn = tinfo.get("thread_instructions_per_node") if tinfo else None
    if ipn and clk and clk.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        issue_rate = sms * 4 * 32 * clk["sm_mhz"] * 1e6          # thread instructions per second
        lups = nodes / (ms_step * 1e-3)
        roof["issue"] = {"thread_instructions_per_lu": ipn, "sms": sms, "sm_mhz": clk["sm_mhz"],
                         "ceiling_mlups": issue_rate / ipn / 1e6, "frac": lups * ipn / issue_rate,
                         "source": tinfo.get("instructions_command")}
        # and the FP32 share: FADD + 2 FFMA + FMUL per update against 128 FP32 lanes per SM, FMA = 2 flops
        fpn = tinfo.get("fp32_flops_per_node")
        if fpn:
            fp32_peak = sms * 128 * 2 * clk["sm_mhz"] * 1e6
            roof["fp32"] = {"flops_per_lu": fpn, "achieved_tflops": lups * fpn / 1e12,
                            "peak_tflops": fp32_peak / 1e12, "frac": lups * fpn / fp32_peak}
    if rank != 0:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0
    base = cpu_baseline(max_seconds=20.0) if ws == 1 and not args.no_cpu_baseline else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded channel initial state, counter-based noise)",
        "config": {"workload": WORKLOAD, "nx": nx, "ny": ny, "nz": nz, "nodes_per_gpu": nodes,
                   "parallelism": f"replicas x{ws}", "l2": "state 830 MB > 126 MB L2, no flush needed",
                   "state_bytes": state_bytes},
        "roofline": roof, "cpu_baseline": base, "e2e": e2e, "gpu_launches": launches,
        "e2e_200_steps": e2e_200,
        "precision_forms": forms, "ensemble": ens, "closure": clo, "single_component": sgl, "phase_field": pfl,
        "clocks": clk, "check": {"mass": red["mass"], "umax": red["umax"], "mass_a": red["mass_a"]},
    }
    print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-precision-forms", action="store_true", help="skip the bf16 / fp16 storage legs")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 48-domain ensemble leg")
    ap.add_argument("--no-closure", action="store_true", help="skip the learned-closure jet leg")
    ap.add_argument("--no-single", action="store_true", help="skip the single-component channel leg")
    ap.add_argument("--no-phasefield", action="store_true", help="skip the phase-field channel leg")
    ap.add_argument("--nz", type=int, default=0, help="shallower channel (profiling runs only)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
