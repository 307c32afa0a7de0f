#!/usr/bin/env python
"""Throughput of the cytokine-diffusion tick on B200.

Workload (default): the human-scale world -- 8 fp32 fields on a 512x256x384
grid (x fastest), Gaussian sigma = 1.5 x (1.2, 0.9, 1.0, 0.8, 1.1, 1.0, 1.3,
0.9), decay (0.05, 0.01, 0.02, 0.03, 0.05, 0.04, 0.06, 0.02) per substep,
200k lognormal(-6, 1) point sources per field, zero padding, seed 0.
One step = one tick = 10 diffusion substeps of all 8 fields + source deposit
+ FP64 totals.  Metric: voxel-steps/s (data voxels x fields x substeps / s).

  python bench.py [--gpus N --steps K --warmup W] [--impl vfd|reference]

N > 1 runs under torchrun: every rank diffuses its own world (independent
units, no data-path collective; weak scaling); the time is the max over
ranks.  `--impl reference` times the CPU restatement of the path (the
reference has no runnable CPU diffusion) on rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "vf-version_7_3_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "voxel-steps/s"
# ncu dram__bytes_read.sum + dram__bytes_write.sum per y/z axis-pass launch of
# this workload (8 fields of 512x256x384), scaled by voxels from the
# 512x256x128 capture in profiles/rf_pass_512x256x128.md (3 x 1038 MB).
AXIS_TRAFFIC_BYTES = 3.11e9


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cfg_by_name(name):
    from vfd import configs
    return {"cfg0": configs.CFG0, "cfg1": configs.CFG1, "cfg4": configs.CFG4}[name]


def fft_contract_bytes(c):
    """Bytes per voxel-step of the canonical 5-sweep 3D FFT convolution
    (8 V + 64 Nc per field and substep, Nc = Fz Fy (Fx / 2 + 1) on the
    minimal padded grid F = n + 2 r per axis, plus 8 B per source deposited
    once per tick), averaged over the world's fields.  The separable
    per-axis passes move 24 B per voxel-step; this is the figure a
    transform-based implementation of the same step has to move."""
    import math
    nx, ny, nz = c["grid"]
    V = nx * ny * nz
    nf = len(c["sigma"])
    tot = 0.0
    for s in c["sigma"]:
        r = int(math.ceil(3.0 * s - 1e-12))
        fx, fy, fz = nx + 2 * r, ny + 2 * r, nz + 2 * r
        nc = fz * fy * (fx // 2 + 1)
        tot += 8.0 * V + 64.0 * nc + 8.0 * c["n_sources"] / c["substeps"]
    return tot / nf / V


def workload_config(c, fft=None):
    nx, ny, nz = c["grid"]
    d = {"workload": f"{c['name']}: {nx}x{ny}x{nz} fp32 x 8 fields, {c['substeps']} substeps "
                     f"per step (tick), {c['n_sources']} sources/field, zero padding, seed {c['seed']}",
         "grid": [nx, ny, nz], "fields": 8, "substeps_per_step": c["substeps"],
         "sources_per_field": c["n_sources"],
         "l2": f"inputs larger than L2: {8 * nx * ny * nz * 4 / 1e9:.2f} GB of fields per world"}
    if fft:
        d["fft"] = list(fft)
    return d


def cpu_baseline(c, n_fields, nthreads=0):
    """FP32 OpenMP CPU port (oracle/vfd_cpu_port.c): one substep of n_fields
    fields of the workload plus their deposit; voxel-steps/s."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from vfd import configs
    nx, ny, nz = c["grid"]
    ins = configs.field_inputs(c["seed"], 0, c["grid"], c["n_sources"], n_fields=n_fields)
    t0 = time.perf_counter()
    for f, (u, idx, amt) in enumerate(ins):
        s = c["sigma"][f]
        oracle.port_substep(u, (s, s, s), (configs.radius(s),) * 3, c["decay"][f], nthreads=nthreads)
        oracle.port_deposit_total(u, idx, amt)
    dt = time.perf_counter() - t0
    vs = nx * ny * nz * n_fields
    return {"value": vs / dt, "unit": METRIC, "cores": oracle.port_threads() if nthreads <= 0 else nthreads,
            "kind": "port",
            "sample": f"{n_fields} field(s) x 1 substep + deposit of the {nx}x{ny}x{nz} world "
                      f"({vs / 1e6:.1f} M voxel-steps), FP32 separable direct convolution, OpenMP",
            "seconds": dt}


def run_reference(args, c):
    """--impl reference: the CPU restatement on the host cores (rank 0 only)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    nf = 1
    for _ in range(args.warmup):
        cpu_baseline(c, nf)
    vals = []
    t_all = 0.0
    for _ in range(args.steps):
        r = cpu_baseline(c, nf)
        vals.append(r["value"])
        t_all += r["seconds"]
    value = args.steps / sum(1.0 / v for v in vals)
    cb = cpu_baseline.__doc__
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(c), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": r["cores"], "kind": "port",
                             "sample": r["sample"] + "; each step is this sample"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's CPU diffusion (Diffuser::diffuseChemCPU) does not run; "
                    "this arm times the FP32 OpenMP restatement of the same method"}
    del cb
    print(json.dumps(line), flush=True)


def run_cfg2(args):
    """Batched ensemble: 32 uneven worlds x 8 fields, 10 substeps per tick, all
    fields of all worlds in one launch per axis pass, tick replayed as a CUDA
    graph.  Beside it: the same worlds through the plain per-field path
    (VFD_METHOD_PLAIN: unfused kernels, one field at a time, no graph)."""
    import torch

    import vfd
    from vfd import configs
    dev = 0
    torch.cuda.set_device(dev)
    c = configs.CFG2
    specs = configs.cfg2_worlds(c["n_worlds"], c["seed"])
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def build(method):
        ws = []
        for sp in specs:
            nx, ny, nz = sp["grid"]
            params = [vfd.field_params(s_, d_) for s_, d_ in zip(sp["sigma"], sp["decay"])]
            w = vfd.World(nx, ny, nz, params, method=method)
            for f, (u, idx, amt) in enumerate(configs.field_inputs(c["seed"], sp["world"], sp["grid"],
                                                                     sp["n_sources"])):
                w.upload(f, u)
                w.set_sources(f, idx, amt)
            ws.append(w)
        return ws

    vox = sum(configs.voxels(sp["grid"]) for sp in specs) * 8 * c["substeps"]
    worlds = build(vfd.METHOD_SEPARABLE)
    batch = vfd.Batch(worlds)
    for _ in range(args.warmup):
        batch.tick(c["substeps"], stream=sh)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    l0 = vfd.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        batch.tick(c["substeps"], stream=sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    launches = vfd.launch_count() - l0
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    value = vox * args.steps / (ms / 1e3)
    # the same worlds ticked one world at a time (separable kernels, no batch, no graph)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for w in worlds:
        w.tick(c["substeps"], stream=sh)
    t0.record(stream)
    for w in worlds:
        w.tick(c["substeps"], stream=sh)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    unbatched = vox / (t0.elapsed_time(t1) / 1e3)
    batch.close()
    for w in worlds:
        w.close()
    # plain per-field path, one world at a time (bounded: 1 tick)
    plain_ms = 0.0
    for sp in specs:
        nx, ny, nz = sp["grid"]
        params = [vfd.field_params(s_, d_) for s_, d_ in zip(sp["sigma"], sp["decay"])]
        w = vfd.World(nx, ny, nz, params, method=vfd.METHOD_PLAIN)
        for f, (u, idx, amt) in enumerate(configs.field_inputs(c["seed"], sp["world"], sp["grid"],
                                                                 sp["n_sources"])):
            w.upload(f, u)
            w.set_sources(f, idx, amt)
        w.tick(1, stream=sh)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        w.tick(c["substeps"], stream=sh)
        p1.record(stream)
        torch.cuda.synchronize(dev)
        plain_ms += p0.elapsed_time(p1)
        w.close()
    plain = vox / (plain_ms / 1e3)
    alg = 24.0 * vox / c["substeps"] * c["substeps"] / 8.0  # bytes: 24 B per voxel-step
    peak, kind = peaks()
    achieved = 24.0 * vox * args.steps / (ms / 1e3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded counter-based generator)",
            "config": {"workload": "batched ensemble: 32 worlds drawn from {96x64x64, 128x96x96, "
                                   "192x128x128, 256x128x192} x 8 fields, 10 substeps per step, "
                                   "500 sources/field, sigma and decay x U[0.5, 2], seed 0",
                       "worlds": [list(sp["grid"]) for sp in specs],
                       "l2": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": "whole step, 24 B per voxel-step (3 axis passes x 8 B)",
                         "peak_source": f"{kind} hbm_gbs"},
            "plain_gpu": {"value": plain, "unit": METRIC,
                          "what": "VFD_METHOD_PLAIN: unfused pad/R2C/C2C/multiply/C2C/C2R/crop kernels, "
                                  "one field per launch sequence, no graph"},
            "unbatched_separable": {"value": unbatched, "unit": METRIC},
            "batched_over_plain": value / plain,
            "gpu_launches": launches, "clocks": clk}
    del alg
    print(json.dumps(line), flush=True)


def run_cfg3(args):
    """Served requests: open-loop Poisson arrivals (precomputed from the seed)
    at 200 req/s for a fixed window; grids drawn from {64x64x32, 128x96x96,
    256x128x192, 512x256x384} with p = {0.4, 0.3, 0.2, 0.1}; 8 fields, 50
    single-substep ticks resident per request, 1e3..2e5 sources per request
    (split over the fields), HBM budget 150 GB.  Reports offered and sustained
    voxel-steps/s and p50/p99 latency (arrival to completion) of the requests
    completed within the measurement."""
    import numpy as np

    import vfd
    from vfd import configs
    c = configs.CFG3
    rng = np.random.default_rng(c["seed"])
    window = args.serve_window
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / c["rate_hz"])
        if t >= window:
            break
        g = c["grids"][int(rng.choice(len(c["grids"]), p=c["probs"]))]
        nsrc = int(rng.integers(c["sources"][0], c["sources"][1] + 1))
        arrivals.append((t, g, nsrc))
    server = vfd.Server(c["hbm_budget_bytes"], max_active=args.serve_slots, substeps_per_tick=1)
    params = [vfd.field_params(s_, d_) for s_, d_ in zip(configs.SIGMA0, configs.DECAY0)]
    offered = 0.0
    ids = []
    t0 = server.clock()
    for k, (ta, g, nsrc) in enumerate(arrivals):
        while server.clock() - t0 < ta:
            time.sleep(0.0005)
        nx, ny, nz = g
        per = [nsrc // 8 + (1 if f < nsrc % 8 else 0) for f in range(8)]
        srcs = [vfd.synth_sources(c["seed"], 1000 + k, f, per[f], nx * ny * nz) for f in range(8)]
        ids.append(server.submit(g, params, c["ticks_per_request"], synth=(c["seed"], 1000 + k, 0.0, 1e-3),
                                 sources=srcs))
        offered += nx * ny * nz * 8 * c["ticks_per_request"]
    # bounded drain: stop measuring at window + grace
    deadline = window + args.serve_grace
    while server.clock() - t0 < deadline:
        st = server.stats()
        if st["completed"] + st["rejected"] >= st["submitted"]:
            break
        time.sleep(0.05)
    elapsed = server.clock() - t0
    st = server.stats()
    server.close()
    sustained = st["voxel_steps_done"] / elapsed
    line = {"metric": METRIC, "value": sustained, "unit": METRIC, "n_gpus": 1, "steps": len(arrivals),
            "warmup": 0, "ms_per_step": 1e3 * elapsed / max(st["completed"], 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded counter-based generator, fields generated on the device)",
            "config": {"workload": f"served requests: Poisson {c['rate_hz']:.0f} req/s for {window:.1f} s, "
                                   "grids {64x64x32, 128x96x96, 256x128x192, 512x256x384} p {0.4,0.3,0.2,0.1}, "
                                   "8 fields, 50 ticks resident, 1e3-2e5 sources, HBM budget 150 GB",
                       "slots": args.serve_slots, "window_s": window, "measured_s": elapsed},
            "offered": {"value": offered / window, "unit": METRIC},
            "latency_s": {"p50": st["p50_latency_s"], "p99": st["p99_latency_s"], "mean": st["mean_latency_s"],
                          "note": "arrival to completion of completed requests; queueing dominates "
                                  "because the offered load exceeds the device's capacity"},
            "requests": {k: st[k] for k in ("submitted", "admitted", "completed", "rejected", "queued", "active",
                                            "rounds")},
            "hbm_peak_bytes": st["hbm_peak"], "busy_s": st["busy_s"], "device_s": st["device_s"],
            "rounds_per_s": st["rounds"] / max(elapsed, 1e-9)}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vfd", choices=["vfd", "reference"])
    ap.add_argument("--config", default="cfg1", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4"])
    ap.add_argument("--serve-window", type=float, default=5.0, help="cfg3: seconds of arrivals")
    ap.add_argument("--serve-grace", type=float, default=10.0, help="cfg3: seconds to keep measuring after")
    ap.add_argument("--serve-slots", type=int, default=16, help="cfg3: max resident requests")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-fields", type=int, default=2,
                    help="fields in the CPU-baseline sample (1 substep each)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-field path timing")
    args = ap.parse_args()
    if args.config == "cfg2" and args.impl == "vfd":
        run_cfg2(args)
        return
    if args.config == "cfg3" and args.impl == "vfd":
        run_cfg3(args)
        return
    c = cfg_by_name(args.config if args.config not in ("cfg2", "cfg3") else "cfg1")
    if args.impl == "reference":
        run_reference(args, c)
        return

    import numpy as np
    import torch

    import vfd
    from vfd import configs

    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local
    torch.cuda.set_device(dev)
    nx, ny, nz = c["grid"]
    V = nx * ny * nz
    nf = 8
    params = [vfd.field_params(s, d) for s, d in zip(c["sigma"], c["decay"])]
    world = vfd.World(nx, ny, nz, params, device=dev)
    ins = configs.field_inputs(c["seed"], rank, c["grid"], c["n_sources"])
    for f, (u, idx, amt) in enumerate(ins):
        world.upload(f, u)
        world.set_sources(f, idx, amt)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        world.tick(c["substeps"], stream=sh)
    torch.cuda.synchronize(dev)
    world.set_profiling(True)
    world.read_profile()
    barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    l0 = vfd.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        world.tick(c["substeps"], stream=sh)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    launches = vfd.launch_count() - l0
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    prof = world.read_profile()
    world.set_profiling(False)
    from vfd import dist as vd
    ms = vd.max_over_ranks(ms, device=f"cuda:{dev}")
    vsteps = V * nf * c["substeps"] * args.steps
    value = vd.aggregate_rate(vsteps, ms / 1e3, ws)

    # roofline of the dominant kernel (axis pass): 8 B per voxel per field per launch
    axis_ms = sum(prof[k][0] for k in ("x", "y", "z"))
    axis_n = sum(prof[k][1] for k in ("x", "y", "z"))
    avg_ms = axis_ms / max(axis_n, 1)
    alg_bytes = 8.0 * V * nf
    peak, peak_kind = peaks()
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": AXIS_TRAFFIC_BYTES,
                "kernel": "rf_col_kernel (y, z) / rf_row_kernel (x): axis passes",
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "peak_source": f"{peak_kind} hbm_gbs",
                "share_of_step": axis_ms / ms if ms > 0 else None,
                "per_pass_ms": {k: prof[k][0] / max(prof[k][1], 1) for k in prof}}

    # e2e through the host-buffer entry point (H2D + tick + D2H every step)
    pin_in = [torch.empty(V, dtype=torch.float32, pin_memory=True) for _ in range(nf)]
    pin_out = [torch.empty(V, dtype=torch.float32, pin_memory=True) for _ in range(nf)]
    host_in = [p.numpy() for p in pin_in]
    host_out = [p.numpy() for p in pin_out]
    for f in range(nf):
        host_in[f][:] = ins[f][0].ravel()
    world.diffuse_host(host_in, host_out, c["substeps"])
    barrier()
    torch.cuda.synchronize(dev)
    args.e2e_steps = max(1, args.e2e_steps)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        for f, (u, idx, amt) in enumerate(ins):
            world.set_sources(f, idx, amt)
        world.diffuse_host(host_in, host_out, c["substeps"])
    t_e2e = time.perf_counter() - t0
    t_e2e = vd.max_over_ranks(t_e2e, device=f"cuda:{dev}")
    e2e = {"value": ws * V * nf * c["substeps"] * args.e2e_steps / t_e2e, "unit": METRIC,
           "h2d_bytes_per_step": nf * V * 4 + sum(i.nbytes + a.nbytes for _, i, a in ins),
           "d2h_bytes_per_step": nf * V * 4,
           "api": "vfd_diffuse_host (pinned host buffers in and out, the diffuseChemGPU contract)",
           "steps": args.e2e_steps}

    # the plain per-field path on the same world (unfused kernels in the
    # reference's order, one field after another, no graph): one tick
    plain = None
    if not args.no_plain and ws == 1:
        pw = vfd.World(nx, ny, nz, params, device=dev, method=vfd.METHOD_PLAIN)
        for f, (u, idx, amt) in enumerate(ins):
            pw.upload(f, u)
            pw.set_sources(f, idx, amt)
        pw.tick(1, stream=sh)
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        pw.tick(c["substeps"], stream=sh)
        q1.record(stream)
        torch.cuda.synchronize(dev)
        plain = {"value": V * nf * c["substeps"] / (q0.elapsed_time(q1) / 1e3), "unit": METRIC,
                 "what": "VFD_METHOD_PLAIN: pad, R2C, C2C y, C2C z, multiply, C2C z, C2C y, C2R, crop as "
                         "separate kernels per field, no graph (1 tick)"}
        pw.close()

    line = None
    if rank == 0:
        cb = None
        if not args.no_cpu_baseline and ws == 1:
            cb = cpu_baseline(c, args.cpu_fields)
            cb.pop("seconds", None)
        try:
            bc = fft_contract_bytes(c)
            contract = {"bytes_per_voxel_step": bc, "achieved_gbs": value * bc / 1e9,
                        "frac": value * bc / 1e9 / peak, "peak": peak,
                        "what": "the whole step against the 5-sweep FFT-convolution byte count "
                                "(8 V + 64 Nc per field-substep, minimal padding); the roofline "
                                "above counts the 24 B per voxel-step the separable passes move"}
        except Exception as exc:  # reported, never fatal
            contract = {"error": repr(exc)}
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded counter-based generator)",
                "config": workload_config(c, world.fft_dims()), "roofline": roofline,
                "fft_contract_roofline": contract,
                "cpu_baseline": cb, "e2e": e2e, "plain_gpu": plain, "gpu_launches": launches,
                "clocks": clk}
    world.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
