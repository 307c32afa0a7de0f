#!/usr/bin/env python
"""Throughput of the cytokine-diffusion tick on B200.

Workload (default): the human-scale world -- 8 fp32 fields on a 512x256x384
grid (x fastest), Gaussian sigma = 1.5 x (1.2, 0.9, 1.0, 0.8, 1.1, 1.0, 1.3,
0.9), decay (0.05, 0.01, 0.02, 0.03, 0.05, 0.04, 0.06, 0.02) per substep,
200k lognormal(-6, 1) point sources per field, zero padding, seed 0.
One step = one tick = 10 diffusion substeps of all 8 fields + source deposit
+ FP64 totals.  Metric: voxel-steps/s (data voxels x fields x substeps / s).

  python bench.py [--gpus N --steps K --warmup W] [--impl vfd|reference]
                  [--config cfg1|cfg2|cfg3|cfg4] [--quick]

At N = 1 the line also carries the other configurations' figures (the
32-world batched ensemble, the served request stream, the general 3D path
the Diffuser drop-in runs) and, outside the timed region, the baseline and
checker leg: the FP32 CPU port timed on the host cores, the per-field error
against the FP64 oracle, and the reference's own GPU kernels + cuFFT.

N > 1 runs under torchrun: every rank diffuses its own world (config 1) or
its own share of the ensemble's worlds (config 2) -- independent units, no
data-path collective, weak scaling; the time is the max over ranks.
`--impl reference` times the CPU restatement of the path (the reference has
no runnable CPU diffusion) on rank 0 only.
"""
import argparse
import json
import math
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
# ncu dram__bytes_read.sum + dram__bytes_write.sum per axis-pass launch,
# averaged over x, y, z (10.89 GB per launch on the 8 x 768x384x576 world,
# profiles/rf_tma_pass_512x256x128.md), scaled to the human-scale world by
# its voxel count (the passes read and write every voxel once).
AXIS_TRAFFIC_BYTES = 3.23e9

# The configurations, written out here so that the reference arm and the CPU
# sample need no import of the product package (vfd/configs.py holds the
# same values).
SIGMA0 = [1.2, 0.9, 1.0, 0.8, 1.1, 1.0, 1.3, 0.9]
DECAY0 = [0.05, 0.01, 0.02, 0.03, 0.05, 0.04, 0.06, 0.02]
CONFIGS = {
    "cfg0": dict(name="plain-small-64x64x32", grid=(64, 64, 32), sigma=SIGMA0, decay=DECAY0,
                 n_sources=500, substeps=1, seed=0),
    "cfg1": dict(name="human-scale-512x256x384", grid=(512, 256, 384), sigma=[1.5 * s for s in SIGMA0],
                 decay=DECAY0, n_sources=200_000, substeps=10, seed=0),
    "cfg4": dict(name="large-768x384x576", grid=(768, 384, 576), sigma=[2.0 * s for s in SIGMA0],
                 decay=DECAY0, n_sources=1_000_000, substeps=10, seed=0),
}


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


def radius(s):
    return int(math.ceil(3.0 * s - 1e-12))


def fft_contract_bytes(c):
    """Bytes per voxel-step of the canonical 5-sweep 3D FFT convolution
    (8 V + 64 Nc per field and substep, Nc = Fz Fy (Fx / 2 + 1) on the
    minimal padded grid F = n + 2 r per axis, plus 8 B per source deposited
    once per tick), averaged over the world's fields."""
    nx, ny, nz = c["grid"]
    V = nx * ny * nz
    tot = 0.0
    for s in c["sigma"]:
        r = radius(s)
        fx, fy, fz = nx + 2 * r, ny + 2 * r, nz + 2 * r
        nc = fz * fy * (fx // 2 + 1)
        tot += 8.0 * V + 64.0 * nc + 8.0 * c["n_sources"] / c["substeps"]
    return tot / len(c["sigma"]) / V


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


# ---------------------------------------------------------------------------
# Baseline and checker leg (outside every timed region of the product):
# the FP32 CPU port timed on the host cores, the per-field error against the
# FP64 oracle, and the reference's own GPU kernels + cuFFT.  The only code in
# this file that runs anything under oracle/.
# ---------------------------------------------------------------------------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def cpu_sample_inputs(c, seed=12345):
    """Fields and sources with the workload's shapes and distributions (U[0,
    1e-3) values, uniform voxels, lognormal(-6, 1) strengths), from numpy:
    the CPU sample loads no product library."""
    import numpy as np
    rng = np.random.default_rng(seed)
    nx, ny, nz = c["grid"]
    V = nx * ny * nz
    out = []
    for _ in range(len(c["sigma"])):
        u = (rng.random((nz, ny, nx), dtype=np.float32) * np.float32(1e-3)).astype(np.float32)
        idx = rng.integers(0, V, c["n_sources"], dtype=np.int32)
        amt = rng.lognormal(-6.0, 1.0, c["n_sources"]).astype(np.float32)
        out.append((u, idx, amt))
    return out


def cpu_sample(c, inputs, nthreads=0):
    """One substep of every field of the workload plus its deposit, FP32
    OpenMP port (oracle/vfd_cpu_port.c); returns voxel-steps/s and seconds."""
    oracle = _oracle()
    nx, ny, nz = c["grid"]
    t0 = time.perf_counter()
    for f, (u, idx, amt) in enumerate(inputs):
        s = c["sigma"][f]
        oracle.port_substep(u, (s, s, s), (radius(s),) * 3, c["decay"][f], nthreads=nthreads)
        oracle.port_deposit_total(u, idx, amt)
    dt = time.perf_counter() - t0
    vs = nx * ny * nz * len(inputs)
    return vs / dt, dt, vs


def cpu_baseline(c, min_seconds=10.0):
    """The CPU sample repeated for about min_seconds on all host threads."""
    oracle = _oracle()
    ins = cpu_sample_inputs(c)
    tot_t, tot_v, reps = 0.0, 0, 0
    while tot_t < min_seconds or reps == 0:
        _, dt, vs = cpu_sample(c, ins)
        tot_t += dt
        tot_v += vs
        reps += 1
    nx, ny, nz = c["grid"]
    return {"value": tot_v / tot_t, "unit": METRIC, "cores": oracle.port_threads(), "kind": "port",
            "sample": f"all 8 fields of the {nx}x{ny}x{nz} world x 1 substep + deposit "
                      f"({tot_v / reps / 1e6:.0f} M voxel-steps), FP32 separable direct convolution, "
                      f"OpenMP, repeated {reps}x ({tot_t:.1f} s)"}


def parity_leg(c, dev):
    """Per field: relative L2, max-abs error and mass error of one tick
    (config 1: 10 substeps + deposit) against the FP64 oracle."""
    import numpy as np

    import vfd
    oracle = _oracle()
    nx, ny, nz = c["grid"]
    V = nx * ny * nz
    params = [vfd.field_params(s, d) for s, d in zip(c["sigma"], c["decay"])]
    out = []
    with vfd.World(nx, ny, nz, params, device=dev) as w:
        srcs = []
        for f in range(8):
            u = vfd.synth_field(c["seed"], 0, f, (nz, ny, nx))
            idx, amt = vfd.synth_sources(c["seed"], 0, f, c["n_sources"], V)
            w.upload(f, u)
            w.set_sources(f, idx, amt)
            srcs.append((u, idx, amt))
        w.tick(c["substeps"])
        mass = w.mass()
        for f, (u, idx, amt) in enumerate(srcs):
            got = w.download(f).astype(np.float64)
            ref, _ = oracle.tick_mt(u, c["sigma"][f], c["decay"][f], c["substeps"], idx, amt)
            d = got - ref
            rel = float(np.sqrt((d * d).sum() / (ref * ref).sum()))
            s = got.sum()
            out.append({"field": f, "rel_l2": rel, "max_abs": float(np.abs(d).max()),
                        "max_abs_over_max_ref": float(np.abs(d).max() / np.abs(ref).max()),
                        "mass_rel_err": abs(mass[f]["total"] - s) / abs(s)})
    return {"against": "FP64 oracle (separable direct sums, oracle.tick_mt), one tick of 10 substeps "
                       "+ deposit, all 8 fields at full size",
            "bar": {"rel_l2": 1e-5, "mass_rel_err": 1e-6},
            "max_rel_l2": max(x["rel_l2"] for x in out), "per_field": out}


def ref_gpu_leg(iters=3):
    """The reference's own kernels + cuFFT (oracle/_ref/libref_replay.so,
    compiled from its convolutionFFT.cu) on one field of the human-scale
    world, in fftDiffuse3D's order, on its power-of-two grid: kernels only,
    and as the reference calls them each tick (plans and buffers re-created,
    Diffuser.cpp:273-274, Diffusion.cu:1686-1687)."""
    import ctypes as C

    import numpy as np
    oracle = _oracle()
    if not oracle.ref_replay_available():
        return {"unavailable": "oracle/_ref/libref_replay.so not built (no reference tree at build time)"}
    c = CONFIGS["cfg1"]
    nx, ny, nz = c["grid"]
    sigma = c["sigma"][6]
    r = radius(sigma)
    t = oracle.gauss_taps(sigma, r)
    win = np.ascontiguousarray(np.einsum("z,y,x->zyx", t, t, t).astype(np.float32))
    k = 2 * r + 1

    def snap(n):  # snapTransformSize, Diffusion.cu:39-70
        n16 = (n + 15) // 16 * 16
        p = 1
        while p < n16:
            p *= 2
        return p
    fx, fy, fz = snap(nx + k - 1), snap(ny + k - 1), snap(nz + k - 1)
    L = C.CDLL(oracle.REF_REPLAY)
    f = L.ref_replay_time
    f.argtypes = [C.c_int] * 6 + [C.c_void_p] + [C.c_int] * 7 + [C.c_float, C.c_int, C.c_void_p]
    f.restype = C.c_int
    ms = (C.c_double * 2)()
    rc = f(nz, ny, nx, fz, fy, fx, win.ctypes.data, k, k, k, r, r, r, nx, 0.0, iters, ms)
    if rc != 0:
        return {"error": f"ref_replay_time returned {rc}"}
    V = nx * ny * nz
    return {"what": "the reference's convolutionFFT.cu kernels + cuFFT (fftDiffuse3D's order), one field of "
                    "the 512x256x384 world, sigma 1.95, one substep",
            "fft": [fx, fy, fz],
            "kernels_only": {"value": V / (ms[0] / 1e3), "unit": METRIC, "ms": ms[0]},
            "as_called_per_tick": {"value": V / (ms[1] / 1e3), "unit": METRIC, "ms": ms[1]}}


def run_reference(args, c):
    """--impl reference: the CPU restatement on the host cores (rank 0 only)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    oracle = _oracle()
    ins = cpu_sample_inputs(c)
    for _ in range(args.warmup):
        cpu_sample(c, ins)
    tot_t, tot_v = 0.0, 0
    for _ in range(args.steps):
        _, dt, vs = cpu_sample(c, ins)
        tot_t += dt
        tot_v += vs
    value = tot_v / tot_t
    nx, ny, nz = c["grid"]
    sample = (f"all 8 fields of the {nx}x{ny}x{nz} world x 1 substep + deposit per step "
              f"({tot_v / args.steps / 1e6:.0f} M voxel-steps), FP32 separable direct convolution, OpenMP")
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (numpy, seeded)",
            "config": workload_config(c), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": oracle.port_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's CPU diffusion (Diffuser::diffuseChemCPU) does not run; "
                    "this arm times the FP32 OpenMP restatement of the same method"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# The other configurations (N = 1 keys of the default line, or --config)
# ---------------------------------------------------------------------------
def run_cfg2(args, dev=0, quiet=False):
    """Batched ensemble: 32 uneven worlds x 8 fields, 10 substeps per tick, all
    fields of the rank's worlds in one launch per axis pass, the pass of
    each axis chosen by vfd_batch_autotune, the tick replayed as a CUDA graph.
    Beside it: the same worlds through the plain per-field path
    (VFD_METHOD_PLAIN: unfused kernels, one field at a time, no graph).
    Under torchrun the worlds are sharded round-robin over the ranks."""
    import torch

    import vfd
    from vfd import configs
    from vfd import dist as vd
    ws, rank, _ = dist_env()
    torch.cuda.set_device(dev)
    c = configs.CFG2
    specs = configs.cfg2_worlds(c["n_worlds"], c["seed"])
    mine = [specs[i] for i in vd.shard(len(specs), rank, ws)]
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def build(method):
        out = []
        for sp in mine:
            nx, ny, nz = sp["grid"]
            params = [vfd.field_params(s_, d_) for s_, d_ in zip(sp["sigma"], sp["decay"])]
            w = vfd.World(nx, ny, nz, params, method=method, device=dev)
            for f, (u, idx, amt) in enumerate(configs.field_inputs(c["seed"], sp["world"], sp["grid"],
                                                                     sp["n_sources"])):
                w.upload(f, u)
                w.set_sources(f, idx, amt)
            out.append(w)
        return out

    vox = sum(configs.voxels(sp["grid"]) for sp in mine) * 8 * c["substeps"]
    worlds = build(vfd.METHOD_SEPARABLE)
    batch = vfd.Batch(worlds)
    t0 = time.perf_counter()
    tuning = batch.autotune(reps=3)
    tune_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        batch.tick(c["substeps"], stream=sh)
    torch.cuda.synchronize(dev)
    vd.barrier()
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
    ms = vd.max_over_ranks(e0.elapsed_time(e1), device=f"cuda:{dev}")
    # whole job: the voxel-steps of every rank's worlds over the slowest rank's time
    value = vd.sum_over_ranks(vox * args.steps, device=f"cuda:{dev}") / (ms / 1e3)
    # the sum of the per-pass times against the graph's tick time: the cost
    # of the launch boundaries inside the graph
    pass_ms = sum(t["ms"] for t in tuning) * c["substeps"]
    batch.close()
    for w in worlds:
        w.close()
    res = {"value": value, "unit": METRIC, "ms_per_tick": ms / args.steps,
           "launches_per_tick": launches / args.steps, "tuning": tuning, "autotune_s": tune_s,
           "graph_vs_pass_sum": {"tick_ms": ms / args.steps, "pass_ms_sum": pass_ms,
                                 "gap_frac": 1.0 - pass_ms / (ms / args.steps)},
           "clocks": clk, "worlds": len(mine)}
    if ws == 1:
        # plain per-field path, one world at a time (bounded: 1 tick)
        plain_ms = 0.0
        for sp in mine:
            nx, ny, nz = sp["grid"]
            params = [vfd.field_params(s_, d_) for s_, d_ in zip(sp["sigma"], sp["decay"])]
            w = vfd.World(nx, ny, nz, params, method=vfd.METHOD_PLAIN, device=dev)
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
        peak, kind = peaks()
        achieved = 24.0 * value / 1e9
        res.update({"plain_gpu": {"value": plain, "unit": METRIC,
                                  "what": "VFD_METHOD_PLAIN: unfused pad/R2C/C2C/multiply/C2C/C2R/crop kernels, "
                                          "one field per launch sequence, no graph"},
                    "batched_over_plain": value / plain,
                    "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                 "frac": achieved / peak, "peak_source": f"{kind} hbm_gbs",
                                 "note": "whole tick, 24 B per voxel-step (3 axis passes x 8 B)"}})
    return res


def run_cfg3(args, dev=0):
    """Served requests: open-loop Poisson arrivals (precomputed from the seed)
    at 200 req/s for a fixed window; grids drawn from {64x64x32, 128x96x96,
    256x128x192, 512x256x384} with p = {0.4, 0.3, 0.2, 0.1}; 8 fields, 50
    single-substep ticks resident per request, 1e3..2e5 sources per request
    (split over the fields), HBM budget 150 GB.  Measured until every
    request has completed or the grace period ends; latency percentiles are
    over every arrival (a request still unfinished at the end counts with the
    time it has waited so far, a lower bound)."""
    import numpy as np

    import vfd
    from vfd import configs
    from vfd import dist as vd
    ws, rank, _ = dist_env()
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
    mine = [arrivals[i] for i in vd.shard(len(arrivals), rank, ws)]
    server = vfd.Server(c["hbm_budget_bytes"], max_active=args.serve_slots, substeps_per_tick=1, device=dev)
    params = [vfd.field_params(s_, d_) for s_, d_ in zip(configs.SIGMA0, configs.DECAY0)]
    offered = 0.0
    ids = []
    t0 = server.clock()
    for k, (ta, g, nsrc) in enumerate(mine):
        while server.clock() - t0 < ta:
            time.sleep(0.0005)
        nx, ny, nz = g
        per = [nsrc // 8 + (1 if f < nsrc % 8 else 0) for f in range(8)]
        srcs = [vfd.synth_sources(c["seed"], 1000 + k, f, per[f], nx * ny * nz) for f in range(8)]
        ids.append(server.submit(g, params, c["ticks_per_request"], synth=(c["seed"], 1000 + k, 0.0, 1e-3),
                                 sources=srcs))
        offered += nx * ny * nz * 8 * c["ticks_per_request"]
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
    return {"value": sustained, "unit": METRIC,
            "offered": {"value": offered / window, "unit": METRIC},
            "window_s": window, "measured_s": elapsed, "slots": args.serve_slots,
            "latency_s": {"p50": st["p50_latency_s"], "p99": st["p99_latency_s"], "mean": st["mean_latency_s"],
                          "p50_completed": st["p50_completed_s"], "p99_completed": st["p99_completed_s"],
                          "censored": st["censored"],
                          "note": "arrival to completion over every arrival; queueing dominates because the "
                                  "offered load exceeds the device's capacity"},
            "requests": {k: st[k] for k in ("submitted", "admitted", "completed", "rejected", "queued", "active",
                                            "rounds")},
            "device_busy_frac": st["device_s"] / elapsed if elapsed > 0 else None,
            "hbm_peak_bytes": st["hbm_peak"], "busy_s": st["busy_s"], "device_s": st["device_s"],
            "host_s": {"batch": st["host_batch_s"], "admit": st["host_admit_s"], "wait": st["host_wait_s"]}}


def run_fft3d(c, dev, stream, steps=3):
    """The general 3D FFT path (VFD_METHOD_FFT3D: fused pruned R2C / C2C /
    C2R with the stored spectrum multiply), the transform the Diffuser
    drop-in runs, on the human-scale grid with the reference's constant-VF
    padding (epiBoundary = nx - 1, baseline 1e-4), 8 fields, one substep per
    tick, against the 5-sweep byte count of that transform."""
    import torch

    import vfd
    nx, ny, nz = c["grid"]
    params = [vfd.field_params(s, d, baseline=1e-4) for s, d in zip(c["sigma"], c["decay"])]
    with vfd.World(nx, ny, nz, params, method=vfd.METHOD_FFT3D, pad_mode=vfd.PAD_CONSTANT_VF,
                   epi_boundary=nx - 1, device=dev) as w:
        for f in range(8):
            w.upload(f, vfd.synth_field(c["seed"], 0, f, (nz, ny, nx)))
        fft = w.fft_dims()
        w.tick(1, stream=stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            w.tick(1, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / steps
        # per-pass device time of one more tick (CUDA events per pass, outside the timed region)
        w.set_profiling(True)
        w.read_profile()
        w.tick(1, stream=stream.cuda_stream)
        torch.cuda.synchronize(dev)
        prof = w.read_profile()
        w.set_profiling(False)
        # through the host-buffer entry point, as the Diffuser drop-in's
        # diffuseChemGPU calls it: pinned pChem in, tChem out, every tick
        Vn = nx * ny * nz
        pin_in = [torch.empty(Vn, dtype=torch.float32, pin_memory=True) for _ in range(8)]
        pin_out = [torch.empty(Vn, dtype=torch.float32, pin_memory=True) for _ in range(8)]
        host_in = [p.numpy() for p in pin_in]
        host_out = [p.numpy() for p in pin_out]
        for f in range(8):
            host_in[f][:] = vfd.synth_field(c["seed"], 0, f, (nz, ny, nx)).ravel()
        w.diffuse_host(host_in, host_out, 1)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(steps):
            w.diffuse_host(host_in, host_out, 1)
        t_host = (time.perf_counter() - t0) / steps
        del pin_in, pin_out, host_in, host_out
    V = nx * ny * nz
    fx, fy, fz = fft
    nc = fz * fy * (fx // 2 + 1)
    alg = 8 * (8.0 * V + 64.0 * nc)
    peak, kind = peaks()
    return {"value": 8 * V / (ms / 1e3), "unit": METRIC, "ms_per_substep": ms, "fft": list(fft),
            "per_pass_ms": {a: prof[a][0] for a in ("x", "y", "z")},
            "e2e": {"value": 8 * V / t_host, "unit": METRIC, "ms_per_tick": t_host * 1e3,
                    "h2d_bytes_per_step": 8 * V * 4, "d2h_bytes_per_step": 8 * V * 4,
                    "api": "vfd_diffuse_host, 1 substep (the drop-in's diffuseChemGPU contract), pinned buffers"},
            "what": "VFD_METHOD_FFT3D, constant-VF padding, 8 fields x 1 substep per tick",
            "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "peak_source": f"{kind} hbm_gbs",
                         "alg_bytes_per_substep": alg,
                         "note": "8 V + 64 Nc per field (5 sweeps of the transform's data)"}}


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vfd", choices=["vfd", "reference"])
    ap.add_argument("--config", default="cfg1", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4"])
    ap.add_argument("--serve-window", type=float, default=3.0, help="cfg3: seconds of arrivals")
    ap.add_argument("--serve-grace", type=float, default=40.0, help="cfg3: seconds to keep measuring after")
    ap.add_argument("--serve-slots", type=int, default=16, help="cfg3: max resident requests")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--quick", action="store_true",
                    help="only the configuration's own figures: no other configurations, no baseline leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-field path timing")
    args = ap.parse_args()
    cname = args.config if args.config in CONFIGS else "cfg1"
    c = CONFIGS[cname]
    if args.impl == "reference":
        run_reference(args, c)
        return

    import torch

    import vfd
    from vfd import configs
    from vfd import dist as vd

    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local
    torch.cuda.set_device(dev)

    if args.config in ("cfg2", "cfg3"):
        res = run_cfg2(args, dev) if args.config == "cfg2" else run_cfg3(args, dev)
        if rank == 0:
            wl = ("batched ensemble: 32 worlds drawn from {96x64x64, 128x96x96, 192x128x128, 256x128x192} x 8 "
                  "fields, 10 substeps per step, 500 sources/field, sigma and decay x U[0.5, 2], seed 0"
                  if args.config == "cfg2" else
                  "served requests: Poisson 200 req/s, grids {64x64x32, 128x96x96, 256x128x192, 512x256x384} "
                  "p {0.4,0.3,0.2,0.1}, 8 fields, 50 ticks resident, 1e3-2e5 sources, HBM budget 150 GB")
            line = {"metric": METRIC, "value": res["value"], "unit": METRIC, "n_gpus": ws,
                    "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": res.get("ms_per_tick"), "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded counter-based generator)",
                    "config": {"workload": wl, "l2": "inputs larger than L2"}, args.config: res,
                    "roofline": res.get("roofline"), "clocks": res.get("clocks")}
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

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
    ms = vd.max_over_ranks(ms, device=f"cuda:{dev}")
    vsteps = V * nf * c["substeps"] * args.steps
    value = vd.aggregate_rate(vsteps, ms / 1e3, ws)

    # roofline of the dominant kernels (the three axis passes, 8 B per voxel
    # per field per launch; per-launch CUDA events on the launching stream)
    axis_ms = sum(prof[k][0] for k in ("x", "y", "z"))
    axis_n = sum(prof[k][1] for k in ("x", "y", "z"))
    avg_ms = axis_ms / max(axis_n, 1)
    alg_bytes = 8.0 * V * nf
    peak, peak_kind = peaks()
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    per_pass = {k: prof[k][0] / max(prof[k][1], 1) for k in prof}
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": AXIS_TRAFFIC_BYTES,
                "kernel": "axis passes: rf_row_tma_kernel (x), rf_col_tma_kernel (y, z)",
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "peak_source": f"{peak_kind} hbm_gbs",
                "share_of_step": axis_ms / ms if ms > 0 else None,
                "per_pass_ms": per_pass,
                "per_pass_frac": {k: alg_bytes / (per_pass[k] / 1e3) / 1e9 / peak for k in ("x", "y", "z")}}

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
    del pin_in, pin_out, host_in, host_out

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
    world.close()
    del ins

    extras = {}
    if ws == 1 and not args.quick:
        for key, fn in (("fft3d", lambda: run_fft3d(c, dev, stream)),
                        ("cfg2", lambda: run_cfg2(argparse.Namespace(steps=5, warmup=3), dev)),
                        ("cfg3", lambda: run_cfg3(args, dev))):
            try:
                extras[key] = fn()
            except Exception as exc:  # reported, never fatal
                extras[key] = {"error": repr(exc)}

    line = None
    if rank == 0:
        cb, parity, ref_gpu = None, None, None
        if ws == 1 and not args.quick and not args.no_cpu_baseline:
            for key in ("cpu_baseline", "parity", "ref_gpu"):
                try:
                    if key == "cpu_baseline":
                        cb = cpu_baseline(c)
                    elif key == "parity":
                        parity = parity_leg(c, dev)
                    else:
                        ref_gpu = ref_gpu_leg()
                except Exception as exc:  # reported, never fatal
                    if key == "cpu_baseline":
                        cb = {"error": repr(exc)}
                    elif key == "parity":
                        parity = {"error": repr(exc)}
                    else:
                        ref_gpu = {"error": repr(exc)}
        bc = fft_contract_bytes(c)
        contract = {"bytes_per_voxel_step": bc, "effective_gbs": value * bc / 1e9,
                    "speedup_over_contract_at_peak": value * bc / 1e9 / peak,
                    "what": "the 5-sweep FFT-convolution byte count (8 V + 64 Nc per field-substep, minimal "
                            "padding): a transform-based step that moved those bytes at the measured copy "
                            "bandwidth would run this many times slower than this step"}
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded counter-based generator)",
                "config": workload_config(c), "roofline": roofline, "fft_contract": contract,
                "cpu_baseline": cb, "e2e": e2e, "plain_gpu": plain, "gpu_launches": launches,
                "clocks": clk, "parity": parity, "ref_gpu": ref_gpu}
        line.update(extras)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
