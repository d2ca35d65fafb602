#!/usr/bin/env python
"""Voxelizer forward+backward throughput (Gvox-evals/s) on one B200.

Workload (default ``mri128x128x96_n50k``): the 128x128x96 complex64 plain
3DGSMR reconstruction at its initial state -- a synthetic 10-ellipsoid
phantom with polynomial phase, 8 ring coils, R=6 variable-density mask with
a 24x24 calibration region, 1e-3 complex noise, and 50,000 Gaussians seeded
from the zero-filled image (random centres, 3-NN isotropic scale, identity
rotation, density 0.2 x image).  One step = preprocess + tile binning +
forward + backward of the voxelizer with a complex standard-normal upstream
gradient.  Units: candidate Gaussian-voxel evaluations E (sum over 8^3 tiles
of |list| x |voxels|) per second, forward+backward counted once.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``--impl reference`` times the CPU port of the reference's own CPU path
(oracle/torch_port.py) on the host cores.  Under torchrun every rank runs
an independent replica (the path has no cross-GPU exchange); rank 0 prints.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BATCH12_COILS = [4, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15, 16]
BATCH12_ACCEL = [4.0 + 4.0 * i / 11 for i in range(12)]
BATCH12 = [((96, 96, 96), 30_000), ((112, 112, 96), 100_000), ((128, 128, 96), 170_000),
           ((128, 128, 128), 240_000), ((144, 144, 112), 310_000), ((160, 160, 96), 380_000),
           ((160, 160, 128), 450_000), ((176, 176, 112), 520_000), ((192, 192, 128), 590_000),
           ((208, 208, 112), 660_000), ((224, 224, 96), 730_000), ((224, 224, 128), 800_000)]

WORKLOADS = {
    "mri128x128x96_n50k": dict(shape=(128, 128, 96), n=50_000, kind="from_image"),
    "batch12": dict(shape=None, n=sum(n for _, n in BATCH12), kind="batch"),
    # the same twelve volumes, each with its own coils (4-16) and mask (R 4-8): a whole
    # reconstruction iteration (SENSE data term, TV, Adam) per graph replay
    "batch12_recon": dict(shape=None, n=sum(n for _, n in BATCH12), kind="batch"),
    "mri128x128x96_n500k": dict(shape=(128, 128, 96), n=500_000, kind="from_image"),
    "cube64_n20k": dict(shape=(64, 64, 64), n=20_000, kind="random"),
    # the large reconstruction at its 2M-Gaussian cap (run with --deterministic)
    "mri256x256x160_n2m": dict(shape=(256, 256, 160), n=2_000_000, kind="phantom"),
}
TILE = 8
# Algorithmic FP32-pipe operations per candidate evaluation (forward 15,
# backward 33: recompute, cutoff test, density / centre / covariance terms).
OPS_FWD, OPS_BWD = 15, 33
SMS, LANES = 148, 128


def max_over_ranks(values, dist, device):
    """Per-rank device times -> their maximum over all ranks (replicas are
    timed by the slowest one)."""
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_rate(units_per_step, steps, world, total_ms):
    """Units processed by all replicas per second, timed by the slowest rank."""
    return units_per_step * steps * world / (total_ms * 1e-3)


def _synthetic(standalone=False):
    """The seeded-input generator (gs_tmi_b200/synthetic.py).  `standalone`:
    load the file on its own, without importing the package (whose import
    maps the product library) -- the reference arm uses no product code."""
    if not standalone:
        from gs_tmi_b200 import synthetic

        return synthetic
    import importlib.util

    name = "gsv_seeded_inputs"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "gs_tmi_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def make_inputs(name, standalone=False):
    synthetic = _synthetic(standalone)
    wl = WORKLOADS[name]
    if wl["kind"] == "from_image":
        case = synthetic.mri_case(wl["shape"], n_coils=8, accel=6.0, calib=24, seed=0)
        gs = synthetic.from_image_init(case.zero_filled, wl["n"], seed=0)
    elif wl["kind"] == "phantom":  # intensity-seeded on the phantom itself (no coil simulation)
        gs = synthetic.from_image_init(synthetic.ellipsoid_phantom(wl["shape"], seed=0), wl["n"], seed=0)
    else:
        gs = synthetic.random_gaussians(wl["n"], wl["shape"], seed=0)
    return gs, synthetic.upstream_grad(wl["shape"], seed=1)


def make_batch_inputs():
    """Twelve phantoms of uneven size, each with intensity-seeded Gaussians
    (30k..800k) and a complex standard-normal upstream gradient."""
    from gs_tmi_b200 import synthetic

    out = []
    for i, (shape, n) in enumerate(BATCH12):
        img = synthetic.ellipsoid_phantom(shape, seed=100 + i)
        gs = synthetic.from_image_init(img, n, seed=100 + i)
        out.append((shape, gs, synthetic.upstream_grad(shape, seed=200 + i)))
    return out


def run_batched(args, rank, world, dist):
    """One iteration = binning of all twelve volumes + ONE persistent forward
    launch + ONE persistent backward launch, captured as one CUDA graph."""
    from gs_tmi_b200 import batched
    from gs_tmi_b200.tile_voxelizer import TileVoxelizer

    local = int(os.environ.get("LOCAL_RANK", 0))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from gs_tmi_b200.autotune import WHOLE_TILE, Autotuner

    items = make_batch_inputs()
    caps, chunks, evals = [], [], 0
    tuner = Autotuner()
    for shape, gs, _ in items:
        vz = TileVoxelizer(shape, device=str(dev))
        total = vz.count_pairs(gs.positions.to(dev), gs.scales.to(dev))
        caps.append(int(total * 1.1) + 1024)
        params = tuple(t.to(dev) for t in gs.tensors())
        plan = __import__("gs_tmi_b200").prepare_and_bin(params, vz._shape)
        chunks.append(32 if args.no_autotune else tuner.pick(plan, params, WHOLE_TILE).chunk)
        tr_ptr, _ = plan.views()
        nt = lib_num_tiles(vz._shape)
        off = tr_ptr - plan.ws_gauss.data_ptr()
        tr = plan.ws_gauss[off:off + 8 * nt].view(torch.int32).reshape(-1, 2).cpu().numpy()
        evals += evals_of(tr, shape)
    sb = batched.StaticBatch([s for s, _, _ in items], [gs.n for _, gs, _ in items], caps, device=str(dev),
                             deterministic=args.deterministic, chunks=chunks)
    for i, (shape, gs, gv) in enumerate(items):
        for dst, src in zip(sb.params[i], gs.tensors()):
            dst.copy_(src.to(dev))
        sb.grad_volumes[i].copy_(gv.to(dev))
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for _ in range(2):
            sb.bin()
            sb.forward()
            sb.backward()
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize(dev)
    if any(sb.overflowed()):
        raise RuntimeError("pair capacity overflow in the batched benchmark")
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        sb.bin()
        sb.forward()
        sb.backward()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    cur = torch.cuda.current_stream(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(cur)
            graph.replay()
            ev[i][1].record(cur)
        torch.cuda.synchronize(dev)
    lat = sorted(a.elapsed_time(b) for a, b in ev)
    total_ms = sum(lat)
    total_ms, = max_over_ranks([total_ms], dist, dev)
    if rank != 0:
        return
    out = {"metric": "fwd+bwd Gvox-evals/s", "value": whole_job_rate(evals, args.steps, world, total_ms) / 1e9,
           "unit": "Gvox-evals/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp32", "data": "synthetic",
           "config": {"workload": "batch12", "volumes": [list(s) for s, _ in BATCH12],
                      "gaussians": [n for _, n in BATCH12], "tile_size": TILE, "evals_per_step": evals,
                      "autotuned_chunk_per_volume": chunks,
                      "launch": "per-volume binning + 1 persistent forward + 1 persistent backward (+finalize), "
                                "one CUDA graph per iteration",
                      "l2": "flushed between steps (256 MB write, untimed)", "parallelism": "replicas"},
           "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                          "min": lat[0], "max": lat[-1]},
           "clocks": clk.summary()}
    print(json.dumps(out), flush=True)


def run_batched_recon(args, rank, world, dist):
    """One iteration = exp(log-scales) + binning of all twelve volumes + ONE
    persistent forward launch + per volume the fused SENSE data term (coil
    product, FFT, masked residual, inverse FFT, adjoint coil sum) and TV +
    ONE persistent backward launch + log-scale chain rule, clipping and one
    fused Adam step over all volumes -- captured as one CUDA graph."""
    from gs_tmi_b200 import batched, synthetic
    from gs_tmi_b200.tile_voxelizer import TileVoxelizer

    local = int(os.environ.get("LOCAL_RANK", 0))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from gs_tmi_b200.autotune import WHOLE_TILE, Autotuner

    tuner = Autotuner()
    cases, inits, caps, chunks, evals = [], [], [], [], 0
    for i, (shape, n) in enumerate(BATCH12):
        case = synthetic.mri_case(shape, n_coils=BATCH12_COILS[i], accel=BATCH12_ACCEL[i], calib=24, seed=100 + i,
                                  device=dev)
        gs = synthetic.from_image_init(case.zero_filled.cpu(), n, seed=100 + i)
        vz = TileVoxelizer(shape, device=str(dev))
        params = tuple(t.to(dev) for t in gs.tensors())
        plan = __import__("gs_tmi_b200").prepare_and_bin(params, vz._shape)
        caps.append(int(plan.total * 2) + 4096)  # the Gaussians move during the timed iterations
        chunks.append(32 if args.no_autotune else tuner.pick(plan, params, WHOLE_TILE).chunk)
        tr_ptr, _ = plan.views()
        nt = lib_num_tiles(vz._shape)
        off = tr_ptr - plan.ws_gauss.data_ptr()
        tr = plan.ws_gauss[off:off + 8 * nt].view(torch.int32).reshape(-1, 2).cpu().numpy()
        evals += evals_of(tr, shape)
        cases.append(case)
        inits.append(gs)
        del plan
    rec = batched.BatchedRecon(cases, inits, caps, device=str(dev), deterministic=args.deterministic, chunks=chunks)
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for _ in range(2):
            rec.step()
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize(dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        rec.step()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    cur = torch.cuda.current_stream(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(cur)
            graph.replay()
            ev[i][1].record(cur)
        torch.cuda.synchronize(dev)
    if any(rec.sb.overflowed()):
        raise RuntimeError("pair capacity overflow in the batched reconstruction benchmark")
    lat = sorted(a.elapsed_time(b) for a, b in ev)
    total_ms = sum(lat)
    total_ms, = max_over_ranks([total_ms], dist, dev)
    if rank != 0:
        return
    out = {"metric": "fwd+bwd Gvox-evals/s", "value": whole_job_rate(evals, args.steps, world, total_ms) / 1e9,
           "unit": "Gvox-evals/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "fp32", "data": "synthetic",
           "config": {"workload": "batch12_recon", "volumes": [list(s) for s, _ in BATCH12],
                      "gaussians": [n for _, n in BATCH12], "coils": BATCH12_COILS,
                      "acceleration": [round(a, 2) for a in BATCH12_ACCEL], "tile_size": TILE,
                      "autotuned_chunk_per_volume": chunks,
                      "evals_per_step": evals, "deterministic": bool(args.deterministic),
                      "iteration": "exp(log-scales), binning x12, 1 persistent forward, SENSE data term + TV x12 "
                                   "(fused kernels + torch.fft), 1 persistent backward, clip x12, 1 fused Adam; "
                                   "one CUDA graph",
                      "l2": "flushed between steps (256 MB write, untimed)", "parallelism": "replicas"},
           "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                          "min": lat[0], "max": lat[-1]},
           "clocks": clk.summary()}
    print(json.dumps(out), flush=True)


def lib_num_tiles(gshape):
    from gs_tmi_b200._lib import lib

    return int(lib.gsv_num_tiles(gshape))


def evals_of(tr, shape):
    d, h, w = shape
    nth, ntw = -(-h // TILE), -(-w // TILE)
    e = 0
    for t in range(tr.shape[0]):
        td, rem = divmod(t, nth * ntw)
        th, tw = divmod(rem, ntw)
        nv = min(TILE, d - td * TILE) * min(TILE, h - th * TILE) * min(TILE, w - tw * TILE)
        e += int(tr[t, 1] - tr[t, 0]) * nv
    return e


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        # start timing only once the sampler is producing rows
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.path)
        if not rows:
            return None
        mhz = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows)}


def count_library_launches(fn, dev):
    """Kernels one call of `fn` launches, read from the CUDA activity trace."""
    try:
        from torch.profiler import ProfilerActivity, profile

        torch.cuda.synchronize(dev)
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize(dev)
        names = [e.name for e in prof.events() if e.device_type.name == "CUDA" and "Memset" not in e.name
                 and "Memcpy" not in e.name]
        return len(names), sorted(set(names))
    except Exception as exc:  # profiler unavailable: report unknown
        return None, [f"profiler unavailable: {exc}"]


def cpu_baseline(gs, gv, shape, seconds=12.0, warm=True):
    """CPU port of the reference's CPU path on a bounded random sample of
    tiles of the same workload, all host threads."""
    from oracle import oracle as O
    from oracle import torch_port

    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    p = tuple(t.numpy() for t in gs.tensors())
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    tr, pid = O.build_tile_pairs(c, r, shape, TILE)
    d, h, w = shape
    nt = tr.shape[0]
    order = np.random.default_rng(0).permutation(nt)
    per_tile = (tr[:, 1] - tr[:, 0]).astype(np.int64) * TILE ** 3  # interior tiles (shape divisible by 8)
    if warm:
        torch_port.time_fwd_bwd(p, shape, TILE, tr, pid, gv.numpy(), order[:2])
    done, evals, t_total, chunk = 0, 0, 0.0, 1
    while t_total < seconds and done < nt:
        tiles = order[done:done + chunk]
        t_total += torch_port.time_fwd_bwd(p, shape, TILE, tr, pid, gv.numpy(), tiles)
        evals += int(per_tile[tiles].sum())
        done += len(tiles)
        chunk = min(chunk * 2, 64)
    return {"value": evals / t_total / 1e9, "unit": "Gvox-evals/s", "cores": torch.get_num_threads(),
            "kind": "port", "seconds": t_total,
            "sample": f"{done} of {nt} tiles (random, seed 0) of the same workload, {evals} evals, "
                      f"{t_total:.1f} s, torch {torch.__version__} FP32 on host cores"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    name = args.workload
    gs, gv = make_inputs(name, standalone=True)
    shape = WORKLOADS[name]["shape"]
    vals, times = [], []
    steps, warm = args.steps, args.warmup
    # each step is a bounded sample so the whole run stays near 90 s of CPU work
    for i in range(warm + steps):
        b = cpu_baseline(gs, gv, shape, seconds=max(0.02, 90.0 / (steps + warm)), warm=(i == 0))
        if i >= warm:
            vals.append(b["value"])
            times.append(b["seconds"])
    v = statistics.mean(vals)
    out = {"metric": "fwd+bwd Gvox-evals/s", "value": v, "unit": "Gvox-evals/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
           "data": "synthetic", "impl": "reference",
           "config": {"workload": name, "volume": list(shape), "gaussians": WORKLOADS[name]["n"],
                      "tile_size": TILE, "parallelism": "replicas"},
           "cpu_baseline": dict(b, value=v),
           "e2e": {"value": v, "unit": "Gvox-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


class Workload:
    """One workload bound to the device: inputs, binning plan, tuned
    execution shape and the three phases of a step as closures."""

    def __init__(self, name, dev, args, flags):
        from gs_tmi_b200._lib import GsvGrads, GsvParams, check, lib
        from gs_tmi_b200.tile_voxelizer import _ptr, _shape, _stream, prepare_and_bin, work_census

        self.name, self.dev = name, dev
        self.shape = shape = WORKLOADS[name]["shape"]
        self.gs, self.gv = make_inputs(name)
        n = self.n = self.gs.n
        params = self.params = tuple(t.to(dev).contiguous() for t in self.gs.tensors())
        gvd = self.gvd = self.gv.to(dev).contiguous()
        gshape = _shape(shape, TILE)
        plan = self.plan = prepare_and_bin(params, gshape, flags)  # sizes the pair workspace (untimed sync)
        cap = plan.capacity
        self.total = plan.total
        outs = self.outs = [torch.empty_like(t) for t in params]
        vol = self.vol = torch.empty(shape, dtype=torch.complex64, device=dev)
        gp = GsvParams(*(t.data_ptr() for t in params), n)
        gg = GsvGrads(*(o.data_ptr() for o in outs))
        wsg, wsp = _ptr(plan.ws_gauss), _ptr(plan.ws_pairs)
        self.tuning, self.tune_times, self.tile_pick, self.tile_times = None, {}, None, {}
        if not args.no_autotune:
            from gs_tmi_b200.autotune import Autotuner

            tuner = Autotuner()
            self.tuning = tuner.pick(plan, params)  # untimed: times every execution shape once
            self.tune_times = next(iter(tuner.timings.values()), {})
            # the tile-edge comparison is reported; the workload's unit stays the reference's 8^3 tiles
            self.tile_pick, _, self.tile_times = tuner.pick_tile_size(params, shape, flags)
        tref = ctypes.byref(self.tuning) if self.tuning is not None else None

        # every launch goes to the stream current at call time (a graph capture's stream included)
        def prep_bin():
            st = _stream(dev)
            check(lib.gsv_prepare(ctypes.byref(gp), gshape, wsg, plan.gauss_bytes, None, st), "prepare")
            check(lib.gsv_bin(gshape, n, wsg, wsp, plan.pair_bytes, cap, st), "bin")

        def fwd():
            check(lib.gsv_forward_ex(gshape, n, wsg, wsp, cap, _ptr(vol), tref, _stream(dev)), "forward")

        def bwd():
            check(lib.gsv_backward_ex(ctypes.byref(gp), gshape, wsg, wsp, cap, _ptr(gvd), ctypes.byref(gg), flags,
                                      tref, _stream(dev)), "backward")

        self.prep_bin, self.fwd, self.bwd = prep_bin, fwd, bwd
        # E from the executed binning, and what the render kernels execute of it
        tr_ptr, _ = plan.views()
        ntiles = lib.gsv_num_tiles(gshape)
        off = tr_ptr - plan.ws_gauss.data_ptr()
        tr_host = plan.ws_gauss[off:off + 8 * ntiles].view(torch.int32).reshape(-1, 2).cpu().numpy()
        self.evals = evals_of(tr_host, shape)
        self.census = work_census(plan)

    def step(self):
        self.prep_bin()
        self.fwd()
        self.bwd()

    def capture(self):
        """The whole step as one CUDA graph: binning writes into the fixed
        pair capacity and nothing in the step synchronises the host, so it
        replays without CPU launch overhead."""
        dev = self.dev
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            self.step()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        g = torch.cuda.CUDAGraph()
        import warnings

        with warnings.catch_warnings():
            warnings.filterwarnings("error", message=".*Graph is empty.*")  # an empty capture: fail
            with torch.cuda.graph(g, stream=side):
                self.step()
        torch.cuda.synchronize(dev)
        return g

    def time_graph(self, graph, steps, warmup, flush):
        """Per-step device time (ms) of graph replays, L2 flushed between."""
        dev = self.dev
        for _ in range(warmup):
            graph.replay()
        torch.cuda.synchronize(dev)
        cur = torch.cuda.current_stream(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(cur)
            graph.replay()
            ev[i][1].record(cur)
        torch.cuda.synchronize(dev)
        _, fl = self.plan.read_status(torch_stream(dev))
        if fl:
            raise RuntimeError(f"voxelizer status flags {fl} during the timed region")
        return [a.elapsed_time(b) for a, b in ev]

    def time(self, steps, warmup, flush, dist=None):
        """Per-step device times (ms) of binning, forward and backward, CUDA
        events on the launching stream, L2 flushed between steps."""
        dev = self.dev
        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize(dev)
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
        cur = torch.cuda.current_stream(dev)
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(cur)
            self.prep_bin()
            ev[i][1].record(cur)
            self.fwd()
            ev[i][2].record(cur)
            self.bwd()
            ev[i][3].record(cur)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        _, fl = self.plan.read_status(torch_stream(dev))
        if fl:
            raise RuntimeError(f"voxelizer status flags {fl} during the timed region")
        return {"step": [ev[i][0].elapsed_time(ev[i][3]) for i in range(steps)],
                "bin": [ev[i][0].elapsed_time(ev[i][1]) for i in range(steps)],
                "fwd": [ev[i][1].elapsed_time(ev[i][2]) for i in range(steps)],
                "bwd": [ev[i][2].elapsed_time(ev[i][3]) for i in range(steps)]}

    def execution(self):
        if self.tuning is None:
            return "default"
        return {"rows_per_lane": self.tuning.rows_per_lane, "chunk": self.tuning.chunk,
                "backward_split": max(1, self.tuning.split),
                "autotune_ms_per_candidate": self.tune_times, "tile_edge_step_ms": self.tile_times,
                "tile_edge_fastest": self.tile_pick}


def torch_stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def roofline_of(wl, t, peak_ops, pk, pk_kind, sm_mhz):
    """FP32-issue roofline of the dominant kernel (the backward) on USEFUL
    work: the included candidates (Mahalanobis <= 9, counted on the device
    by the work census) times the algorithmic FP32 operations each one
    needs, over the backward's CUDA-event time.  Candidates outside the
    cutoff do no useful work, so they count nothing here."""
    d, h, w = wl.shape
    bwd_ms, fwd_ms = statistics.mean(t["bwd"]), statistics.mean(t["fwd"])
    useful = wl.census["included"]
    ach_bwd = useful * OPS_BWD / (bwd_ms * 1e-3)
    ach_fwd = useful * OPS_FWD / (fwd_ms * 1e-3)
    traffic, pipes = None, None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        rec = json.load(open(tpath)).get(wl.name, {})
        traffic, pipes = rec.get("k_backward8"), rec.get("k_backward8_pipes")
    vol_bytes = 2 * 8 * d * h * w  # write the volume, read its gradient
    c = wl.census
    return {"bound": "fp32_issue", "kernel": "gsv_backward (k_backward8 + k_finalize)",
            "achieved": ach_bwd / 1e12, "peak": peak_ops / 1e12, "unit": "TOP/s", "frac": ach_bwd / peak_ops,
            "traffic": traffic, "ops_per_eval": OPS_BWD, "units": "included candidates (m <= 9)",
            "units_per_launch": useful,
            "peak_source": f"{SMS} SMs x {LANES} FP32 lanes x sm_max_mhz {sm_mhz:.0f} ({pk_kind} peaks)",
            "forward": {"achieved": ach_fwd / 1e12, "frac": ach_fwd / peak_ops, "ops_per_eval": OPS_FWD},
            "work": {"candidates": wl.evals, "included": useful, "evaluated_after_cull": c["evaluated"],
                     "exp_block_lanes": c["exp_block_lanes"], "empty_kept_slots": c["empty_kept_slots"],
                     "lane_efficiency": useful / max(c["exp_block_lanes"], 1)},
            "pipes_ncu": pipes,
            "hbm": {"volume_gbs": vol_bytes / ((fwd_ms + bwd_ms) * 1e-3) / 1e9, "peak_gbs": pk.get("hbm_gbs")}}


def reference_cuda_baseline(wl, flush, reps):
    """The reference's own CUDA voxelizer (compiled from its sources into
    oracle/_ref/) on the same B200 and the same inputs: its forward and
    backward kernels alone, and its full step (torch preprocess, torch
    binning with the host sync, kernels, autograd tail), next to this
    build's kernels and full step through the public module.  Median of
    `reps` CUDA-event timings, L2 flushed before each."""
    try:
        from oracle import ref_cuda, torch_port
    except Exception as exc:  # noqa: BLE001
        return {"unavailable": f"reference extension not loadable: {exc}"}
    if ref_cuda.REF is None:
        return {"unavailable": "reference extension not built (oracle/build_ref.py needs the reference sources)"}
    import gs_tmi_b200

    REF = ref_cuda.REF
    dev, shape = wl.dev, wl.shape
    d, h, w = shape
    params, g = wl.params, wl.gvd
    with torch.no_grad():
        center, cov_inv, half = torch_port.preprocess(*params[:3], shape)
        tr, pid = torch_port.build_tile_pairs_torch(center, torch_port.radius_vox(params[1], half), shape, TILE)
    gr, gi = g.real.contiguous(), g.imag.contiguous()
    dr, di = params[3], params[4]

    def ref_kernels():
        REF.forward(center, cov_inv, dr, di, tr, pid, half, TILE, d, h, w)
        REF.backward(center, cov_inv, dr, di, tr, pid, half, gr, gi, TILE, d, h, w)

    def ref_full():
        ps = [p.detach().requires_grad_(True) for p in params]
        ref_cuda.reference_step(ps, shape, TILE).backward(g)

    def our_full():
        ps = [p.detach().requires_grad_(True) for p in params]
        gs_tmi_b200.voxelize(*ps, shape, TILE).backward(g)

    def timed(fn):
        fn()
        out = []
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(dev)
            out.append(e0.elapsed_time(e1))
        return statistics.median(out)

    r = {"ref_kernels_ms": timed(ref_kernels), "kernels_ms": timed(lambda: (wl.fwd(), wl.bwd())),
         "ref_full_step_ms": timed(ref_full), "full_step_ms": timed(our_full)}
    r["speedup_kernels"] = r["ref_kernels_ms"] / r["kernels_ms"]
    r["speedup_full_step"] = r["ref_full_step_ms"] / r["full_step_ms"]
    r["reps"] = reps
    r["what"] = ("kernels: forward + backward launches alone (this build: autotuned shape, atomic backward + "
                 "finalize to raw-parameter gradients; reference: its two kernels, gradients to center/cov_inv); "
                 "full step: preprocess + binning + forward + backward through each build's public module, "
                 "autograd included")
    return r


def run_ours(args, rank, world, dist):
    from gs_tmi_b200 import TileVoxelizer
    from gs_tmi_b200._lib import GSV_BACKWARD_DETERMINISTIC

    local = int(os.environ.get("LOCAL_RANK", 0))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    name = args.workload
    flags = GSV_BACKWARD_DETERMINISTIC if args.deterministic else 0
    wl = Workload(name, dev, args, flags)
    shape, gs, gv, n = wl.shape, wl.gs, wl.gv, wl.n
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize(dev)
    n_launch, kernel_names = (None, []) if args.no_launch_count else count_library_launches(wl.step, dev)

    graph = None if args.eager else wl.capture()
    with ClockSampler(local) as clk:
        # per-phase breakdown from eagerly launched steps; the headline from graph replays of the
        # same step (the launch mode of the graph-captured reconstruction loops) unless --eager
        t = wl.time(args.steps, args.warmup, flush, dist)
        eager_ms = sum(t["step"])
        if graph is not None:
            if dist:
                dist.barrier()
            total_ms = sum(wl.time_graph(graph, args.steps, args.warmup, flush))
            if dist:
                dist.barrier()
        else:
            total_ms = eager_ms

        # e2e through the public module with pinned host buffers
        vox = TileVoxelizer(shape, tile_size=TILE, device=str(dev), deterministic=args.deterministic,
                            autotune=not args.no_autotune)
        host_in = [x.pin_memory() for x in gs.tensors()]
        gv_host = gv.pin_memory()
        host_out = [torch.empty(x.shape, dtype=x.dtype).pin_memory() for x in gs.tensors()]
        vol_host = torch.empty(shape, dtype=torch.complex64).pin_memory()
        h2d = sum(x.numel() * x.element_size() for x in host_in) + gv_host.numel() * 8
        d2h = sum(x.numel() * x.element_size() for x in host_out) + vol_host.numel() * 8
        up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

        def e2e_step():
            # copies overlap compute the way a caller with two copy streams would run it:
            # the upstream gradient uploads during binning + forward, the volume downloads
            # during the backward
            main = torch.cuda.current_stream(dev)
            ps = [x.to(dev, non_blocking=True).requires_grad_(True) for x in host_in]
            up.wait_stream(main)
            with torch.cuda.stream(up):
                g = gv_host.to(dev, non_blocking=True)
            v = vox(ps[0], ps[1], ps[2], torch.complex(ps[3], ps[4]))
            down.wait_stream(main)
            with torch.cuda.stream(down):
                vol_host.copy_(v.detach(), non_blocking=True)
            main.wait_stream(up)
            g.record_stream(main)
            v.backward(g)
            for o, p in zip(host_out, ps):
                o.copy_(p.grad, non_blocking=True)
            main.wait_stream(down)

        for _ in range(args.warmup):
            e2e_step()
        torch.cuda.synchronize(dev)
        cur = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        e0.record(cur)
        for _ in range(args.steps):
            e2e_step()
        e1.record(cur)
        torch.cuda.synchronize(dev)
        e2e_ms = e0.elapsed_time(e1)

        total_ms, e2e_ms, eager_ms = max_over_ranks([total_ms, e2e_ms, eager_ms], dist, dev)
        extra = {}
        if rank == 0 and world == 1 and not args.no_extras:
            # the BASELINE voxelizer micro-benchmark (64^3, N = 20,000) on the same box
            if name != "cube64_n20k":
                small = Workload("cube64_n20k", dev, args, flags)
                ts_ = small.time(args.steps, args.warmup, flush)
                small_ms = sum(ts_["step"]) if args.eager else sum(
                    small.time_graph(small.capture(), args.steps, args.warmup, flush))
                extra["cube64_n20k"] = {
                    "value": small.evals * args.steps / (small_ms * 1e-3) / 1e9, "unit": "Gvox-evals/s",
                    "ms_per_step": small_ms / args.steps, "eager_ms_per_step": sum(ts_["step"]) / args.steps,
                    "evals_per_step": small.evals,
                    "breakdown_ms": {"prepare_bin": statistics.mean(ts_["bin"]),
                                     "forward": statistics.mean(ts_["fwd"]),
                                     "backward": statistics.mean(ts_["bwd"])},
                    "execution": small.execution(), "included": small.census["included"], "work": small.census}
                del small
            extra["reference_cuda"] = reference_cuda_baseline(wl, flush, reps=max(args.steps, 5))
    if rank != 0:
        return
    pk, pk_kind = peaks()
    clocks = clk.summary()
    sm_mhz = float(pk.get("sm_max_mhz", 1965.0))
    peak_ops = SMS * LANES * sm_mhz * 1e6
    evals = wl.evals
    value = whole_job_rate(evals, args.steps, world, total_ms) / 1e9
    out = {
        "metric": "fwd+bwd Gvox-evals/s", "value": value, "unit": "Gvox-evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": name, "volume": list(shape), "gaussians": n, "tile_size": TILE, "pairs": wl.total,
                   "evals_per_step": evals, "deterministic": bool(args.deterministic),
                   "execution": wl.execution(),
                   "launch": "eager" if graph is None else "one CUDA graph per step (preprocess, binning, "
                                                           "forward, backward)",
                   "l2": "flushed between steps (256 MB write, untimed)", "parallelism": "replicas"},
        "eager_ms_per_step": eager_ms / args.steps,
        "breakdown_ms": {"prepare_bin": statistics.mean(t["bin"]), "forward": statistics.mean(t["fwd"]),
                         "backward": statistics.mean(t["bwd"]), "launch": "eager"},
        "roofline": roofline_of(wl, t, peak_ops, pk, pk_kind, sm_mhz),
        "e2e": {"value": whole_job_rate(evals, args.steps, world, e2e_ms) / 1e9, "unit": "Gvox-evals/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms / args.steps,
                "api": "gs_tmi_b200.TileVoxelizer forward + autograd backward; upstream-gradient upload and "
                       "volume download on copy streams overlapping the forward / backward"},
        "gpu_launches": None if n_launch is None else n_launch * args.steps,
        "launches_per_step": n_launch, "kernels": kernel_names,
        "clocks": clocks,
    }
    out.update({k: v for k, v in extra.items()})
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(gs, gv, shape)
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="mri128x128x96_n50k")
    ap.add_argument("--deterministic", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-launch-count", action="store_true", help="skip the CUDA activity trace (under ncu)")
    ap.add_argument("--no-autotune", action="store_true", help="default execution shape, no tuning pass")
    ap.add_argument("--eager", action="store_true", help="time eagerly launched steps instead of graph replays")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the 64^3 line and the reference-CUDA baseline (under ncu)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "batch12":
            run_batched(args, rank, world, dist)
        elif args.workload == "batch12_recon":
            run_batched_recon(args, rank, world, dist)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
