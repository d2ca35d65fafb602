"""Project-written autotuner for the voxelizer's execution shape.

Two knobs change speed but not results (every candidate evaluates the same
(voxel, Gaussian) pairs of the same tile lists with the same arithmetic):

* execution tile shape -- a CTA covers the whole 8^3 binning tile (two
  8-voxel rows per lane) or a 4x8x8 half tile (one row per lane: fewer
  registers, twice the CTAs);
* Gaussian batch -- how many Gaussians a warp stages in shared memory at a
  time (8, 16 or 32);
* backward list split -- how many CTAs share one tile's Gaussian list in the
  backward (1, 2 or 4): more CTAs for volumes with too few tiles to fill
  the GPU.

``Autotuner.pick`` times every candidate's forward + backward on the binned
problem at hand with CUDA events and keeps the fastest, cached per
(volume shape, Gaussian-count bucket, backward mode); the cache can be
persisted as JSON.  The deterministic backward always runs whole tiles, so
only the forward takes the half-tile shape there.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import threading
from typing import Dict, Optional, Tuple

import torch

from ._lib import GsvGrads, GsvParams, GsvTuning, check, lib

# (rows per lane, Gaussian batch[, backward list split])
CANDIDATES: Tuple[Tuple[int, ...], ...] = ((2, 32), (2, 16), (1, 32), (1, 16), (1, 8), (2, 32, 2), (1, 32, 2),
                                           (1, 32, 4))
TILE_SIZES: Tuple[int, ...] = (8, 4)  # binning tile edges compared by pick_tile_size
WHOLE_TILE: Tuple[Tuple[int, int], ...] = ((2, 32), (2, 16), (2, 8))  # batched launches


def tuning_of(c) -> GsvTuning:
    """GsvTuning of a candidate or cache entry (rows per lane, batch[, split])."""
    return GsvTuning(int(c[0]), int(c[1]), 0, int(c[2]) if len(c) > 2 else 1)


def label_of(c) -> str:
    return "/".join(str(int(x)) for x in c) if len(c) > 2 and int(c[2]) > 1 else f"{int(c[0])}/{int(c[1])}"


def _ptr(t):
    return None if t is None or t.numel() == 0 else ctypes.c_void_p(t.data_ptr())


class Autotuner:
    def __init__(self, path: Optional[str] = None, reps: int = 3):
        self.path = path
        self.reps = reps
        self.cache: Dict[str, Tuple[int, int]] = {}
        self.timings: Dict[str, Dict[str, float]] = {}
        self._lock = threading.Lock()
        if path and os.path.exists(path):
            with open(path) as f:
                self.cache = {k: tuple(v) for k, v in json.load(f).items()}

    @staticmethod
    def key(shape, n: int, deterministic: bool) -> str:
        b = int(math.ceil(math.log2(max(n, 1))))
        return f"{shape.d}x{shape.h}x{shape.w}/ts{shape.tile_size}/n2^{b}/{'det' if deterministic else 'atomic'}"

    def save(self):
        if self.path:
            with open(self.path, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)

    def pick(self, plan, params, candidates=CANDIDATES) -> GsvTuning:
        """Tuning for a binned problem (a BinPlan and its parameter tensors)."""
        shape = plan.shape
        det = bool(plan.flags & 1)
        k = self.key(shape, plan.n, det) + ("" if candidates == CANDIDATES else "/" + ",".join(
            f"{a}.{b}" for a, b in candidates))
        with self._lock:
            if k in self.cache:
                return tuning_of(self.cache[k])
            if shape.tile_size != 8 or plan.n == 0 or plan.capacity == 0:
                self.cache[k] = (2, 32)
                return GsvTuning(2, 32)
            best, times = self._measure(plan, params, candidates)
            self.cache[k] = best
            self.timings[k] = times
            self.save()
            return tuning_of(best)

    def _measure(self, plan, params, candidates):
        dev = plan.device
        st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        vol = torch.empty((plan.shape.d, plan.shape.h, plan.shape.w), dtype=torch.complex64, device=dev)
        gvol = torch.randn_like(vol)
        outs = [torch.empty_like(t) for t in params]
        gp = GsvParams(*(t.data_ptr() for t in params), plan.n)
        gg = GsvGrads(*(o.data_ptr() for o in outs))
        times = {}
        for cand in candidates:
            tun = tuning_of(cand)

            def run():
                check(lib.gsv_forward_ex(plan.shape, plan.n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.capacity,
                                         _ptr(vol), ctypes.byref(tun), st), "gsv_forward_ex")
                check(lib.gsv_backward_ex(ctypes.byref(gp), plan.shape, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs),
                                          plan.capacity, _ptr(gvol), ctypes.byref(gg), plan.flags, ctypes.byref(tun),
                                          st), "gsv_backward_ex")

            run()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.reps):
                run()
            e1.record()
            torch.cuda.synchronize(dev)
            times[label_of(cand)] = e0.elapsed_time(e1) / self.reps
        best = min(candidates, key=lambda c: times[label_of(c)])
        return tuple(best), times


    def pick_tile_size(self, params, volume_shape, flags: int = 0) -> Tuple[int, GsvTuning, Dict[str, float]]:
        """Binning tile edge for a problem: times one whole step (preprocess,
        binning, forward, backward) at each edge of TILE_SIZES -- edge 8 with
        its best execution shape (pick), edge 4 on the generic one-voxel-per-
        thread kernels -- and keeps the fastest, cached like pick.  On a
        cubic volume the edges include the same (voxel, Gaussian) pairs and
        differ only by FP32 summation order.  On a non-cubic one the
        reference's radius 3 max_j(s_j hs_j) can cut a rotated anisotropic
        Gaussian at its tile box, and the cut depends on the edge: the
        included pairs then differ, as they do in the reference."""
        from .tile_voxelizer import _shape, prepare_and_bin

        n = int(params[0].shape[0])
        d, h, w = (int(x) for x in volume_shape)
        k = f"{d}x{h}x{w}/n2^{int(math.ceil(math.log2(max(n, 1))))}/{'det' if flags & 1 else 'atomic'}/tile"
        with self._lock:
            if k in self.cache:
                ts, *shape_t = self.cache[k]
                return int(ts), tuning_of(shape_t), self.timings.get(k, {})
        times, tunings = {}, {}
        dev = params[0].device
        st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        vol = torch.empty((d, h, w), dtype=torch.complex64, device=dev)
        gvol = torch.randn_like(vol)
        outs = [torch.empty_like(t) for t in params]
        gp = GsvParams(*(t.data_ptr() for t in params), n)
        gg = GsvGrads(*(o.data_ptr() for o in outs))
        for ts in TILE_SIZES:
            shape = _shape((d, h, w), ts)
            plan = prepare_and_bin(params, shape, flags)
            tun = self.pick(plan, params) if ts == 8 else GsvTuning(2, 32)
            tunings[ts] = tun

            def run():
                check(lib.gsv_prepare(ctypes.byref(gp), shape, _ptr(plan.ws_gauss), plan.gauss_bytes, None, st),
                      "gsv_prepare")
                check(lib.gsv_bin(shape, n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.pair_bytes,
                                  plan.capacity, st), "gsv_bin")
                check(lib.gsv_forward_ex(shape, n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.capacity,
                                         _ptr(vol), ctypes.byref(tun), st), "gsv_forward_ex")
                check(lib.gsv_backward_ex(ctypes.byref(gp), shape, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs),
                                          plan.capacity, _ptr(gvol), ctypes.byref(gg), flags, ctypes.byref(tun),
                                          st), "gsv_backward_ex")

            run()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.reps):
                run()
            e1.record()
            torch.cuda.synchronize(dev)
            times[str(ts)] = e0.elapsed_time(e1) / self.reps
        best = min(TILE_SIZES, key=lambda t: times[str(t)])
        with self._lock:
            t = tunings[best]
            self.cache[k] = (best, t.rows_per_lane, t.chunk, max(1, t.split))
            self.timings[k] = times
            self.save()
        return best, tunings[best], times


_default: Optional[Autotuner] = None


def default_tuner() -> Autotuner:
    """Process-wide tuner; GSV_AUTOTUNE_CACHE names an optional JSON cache."""
    global _default
    if _default is None:
        _default = Autotuner(os.environ.get("GSV_AUTOTUNE_CACHE"))
    return _default
