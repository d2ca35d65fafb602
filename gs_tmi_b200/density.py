"""Adaptive density control on the device, and the graph-replayed fit that
uses it.

The reference densifies on the host (trainer.py:294-424,
gaussian_model.py:85-222): every split, clone or prune re-creates the five
nn.Parameters, rebuilds the Adam optimizer and transplants its moments,
with several `.item()` synchronisations on the way.  A CUDA-graph-replayed
fit then has to be re-captured after every event.

Here the Gaussians live in capacity-sized rows whose live count is a device
word (`LiveGaussianParams`).  `gsv_density_control` applies the reference's
split / clone / prune decisions and the Adam-state transplant to those rows
in place, and the voxelizer skips the rows past the live count
(`gsv_prepare_live`), so the densifying iteration is one more CUDA graph
(`fit_live`).  The host only intervenes when the rows or the pair capacity
run out: the iteration is undone from its in-graph snapshot, the buffers
grow, and the graphs are captured again.
"""
from __future__ import annotations

import ctypes
import time
from typing import Callable, Dict, List, Optional

import torch
import torch.nn as nn

from ._lib import GSV_DENSITY_ROW_OVERFLOW, GsvDensityConfig, GsvDensityRows, check, lib
from .sense import (FitConfig, FitResult, GaussianParams, _sync, data_term_reference, hard_data_consistency,
                    magnitude_tv, magnitude_tv_fused, make_optimizer, nmse, psnr, sense_data_term, sense_workspace,
                    ssim3d, transplant)
from .synthetic import GaussianSet, MRICase

_NAMES = ("positions", "log_scales", "rotations", "density_r", "density_i")
_WIDTHS = (3, 3, 4, 1, 1)
MIN_KEEP = 100  # trainer.py:345: prune only if at least 100 rows survive


def _stream_ptr(dev: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


class LiveGaussianParams(GaussianParams):
    """GaussianParams over `capacity` rows, of which the first ``live[0]``
    (a device int32) are Gaussians.  The other rows are parked: zero
    position, density and log-scale, identity rotation."""

    def __init__(self, init: GaussianSet, device, capacity: int):
        nn.Module.__init__(self)
        dev = torch.device(device)
        n = int(init.positions.shape[0])
        if n > capacity:
            raise ValueError(f"{n} Gaussians do not fit {capacity} rows")
        src = [init.positions.to(dev), torch.log(init.scales.to(dev).clamp_min(1e-8)), init.rotations.to(dev),
               init.density_r.to(dev), init.density_i.to(dev)]
        for name, t, w in zip(_NAMES, src, _WIDTHS):
            buf = torch.zeros((capacity, w) if w > 1 else (capacity,), dtype=torch.float32, device=dev)
            buf[:n] = t.float().reshape(buf[:n].shape)
            if name == "rotations":
                buf[n:, 0] = 1.0
            setattr(self, name, nn.Parameter(buf))
        self.live = torch.tensor([n], dtype=torch.int32, device=dev)

    @property
    def n(self) -> int:
        return int(self.live.item())

    @property
    def capacity(self) -> int:
        return int(self.positions.shape[0])

    def replace(self, new: List[torch.Tensor]):
        raise RuntimeError("live rows change in place (gsv_density_control), not by replacement")

    def snapshot(self) -> GaussianSet:
        n = self.n
        return GaussianSet(self.positions.detach()[:n].clone(), torch.exp(self.log_scales.detach()[:n]),
                           self.rotations.detach()[:n].clone(), self.density_r.detach()[:n].clone(),
                           self.density_i.detach()[:n].clone())

    @torch.no_grad()
    def grown(self, capacity: int) -> "LiveGaussianParams":
        """The same rows in `capacity` >= the current capacity rows."""
        if capacity < self.capacity:
            raise ValueError("rows only grow")
        out = LiveGaussianParams.__new__(LiveGaussianParams)
        nn.Module.__init__(out)
        for name, t, w in zip(_NAMES, self.tensors(), _WIDTHS):
            buf = torch.zeros((capacity, w) if w > 1 else (capacity,), dtype=torch.float32, device=t.device)
            buf[:self.capacity] = t.detach()
            if name == "rotations":
                buf[self.capacity:, 0] = 1.0
            setattr(out, name, nn.Parameter(buf))
        out.live = self.live.clone()
        return out


class DeviceDensity:
    """Workspace, split noise and report of `gsv_density_control` for rows of
    `capacity`; calling it enqueues one density-control step on the current
    stream (no host synchronisation, CUDA-graph capturable)."""

    def __init__(self, capacity: int, cfg: FitConfig, device, seed: int = 0,
                 counter: Optional[torch.Tensor] = None):
        dev = torch.device(device)
        self.device = dev
        self.capacity = int(capacity)
        nbytes = int(lib.gsv_density_workspace_bytes(self.capacity))
        if nbytes == 0:
            raise ValueError(f"invalid row capacity {capacity}")
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.noise = torch.empty((self.capacity, 6), dtype=torch.float32, device=dev)
        self.report = torch.zeros(4, dtype=torch.int32, device=dev)
        self.counter = counter if counter is not None else torch.zeros(1, dtype=torch.int64, device=dev)
        self.seed = int(seed) & ((1 << 64) - 1)
        self.long_axis = bool(cfg.long_axis_split)
        self.cfg = GsvDensityConfig(cfg.grad_threshold, cfg.scale_threshold, cfg.opacity_threshold, cfg.max_scale,
                                    cfg.long_axis_offset_factor, int(cfg.long_axis_split), int(cfg.use_cloning),
                                    MIN_KEEP, int(cfg.max_points))

    def rows(self, p: LiveGaussianParams, opt: Optional[torch.optim.Optimizer]) -> GsvDensityRows:
        r = GsvDensityRows()
        for name, t in zip(_NAMES, p.tensors()):
            if not t.is_contiguous() or t.dtype != torch.float32 or t.shape[0] != self.capacity:
                raise ValueError(f"{name}: expected contiguous float32 rows of {self.capacity}")
            setattr(r, name, t.data_ptr())
        states = [opt.state.get(t, {}) if opt is not None else {} for t in p.tensors()]
        if all("exp_avg" in st for st in states):
            for k, (t, st) in enumerate(zip(p.tensors(), states)):
                for key, dst in (("exp_avg", r.exp_avg), ("exp_avg_sq", r.exp_avg_sq)):
                    m = st[key]
                    if m.shape != t.shape or not m.is_contiguous() or m.dtype != torch.float32:
                        raise ValueError(f"Adam {key} of {_NAMES[k]} does not match its rows")
                    dst[k] = m.data_ptr()
        r.capacity = self.capacity
        return r

    def __call__(self, p: LiveGaussianParams, opt: Optional[torch.optim.Optimizer], pos_grad: torch.Tensor,
                 noise: Optional[torch.Tensor] = None) -> torch.Tensor:
        """One step; returns the device report [flags, split, cloned, pruned]."""
        if pos_grad.shape != (self.capacity, 3) or not pos_grad.is_contiguous():
            raise ValueError("pos_grad must be contiguous [capacity, 3]")
        st = _stream_ptr(self.device)
        if noise is None and not self.long_axis:
            check(lib.gsv_normal_fill(ctypes.c_void_p(self.noise.data_ptr()), self.noise.numel(), self.seed,
                                      ctypes.c_void_p(self.counter.data_ptr()), st), "gsv_normal_fill")
            noise = self.noise
        if noise is not None and (noise.shape != (self.capacity, 6) or not noise.is_contiguous()):
            raise ValueError("noise must be contiguous [capacity, 6]")
        rows = self.rows(p, opt)
        check(lib.gsv_density_control(ctypes.byref(rows), ctypes.c_void_p(pos_grad.data_ptr()),
                                      ctypes.c_void_p(noise.data_ptr() if noise is not None else None),
                                      ctypes.byref(self.cfg), ctypes.c_void_p(p.live.data_ptr()),
                                      ctypes.c_void_p(self.report.data_ptr()), ctypes.c_void_p(self.ws.data_ptr()),
                                      self.ws.numel(), st), "gsv_density_control")
        return self.report


def philox_noise(seed: int, device) -> Callable[[int], torch.Tensor]:
    """The split noise of `DeviceDensity` for `n` rows, as a callable for the
    host-side density control (sense.fit's `split_noise`): each call draws
    the next stream, so a host fit sees the same noise as `fit_live`."""
    dev = torch.device(device)
    counter = torch.zeros(1, dtype=torch.int64, device=dev)
    seed = int(seed) & ((1 << 64) - 1)

    def draw(n: int) -> torch.Tensor:
        out = torch.empty((n, 6), dtype=torch.float32, device=dev)
        check(lib.gsv_normal_fill(ctypes.c_void_p(out.data_ptr()), out.numel(), seed,
                                  ctypes.c_void_p(counter.data_ptr()), _stream_ptr(dev)), "gsv_normal_fill")
        return out

    return draw


# ---------------------------------------------------------------------------
# the fit
# ---------------------------------------------------------------------------

class _LiveStep:
    """The training iteration over live rows as two CUDA graphs: the plain
    iteration (voxelize -> coils -> FFT -> mask -> loss -> backward -> clip
    -> Adam -> lr decay) and the same iteration followed by density control
    (with the lr decay skipped when it changed the rows, trainer.py:424).
    Each graph first snapshots rows, Adam state, learning rates, live count
    and noise counter, so an iteration that ran out of pair capacity or rows
    is undone on the host."""

    def __init__(self, p: LiveGaussianParams, opt, vox, S, mask_c, ku, cfg: FitConfig, capacity: int,
                 density: DeviceDensity, lrs: List[torch.Tensor]):
        self.p, self.opt, self.cfg, self.density, self.lrs = p, opt, cfg, density, lrs
        self.svox = vox.static(p.capacity, capacity, live=p.live)
        self.capacity = capacity
        dev = p.positions.device
        self.device = dev
        for t in p.tensors():
            t.grad = torch.zeros_like(t)
        self.pos_grad = torch.zeros_like(p.positions)
        self.loss = torch.zeros((), device=dev)
        self.host = torch.zeros(5, dtype=torch.int32).pin_memory()  # [voxelizer flags, density report x4]
        self.S, self.mask_c, self.ku = S, mask_c, ku
        self.ws = sense_workspace(dev) if cfg.fused_sense else None
        self.ws_tv = sense_workspace(dev) if cfg.fused_sense else None
        self.graphs: Dict[bool, Optional[torch.cuda.CUDAGraph]] = {False: None, True: None}
        self.stream = torch.cuda.Stream(dev)
        self._refresh_snapshot()

    def _refresh_snapshot(self):
        state = []
        for t in self.p.tensors():
            st = self.opt.state.get(t, {})
            state += [st[k] for k in ("exp_avg", "exp_avg_sq", "step") if k in st]
        # Adam creates its state at its first step: an undo before that drops it
        self.had_state = bool(state)
        self.live = self.p.tensors() + state + list(self.lrs) + [self.p.live, self.density.counter]
        self.snap = [torch.empty_like(t) for t in self.live]

    def _body(self, densify: bool):
        torch._foreach_copy_(self.snap, self.live)
        p, cfg = self.p, self.cfg
        for t in p.tensors():
            t.grad.zero_()
        vol = self.svox(p.positions, torch.exp(p.log_scales), p.rotations, torch.complex(p.density_r, p.density_i))
        if cfg.fused_sense:
            loss = sense_data_term(vol, self.S, self.mask_c[0], self.ku, self.ws)
        else:
            loss = data_term_reference(vol, self.S, self.mask_c, self.ku)
        if cfg.tv_weight > 0:
            tv = magnitude_tv_fused(vol, self.ws_tv) if cfg.fused_sense else magnitude_tv(vol)
            loss = loss + cfg.tv_weight * tv
        loss.backward()
        self.pos_grad.copy_(p.positions.grad)
        if cfg.max_grad_norm > 0:
            torch.nn.utils.clip_grad_norm_(p.tensors(), cfg.max_grad_norm)
        self.opt.step()
        with torch.no_grad():
            if densify:
                report = self.density(p, self.opt, self.pos_grad)
                changed = (report[0] & 7) != 0
                torch._foreach_mul_(self.lrs, torch.where(changed, 1.0, cfg.gamma).float())
                self.host[1:].copy_(report, non_blocking=True)
            else:
                torch._foreach_mul_(self.lrs, cfg.gamma)
        self.loss.copy_(loss.detach())
        self.host[:1].copy_(self.svox.plan.flags_dev, non_blocking=True)

    def eager(self, densify: bool):
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.stream):
            self._body(densify)
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    def capture(self, densify: bool, pool=None):
        self._refresh_snapshot()
        g = torch.cuda.CUDAGraph()
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.stream):
            if pool is None:
                g.capture_begin()
            else:
                g.capture_begin(pool=pool)
            try:
                self._body(densify)
            finally:
                g.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(self.stream)
        self.graphs[densify] = g
        return g

    def replay(self, densify: bool):
        self.graphs[densify].replay()

    def check(self, densify: bool) -> Optional[str]:
        """None, "pairs" (pair capacity overflow) or "rows" (row overflow)."""
        torch.cuda.current_stream(self.device).synchronize()
        if int(self.host[0]) & 1:
            return "pairs"
        if densify and int(self.host[1]) & GSV_DENSITY_ROW_OVERFLOW:
            return "rows"
        return None

    def report(self) -> List[int]:
        return [int(v) for v in self.host[1:]]

    @torch.no_grad()
    def undo(self):
        torch._foreach_copy_(self.live, self.snap)
        if not self.had_state:
            for t in self.p.tensors():
                self.opt.state.pop(t, None)


def initial_rows(n: int, max_points: int) -> int:
    """Row capacity for `n` starting Gaussians: room for a doubling, at least
    64k rows, at most `max_points`, a multiple of 1024."""
    want = min(int(max_points), max(2 * n, 65536))
    return max(n, ((want + 1023) // 1024) * 1024 if want < max_points else want)


def fit_live(case: MRICase, init: GaussianSet, cfg: FitConfig, device="cuda:0", stop_nmse: Optional[float] = None,
             log: Optional[Callable] = None, eval_ssim: bool = True, capacity_margin: float = 2.0,
             row_capacity: Optional[int] = None, stats: Optional[Dict] = None) -> FitResult:
    """The plain 3DGSMR fit with every iteration, densifying ones included,
    replayed from one of two CUDA graphs over live rows.  Graphs are
    captured once, and again only after a pair-capacity or row overflow
    (the iteration is undone and re-run with larger buffers).  The pair
    capacity starts at `capacity_margin` x the initial pair count, since
    densification grows it without a host recount.  The split noise comes
    from the library's Philox stream keyed by ``cfg.seed``."""
    from .tile_voxelizer import TileVoxelizer

    dev = torch.device(device)
    shape = tuple(case.ground_truth.shape)
    vox = TileVoxelizer(shape, tile_size=cfg.tile_size, device=str(dev), deterministic=cfg.deterministic)
    S = case.sensitivity_maps.to(dev).to(torch.complex64).contiguous()
    mask = case.mask.to(dev).float().contiguous()
    ku = case.kspace_undersampled.to(dev).to(torch.complex64).contiguous()
    gt = case.ground_truth.to(dev)
    mask_c = mask.unsqueeze(0)
    n0 = int(init.positions.shape[0])
    p = LiveGaussianParams(init, dev, row_capacity or initial_rows(n0, cfg.max_points))
    lrs = [torch.tensor(v, device=dev) for v in (cfg.position_lr, cfg.scale_lr, cfg.rotation_lr, cfg.density_lr,
                                                   cfg.density_lr)]
    opt = make_optimizer(p, cfg, lrs=lrs, capturable=True)
    density = DeviceDensity(p.capacity, cfg, dev, seed=cfg.seed)
    res = FitResult(params=p)
    st = stats if stats is not None else {}
    for k in ("captures", "overflows", "row_growths", "events"):
        st.setdefault(k, 0)
    st.setdefault("capture_seconds", 0.0)

    def pair_capacity() -> int:
        n = p.n
        total = vox.count_pairs(p.positions.detach()[:n], torch.exp(p.log_scales.detach()[:n])) if n else 0
        return int(total * capacity_margin) + 4096

    def grow_rows():
        nonlocal p, opt, density
        cap = min(int(cfg.max_points), 2 * p.capacity)
        if cap <= p.capacity:
            raise RuntimeError("row overflow at max_points rows")
        p2 = p.grown(cap)
        opt2 = make_optimizer(p2, cfg, lrs=lrs, capturable=True)
        transplant(opt, opt2, torch.ones(p.capacity, dtype=torch.bool, device=dev), cap)
        density = DeviceDensity(cap, cfg, dev, seed=cfg.seed, counter=density.counter)
        p, opt = p2, opt2
        res.params = p

    pairs_cap = pair_capacity()
    step: Optional[_LiveStep] = None
    pool = None
    wall = 0.0
    _sync(dev)
    t0 = time.perf_counter()
    for it in range(cfg.iterations):
        densify = cfg.densify_from <= it <= cfg.densify_until and it % cfg.densify_every == 0
        while True:
            if step is None:
                step = _LiveStep(p, opt, vox, S, mask_c, ku, cfg, pairs_cap, density, lrs)
            fresh = step.graphs[densify] is None
            tc = time.perf_counter()
            if fresh:
                step.eager(densify)
            else:
                step.replay(densify)
            bad = step.check(densify)
            if bad is None:
                if fresh:
                    g = step.capture(densify, pool)
                    if pool is None:
                        pool = g.pool()
                    st["captures"] += 1
                    st["capture_seconds"] += time.perf_counter() - tc
                break
            step.undo()
            if bad == "pairs":
                st["overflows"] += 1
                pairs_cap = step.capacity * 2
            else:
                st["row_growths"] += 1
                grow_rows()
            step = None
        if densify and step.report()[0] & 7:
            st["events"] += 1
        last = it == cfg.iterations - 1
        if (it % cfg.eval_every == 0) or last:
            _sync(dev)
            wall += time.perf_counter() - t0
            with torch.no_grad():
                n = p.n
                v = vox(p.positions[:n], torch.exp(p.log_scales[:n]), p.rotations[:n],
                        torch.complex(p.density_r[:n], p.density_i[:n]))
                rec = hard_data_consistency(v, S, mask, ku)
                e = nmse(rec, gt)
            row = {"iteration": it, "loss": float(step.loss), "nmse": e, "n_points": n, "seconds": wall}
            res.history.append(row)
            if log:
                log(row)
            done = stop_nmse is not None and e <= stop_nmse
            if last or done:
                res.final_nmse = e
                res.final_psnr = psnr(rec, gt)
                if eval_ssim:
                    res.final_ssim = ssim3d(rec, gt)
                if done:
                    break
            _sync(dev)
            t0 = time.perf_counter()
    res.seconds = wall
    res.params = p
    return res
