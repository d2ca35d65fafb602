"""Drop-in ``TileVoxelizer`` for 3DGSMR, backed by the sm_100a C ABI.

Mirrors the reference plugin surface of 3DGS/3dgsVC/gaussian/tile_voxelizer.py:

* ``TileVoxelizer(volume_shape, tile_size=8, max_radius=20, use_cuda=True,
  strict_cuda=False, device="cuda:0")`` and ``forward(positions, scales,
  rotations, density, chunk_size=4096)``  (reference :247-322).  Returns a
  complex64 (D,H,W) volume, which the reference callers accept as-is
  (trainers/trainer.py:231-235, test.py:162-163).
* ``build_tile_pairs(center_vox, radius_vox, volume_shape, tile_size)``
  (reference :87-162), on the device, bit-exact.
* ``_TileVoxelizeCUDA`` with the reference's 11-argument autograd signature
  (reference :165-207), for A/B runs against the reference kernels.

Differences by design: there is no CPU fallback (``use_cuda=False`` raises,
as does a missing library), the preprocess, binning, forward, backward and
the autograd chain rule to (positions, scales, rotations, density) all run
in the library's kernels, and the pair total is the only host sync (the
same one the reference makes at :118).
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Tuple

import torch
import torch.nn as nn

from . import _lib
from ._lib import GsvGrads, GsvParams, GsvShape, check, lib

INT32_MAX = 2**31 - 1


def _ptr(t: Optional[torch.Tensor]):
    if t is None or t.numel() == 0:
        return None
    return ctypes.c_void_p(t.data_ptr())


def _stream(device: torch.device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _shape(volume_shape, tile_size) -> GsvShape:
    d, h, w = (int(x) for x in volume_shape)
    ts = int(tile_size)
    if min(d, h, w, ts) <= 0:
        raise ValueError(f"invalid volume shape {volume_shape} / tile size {tile_size}")
    return GsvShape(d, h, w, ts)


def _f32(t: torch.Tensor) -> torch.Tensor:
    return t.detach().float().contiguous()


def _require_cuda(*ts: torch.Tensor) -> torch.device:
    dev = ts[0].device
    for t in ts:
        if t.device.type != "cuda" or t.device != dev:
            raise ValueError("all voxelizer inputs must be CUDA tensors on one device "
                             f"(got {[str(x.device) for x in ts]})")
    return dev


class BinPlan:
    """Workspace of one voxelization (records, tile lists) shared by its
    forward and backward; allocated from torch's caching allocator."""

    def __init__(self, shape: GsvShape, n: int, device: torch.device, flags: int = 0,
                 capacity: Optional[int] = None):
        self.shape, self.n, self.device, self.flags = shape, n, device, flags
        self.gauss_bytes = lib.gsv_gauss_workspace_bytes(n, shape)
        if self.gauss_bytes == 0:
            raise ValueError(f"unsupported problem size n={n} shape=({shape.d},{shape.h},{shape.w})")
        self.ws_gauss = torch.empty(self.gauss_bytes, dtype=torch.uint8, device=device)
        self.capacity = capacity
        self.ws_pairs = None
        self.pair_bytes = 0
        self.total = None

    def alloc_pairs(self, capacity: int):
        self.capacity = int(capacity)
        self.pair_bytes = lib.gsv_pair_workspace_bytes(self.capacity, self.shape, self.flags)
        self.ws_pairs = torch.empty(max(self.pair_bytes, 1), dtype=torch.uint8, device=self.device)

    def read_status(self, stream) -> Tuple[int, int]:
        total, flags = ctypes.c_int64(0), ctypes.c_int32(0)
        check(lib.gsv_read_status(self.shape, self.n, _ptr(self.ws_gauss), ctypes.byref(total),
                                  ctypes.byref(flags), stream), "gsv_read_status")
        return int(total.value), int(flags.value)

    def views(self):
        tr, pid = ctypes.c_void_p(), ctypes.c_void_p()
        check(lib.gsv_bin_views(self.shape, self.n, _ptr(self.ws_gauss), _ptr(self.ws_pairs),
                                self.capacity, ctypes.byref(tr), ctypes.byref(pid)), "gsv_bin_views")
        return tr.value, pid.value


def _raise_flags(flags: int, total: int):
    if flags & _lib.GSV_FLAG_SCAN_STALLED:
        raise RuntimeError("the preprocess's pair-count scan timed out waiting for a block (results invalid)")
    if flags & _lib.GSV_FLAG_EMPTY_BOX:
        raise ValueError("a Gaussian has an empty tile box (negative scale radius)")
    if flags & _lib.GSV_FLAG_TOO_MANY_PAIRS or total > INT32_MAX:
        raise RuntimeError(f"{total} (tile, Gaussian) pairs exceed the int32 tile ranges")


def prepare_and_bin(params: Tuple[torch.Tensor, ...], shape: GsvShape, flags: int = 0) -> BinPlan:
    """Preprocess + bin on the current stream; reads the pair total back
    (one host sync, as the reference does at tile_voxelizer.py:118)."""
    pos, scl, rot, dr, di = params
    dev = pos.device
    n = int(pos.shape[0])
    st = _stream(dev)
    plan = BinPlan(shape, n, dev, flags)
    gp = GsvParams(pos.data_ptr(), scl.data_ptr(), rot.data_ptr(), dr.data_ptr(), di.data_ptr(), n)
    check(lib.gsv_prepare(ctypes.byref(gp), shape, _ptr(plan.ws_gauss), plan.gauss_bytes, None, st),
          "gsv_prepare")
    total, fl = plan.read_status(st)
    _raise_flags(fl, total)
    plan.total = total
    plan.alloc_pairs(total)
    check(lib.gsv_bin(shape, n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.pair_bytes, plan.capacity, st),
          "gsv_bin")
    return plan


def work_census(plan: BinPlan, cull: bool = True) -> dict:
    """What the tile-8 render kernels do on a binned problem
    (gsv_count_work): included candidates, candidates evaluated after the
    extent cull, lanes issued by the exp / FMA blocks and kept slots without
    an included voxel.  Synchronises the current stream."""
    out = torch.zeros(4, dtype=torch.int64, device=plan.device)
    tune = _lib.GsvTuning(2, 32, 0 if cull else _lib.GSV_TUNE_NO_CULL)
    check(lib.gsv_count_work(plan.shape, plan.n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.capacity or 0,
                             ctypes.byref(tune), _ptr(out), _stream(plan.device)), "gsv_count_work")
    inc, ev, lanes, empty = (int(x) for x in out.cpu())
    return {"included": inc, "evaluated": ev, "exp_block_lanes": lanes, "empty_kept_slots": empty}


class _VoxelizeFn(torch.autograd.Function):
    """Fused voxelizer: raw Gaussian parameters -> complex64 volume.

    Forward = TileVoxelizer.forward's preprocess + binning + tile forward
    (reference tile_voxelizer.py:282-309); backward = the tile backward plus
    the autograd tail through :284-290 and :77-84, all in the library."""

    @staticmethod
    def forward(ctx, positions, scales, rotations, density_r, density_i, shape, deterministic, tuner=None):
        params = tuple(_f32(t) for t in (positions, scales, rotations, density_r, density_i))
        dev = _require_cuda(*params)
        flags = _lib.GSV_BACKWARD_DETERMINISTIC if deterministic else 0
        with torch.cuda.device(dev):
            plan = prepare_and_bin(params, shape, flags)
            plan.tuning = tuner.pick(plan, params) if tuner is not None else None
            vol = torch.empty((shape.d, shape.h, shape.w), dtype=torch.complex64, device=dev)
            check(lib.gsv_forward_ex(shape, plan.n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.capacity,
                                     _ptr(vol), _tuning_ref(plan), _stream(dev)), "gsv_forward")
        ctx.plan = plan
        ctx.save_for_backward(*params)
        return vol

    @staticmethod
    def backward(ctx, grad_vol):
        params = ctx.saved_tensors
        plan: BinPlan = ctx.plan
        dev = plan.device
        g = grad_vol.resolve_conj().to(torch.complex64).contiguous()
        outs = [torch.empty_like(t) for t in params]
        with torch.cuda.device(dev):
            backward_into(plan, params, g, outs)
        return (*outs, None, None, None)


def _tuning_ref(plan):
    t = getattr(plan, "tuning", None)
    return ctypes.byref(t) if t is not None else None


def backward_into(plan: BinPlan, params, grad_vol: torch.Tensor, outs) -> None:
    pos, scl, rot, dr, di = params
    gp = GsvParams(pos.data_ptr(), scl.data_ptr(), rot.data_ptr(), dr.data_ptr(), di.data_ptr(), plan.n)
    gg = GsvGrads(*(o.data_ptr() for o in outs))
    check(lib.gsv_backward_ex(ctypes.byref(gp), plan.shape, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs),
                              plan.capacity, _ptr(grad_vol), ctypes.byref(gg), plan.flags, _tuning_ref(plan),
                              _stream(plan.device)), "gsv_backward")


class StaticPlan(BinPlan):
    """Workspace preallocated for `n` Gaussians and a fixed pair capacity.
    The voxelizer then makes no host synchronisation and no allocation of
    its own, so a whole iteration can be captured in a CUDA graph.  Pairs
    beyond the capacity are dropped and GSV_FLAG_CAPACITY_OVERFLOW is latched
    in ``flags_dev`` (copy it out and check it after each replay)."""

    def __init__(self, shape: GsvShape, n: int, device: torch.device, capacity: int, flags: int = 0,
                 live: Optional[torch.Tensor] = None):
        super().__init__(shape, n, device, flags)
        self.alloc_pairs(capacity)
        # live: device int32 [1]; only the first live[0] of the n rows are
        # Gaussians (rows managed by gsv_density_control)
        if live is not None and (live.dtype != torch.int32 or not live.is_cuda or live.numel() != 1):
            raise ValueError("live must be a one-element int32 tensor on the plan's device")
        self.live = live
        fl, tot = ctypes.c_void_p(), ctypes.c_void_p()
        check(lib.gsv_status_views(shape, n, _ptr(self.ws_gauss), ctypes.byref(fl), ctypes.byref(tot)),
              "gsv_status_views")
        base = self.ws_gauss.data_ptr()
        self.flags_dev = self.ws_gauss[fl.value - base:fl.value - base + 4].view(torch.int32)
        self.total_dev = self.ws_gauss[tot.value - base:tot.value - base + 8].view(torch.int64)


class _VoxelizeStaticFn(torch.autograd.Function):
    """Same math as _VoxelizeFn on a StaticPlan: no host sync, no workspace
    allocation (CUDA-graph capturable)."""

    @staticmethod
    def forward(ctx, positions, scales, rotations, density_r, density_i, plan):
        params = tuple(_f32(t) for t in (positions, scales, rotations, density_r, density_i))
        dev = plan.device
        if int(params[0].shape[0]) != plan.n:
            raise ValueError(f"static plan is sized for {plan.n} Gaussians, got {int(params[0].shape[0])}")
        st = _stream(dev)
        gp = GsvParams(*(t.data_ptr() for t in params), plan.n)
        if plan.live is None:
            check(lib.gsv_prepare(ctypes.byref(gp), plan.shape, _ptr(plan.ws_gauss), plan.gauss_bytes, None, st),
                  "gsv_prepare")
        else:
            check(lib.gsv_prepare_live(ctypes.byref(gp), _ptr(plan.live), plan.shape, _ptr(plan.ws_gauss),
                                       plan.gauss_bytes, None, st), "gsv_prepare_live")
        check(lib.gsv_bin(plan.shape, plan.n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.pair_bytes,
                          plan.capacity, st), "gsv_bin")
        vol = torch.empty((plan.shape.d, plan.shape.h, plan.shape.w), dtype=torch.complex64, device=dev)
        check(lib.gsv_forward(plan.shape, plan.n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.capacity,
                              _ptr(vol), st), "gsv_forward")
        ctx.plan = plan
        ctx.save_for_backward(*params)
        return vol

    @staticmethod
    def backward(ctx, grad_vol):
        params = ctx.saved_tensors
        g = grad_vol.resolve_conj().to(torch.complex64).contiguous()
        outs = [torch.empty_like(t) for t in params]
        backward_into(ctx.plan, params, g, outs)
        return (*outs, None)


def voxelize(positions: torch.Tensor, scales: torch.Tensor, rotations: torch.Tensor,
             density_r: torch.Tensor, density_i: torch.Tensor, volume_shape, tile_size: int = 8,
             deterministic: bool = False, tuner=None) -> torch.Tensor:
    """Functional form: complex64 (D,H,W) volume, differentiable in all five
    parameter tensors.  `tuner`: an autotune.Autotuner picking the execution
    shape (results do not depend on it)."""
    return _VoxelizeFn.apply(positions, scales, rotations, density_r, density_i,
                             _shape(volume_shape, tile_size), bool(deterministic), tuner)


# ---------------------------------------------------------------------------
# Reference-compatible pieces
# ---------------------------------------------------------------------------

def build_tile_pairs(center_vox: torch.Tensor, radius_vox: torch.Tensor, volume_shape, tile_size: int):
    """Device binning with the reference's signature and outputs
    (tile_voxelizer.py:87-162): ``tile_ranges`` int32 [T,2] (empty tiles
    (0,0)) and ``pair_ids`` int32 [P], ascending Gaussian id per tile."""
    center = _f32(center_vox)
    radius = _f32(radius_vox)
    dev = _require_cuda(center, radius)
    shape = _shape(volume_shape, tile_size)
    n = int(center.shape[0])
    ntiles = int(lib.gsv_num_tiles(shape))
    with torch.cuda.device(dev):
        st = _stream(dev)
        plan = BinPlan(shape, n, dev)
        check(lib.gsv_build_tile_pairs_count(_ptr(center), _ptr(radius), n, shape, _ptr(plan.ws_gauss),
                                             plan.gauss_bytes, None, st), "gsv_build_tile_pairs_count")
        total, fl = plan.read_status(st)
        _raise_flags(fl, total)
        tile_ranges = torch.zeros((ntiles, 2), dtype=torch.int32, device=dev)
        pair_ids = torch.empty((total,), dtype=torch.int32, device=dev)
        if total == 0:
            return tile_ranges, pair_ids
        plan.alloc_pairs(total)
        check(lib.gsv_build_tile_pairs_fill(shape, n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.pair_bytes,
                                            total, _ptr(tile_ranges), _ptr(pair_ids), st),
              "gsv_build_tile_pairs_fill")
    return tile_ranges, pair_ids


class _TileVoxelizeCUDA(torch.autograd.Function):
    """The reference's autograd wrapper signature (tile_voxelizer.py:165-207):
    (center_vox, cov_inv, density_r, density_i, tile_ranges, pair_ids,
    half_shape, tile_size, d, h, w) -> (vol_r [V], vol_i [V])."""

    @staticmethod
    def forward(ctx, center_vox, cov_inv, density_r, density_i, tile_ranges, pair_ids, half_shape, tile_size,
                d_size, h_size, w_size):
        c, m = _f32(center_vox), _f32(cov_inv)
        dr, di, hs = _f32(density_r), _f32(density_i), _f32(half_shape)
        tr = tile_ranges.detach().int().contiguous()
        pid = pair_ids.detach().int().contiguous()
        dev = _require_cuda(c, m, dr, di, tr, hs)
        n = int(c.shape[0])
        v = d_size * h_size * w_size
        vol_r = torch.empty(v, dtype=torch.float32, device=dev)
        vol_i = torch.empty(v, dtype=torch.float32, device=dev)
        with torch.cuda.device(dev):
            check(lib.gsv_tile_forward(_ptr(c), _ptr(m), _ptr(dr), _ptr(di), _ptr(tr), _ptr(pid), _ptr(hs), n,
                                       int(tr.shape[0]), int(tile_size), int(d_size), int(h_size), int(w_size),
                                       _ptr(vol_r), _ptr(vol_i), _stream(dev)), "gsv_tile_forward")
        ctx.save_for_backward(c, m, dr, di, tr, pid, hs)
        ctx.dims = (int(tile_size), int(d_size), int(h_size), int(w_size))
        return vol_r, vol_i

    @staticmethod
    def backward(ctx, grad_vol_r, grad_vol_i):
        c, m, dr, di, tr, pid, hs = ctx.saved_tensors
        ts, d, h, w = ctx.dims
        v = d * h * w
        gr = grad_vol_r.float().contiguous() if grad_vol_r is not None else torch.zeros(v, device=c.device)
        gi = grad_vol_i.float().contiguous() if grad_vol_i is not None else torch.zeros(v, device=c.device)
        n = int(c.shape[0])
        gc = torch.empty_like(c)
        gm = torch.empty((n, 9), dtype=torch.float32, device=c.device)
        gdr, gdi = torch.empty_like(dr), torch.empty_like(di)
        with torch.cuda.device(c.device):
            check(lib.gsv_tile_backward(_ptr(c), _ptr(m), _ptr(dr), _ptr(di), _ptr(tr), _ptr(pid), _ptr(hs),
                                        _ptr(gr), _ptr(gi), n, int(tr.shape[0]), ts, d, h, w, _ptr(gc), _ptr(gm),
                                        _ptr(gdr), _ptr(gdi), _stream(c.device)), "gsv_tile_backward")
        return gc, gm.reshape(-1, 3, 3), gdr, gdi, None, None, None, None, None, None, None


class TileVoxelizer(nn.Module):
    """Drop-in replacement of the reference ``TileVoxelizer`` (tile_voxelizer.py:247-322).

    Same constructor and forward signature.  ``backend`` is always
    ``"tile_cuda"``; ``use_cuda=False`` or a machine without CUDA raises
    instead of falling back to a CPU path.  ``max_radius`` is stored and
    unused, as in the reference.  ``deterministic=True`` selects the
    fixed-order backward (bitwise reproducible gradients); ``autotune=True``
    lets the project autotuner pick the execution tile shape and Gaussian
    batch per (volume, Gaussian-count bucket) -- results do not change."""

    def __init__(self, volume_shape: Tuple[int, int, int], tile_size: int = 8, max_radius: int = 20,
                 use_cuda: bool = True, strict_cuda: bool = False, device: str = "cuda:0",
                 deterministic: bool = False, autotune: bool = False):
        super().__init__()
        self.volume_shape = tuple(int(x) for x in volume_shape)
        self.tile_size = int(tile_size)
        self.max_radius = max_radius
        self.device = device
        self.strict_cuda = strict_cuda
        self.deterministic = bool(deterministic)
        if not use_cuda:
            raise RuntimeError("gs_tmi_b200.TileVoxelizer has no CPU backend (use_cuda=False requested)")
        if not torch.cuda.is_available():
            raise RuntimeError("gs_tmi_b200.TileVoxelizer needs a CUDA device (sm_100a)")
        self.use_cuda = True
        self.backend = "tile_cuda"
        self._shape = _shape(self.volume_shape, self.tile_size)
        self.tuner = None
        if autotune:
            from .autotune import default_tuner

            self.tuner = default_tuner()

    def forward(self, positions: torch.Tensor, scales: torch.Tensor, rotations: torch.Tensor,
                density: torch.Tensor, chunk_size: int = 4096) -> torch.Tensor:
        del chunk_size
        if torch.is_complex(density):
            dr, di = density.real, density.imag
        else:
            dr, di = density, torch.zeros_like(density)
        return _VoxelizeFn.apply(positions, scales, rotations, dr, di, self._shape, self.deterministic, self.tuner)

    def static(self, n: int, capacity: int, live: Optional[torch.Tensor] = None) -> "StaticVoxelizer":
        """A sync-free, allocation-free variant for `n` Gaussians and at most
        `capacity` (tile, Gaussian) pairs, for CUDA-graph capture.  With
        `live` (device int32 [1]) only the first live[0] rows are Gaussians."""
        flags = _lib.GSV_BACKWARD_DETERMINISTIC if self.deterministic else 0
        dev = torch.device(self.device) if not isinstance(self.device, torch.device) else self.device
        return StaticVoxelizer(StaticPlan(self._shape, int(n), dev, int(capacity), flags, live=live))

    def count_pairs(self, positions: torch.Tensor, scales: torch.Tensor) -> int:
        """Pair total of the current parameters (one host sync)."""
        params = (_f32(positions), _f32(scales), _f32(positions).new_zeros(positions.shape[0], 4),
                  _f32(positions).new_zeros(positions.shape[0]), _f32(positions).new_zeros(positions.shape[0]))
        params[2][:, 0] = 1.0
        plan = BinPlan(self._shape, int(positions.shape[0]), positions.device)
        gp = GsvParams(*(t.data_ptr() for t in params), plan.n)
        st = _stream(positions.device)
        check(lib.gsv_prepare(ctypes.byref(gp), self._shape, _ptr(plan.ws_gauss), plan.gauss_bytes, None, st),
              "gsv_prepare")
        total, fl = plan.read_status(st)
        _raise_flags(fl, total)
        return total

    def extra_repr(self) -> str:
        return (f"volume_shape={self.volume_shape}, tile_size={self.tile_size}, "
                f"backend={self.backend}, deterministic={self.deterministic}")


class StaticVoxelizer:
    """Callable with TileVoxelizer's forward signature over a StaticPlan."""

    def __init__(self, plan: StaticPlan):
        self.plan = plan

    def __call__(self, positions, scales, rotations, density, chunk_size: int = 4096):
        if torch.is_complex(density):
            dr, di = density.real, density.imag
        else:
            dr, di = density, torch.zeros_like(density)
        return _VoxelizeStaticFn.apply(positions, scales, rotations, dr, di, self.plan)


def num_tiles(volume_shape, tile_size: int) -> int:
    d, h, w = volume_shape
    return math.ceil(d / tile_size) * math.ceil(h / tile_size) * math.ceil(w / tile_size)
