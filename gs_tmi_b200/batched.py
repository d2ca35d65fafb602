"""Many volumes, one persistent launch: batched voxelization.

Each volume keeps its own Gaussians, workspace and tile lists (binned with
the regular per-volume entry points); the forward and the backward of all
volumes then run as single persistent launches whose CTAs pull (volume,
tile) work items from an atomic counter (``gsv_forward_batched`` /
``gsv_backward_batched`` in include/gsv.h).

* ``BatchedVoxelizer`` -- autograd-aware, sizes everything per call (one
  host sync per volume for the pair totals, like the single-volume path).
* ``StaticBatch`` -- fixed Gaussian counts and pair capacities: binning,
  forward and backward only enqueue work, so a whole batched iteration can
  be captured in a CUDA graph and replayed.
* ``BatchedRecon`` -- a whole plain-reconstruction iteration over the batch
  (SENSE data term and TV per volume, Adam over all parameters) on top of a
  StaticBatch, also only enqueued work.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import torch

from . import _lib
from ._lib import GsvBatchItem, GsvGrads, GsvParams, check, lib
from .tile_voxelizer import StaticPlan, _f32, _ptr, _shape, _stream, prepare_and_bin


def _item(shape, params, plan, volume, grad_volume=None, grads=None, chunk=32) -> GsvBatchItem:
    pos, scl, rot, dr, di = params
    gp = GsvParams(pos.data_ptr(), scl.data_ptr(), rot.data_ptr(), dr.data_ptr(), di.data_ptr(), plan.n)
    gg = GsvGrads(*(g.data_ptr() for g in grads)) if grads is not None else GsvGrads()
    return GsvBatchItem(shape, gp, plan.ws_gauss.data_ptr(), plan.ws_pairs.data_ptr(), plan.capacity,
                        volume.data_ptr(), grad_volume.data_ptr() if grad_volume is not None else None, gg,
                        int(chunk))


def _setup(items: List[GsvBatchItem], flags: int, device) -> torch.Tensor:
    count = len(items)
    nbytes = lib.gsv_batch_workspace_bytes(count)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=device)
    arr = (GsvBatchItem * count)(*items)
    check(lib.gsv_batch_setup(arr, count, flags, _ptr(ws), nbytes, _stream(device)), "gsv_batch_setup")
    return ws


class _BatchFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, bv, *flat):
        dev = flat[0].device
        groups = [tuple(_f32(t) for t in flat[5 * i:5 * i + 5]) for i in range(len(bv.shapes))]
        plans, vols, items = [], [], []
        with torch.cuda.device(dev):
            for shape, params in zip(bv.gshapes, groups):
                plan = prepare_and_bin(params, shape, bv.flags)
                vol = torch.empty((shape.d, shape.h, shape.w), dtype=torch.complex64, device=dev)
                plans.append(plan)
                vols.append(vol)
                items.append(_item(shape, params, plan, vol))
            ws = _setup(items, bv.flags, dev)
            check(lib.gsv_forward_batched(_ptr(ws), len(items), _stream(dev)), "gsv_forward_batched")
        ctx.bv, ctx.plans = bv, plans
        ctx.save_for_backward(*[t for g in groups for t in g])
        return tuple(vols)

    @staticmethod
    def backward(ctx, *grad_vols):
        bv, plans = ctx.bv, ctx.plans
        saved = ctx.saved_tensors
        dev = saved[0].device
        outs, items, keep = [], [], []
        for i, (shape, plan) in enumerate(zip(bv.gshapes, plans)):
            params = saved[5 * i:5 * i + 5]
            gv = grad_vols[i]
            gv = (torch.zeros((shape.d, shape.h, shape.w), dtype=torch.complex64, device=dev) if gv is None
                  else gv.resolve_conj().to(torch.complex64).contiguous())
            o = [torch.empty_like(t) for t in params]
            outs += o
            keep.append(gv)
            items.append(_item(shape, params, plan, gv, gv, o))
        with torch.cuda.device(dev):
            ws = _setup(items, bv.flags, dev)
            check(lib.gsv_backward_batched(_ptr(ws), len(items), bv.flags, _stream(dev)), "gsv_backward_batched")
        return (None, *outs)


class BatchedVoxelizer:
    """Voxelize several volumes in one persistent forward launch and one
    persistent backward launch.  Tile edge 8 (the reference default)."""

    def __init__(self, shapes: Sequence[Tuple[int, int, int]], device="cuda:0", deterministic: bool = False):
        self.shapes = [tuple(int(x) for x in s) for s in shapes]
        self.gshapes = [_shape(s, 8) for s in self.shapes]
        self.device = torch.device(device)
        self.flags = _lib.GSV_BACKWARD_DETERMINISTIC if deterministic else 0

    def __call__(self, param_sets) -> Tuple[torch.Tensor, ...]:
        if len(param_sets) != len(self.shapes):
            raise ValueError("one parameter set per volume")
        flat = []
        for ps in param_sets:
            pos, scl, rot, den = ps
            if torch.is_complex(den):
                flat += [pos, scl, rot, den.real, den.imag]
            else:
                flat += [pos, scl, rot, den, torch.zeros_like(den)]
        return _BatchFn.apply(self, *flat)


class StaticBatch:
    """Fixed-size batch for CUDA-graph capture: the caller writes parameters
    into ``params[i]`` and upstream gradients into ``grad_volumes[i]``;
    ``bin()``, ``forward()`` and ``backward()`` only enqueue work."""

    def __init__(self, shapes, ns, capacities, device="cuda:0", deterministic: bool = False, chunks=None):
        self.device = torch.device(device)
        self.flags = _lib.GSV_BACKWARD_DETERMINISTIC if deterministic else 0
        self.gshapes = [_shape(s, 8) for s in shapes]
        self.plans, self.params, self.volumes, self.grad_volumes, self.grads = [], [], [], [], []
        items = []
        dev = self.device
        chunks = chunks or [32] * len(self.gshapes)
        for shape, n, cap, chunk in zip(self.gshapes, ns, capacities, chunks):
            plan = StaticPlan(shape, int(n), dev, int(cap), self.flags)
            params = [torch.zeros(n, 3, device=dev), torch.full((n, 3), 1e-2, device=dev),
                      torch.zeros(n, 4, device=dev), torch.zeros(n, device=dev), torch.zeros(n, device=dev)]
            params[2][:, 0] = 1.0
            vol = torch.zeros((shape.d, shape.h, shape.w), dtype=torch.complex64, device=dev)
            gvol = torch.zeros_like(vol)
            grads = [torch.zeros_like(t) for t in params]
            self.plans.append(plan)
            self.params.append(params)
            self.volumes.append(vol)
            self.grad_volumes.append(gvol)
            self.grads.append(grads)
            items.append(_item(shape, params, plan, vol, gvol, grads, chunk))
        self.count = len(items)
        self.ws = _setup(items, self.flags, dev)

    def bin(self):
        st = _stream(self.device)
        for shape, plan, params in zip(self.gshapes, self.plans, self.params):
            gp = GsvParams(*(t.data_ptr() for t in params), plan.n)
            check(lib.gsv_prepare(ctypes.byref(gp), shape, _ptr(plan.ws_gauss), plan.gauss_bytes, None, st),
                  "gsv_prepare")
            check(lib.gsv_bin(shape, plan.n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.pair_bytes,
                              plan.capacity, st), "gsv_bin")

    def forward(self):
        check(lib.gsv_forward_batched(_ptr(self.ws), self.count, _stream(self.device)), "gsv_forward_batched")

    def backward(self):
        check(lib.gsv_backward_batched(_ptr(self.ws), self.count, self.flags, _stream(self.device)),
              "gsv_backward_batched")

    def overflowed(self) -> List[bool]:
        return [bool(int(p.flags_dev.item()) & _lib.GSV_FLAG_CAPACITY_OVERFLOW) for p in self.plans]


class BatchedRecon:
    """One plain-reconstruction iteration over several volumes at once:
    scales = exp(log-scales), per-volume binning, ONE persistent forward
    launch, per volume the fused SENSE data term and magnitude TV (their
    volume gradients written straight into the batch's upstream gradients),
    ONE persistent backward launch, the chain rule to the log-scales, a
    per-volume gradient-norm clip and one fused Adam step over every
    volume's parameters.  ``step()`` only enqueues work, so one CUDA graph
    captures the whole iteration.

    cases: synthetic.MRICase per volume (on any device); inits: GaussianSet
    per volume; capacities: static pair capacity per volume."""

    def __init__(self, cases, inits, capacities, device="cuda:0", deterministic: bool = False, chunks=None,
                 tv_weight: float = 0.1, max_grad_norm: float = 1.0, lrs=(1e-3, 5e-3, 1e-3, 1e-2, 1e-2)):
        from . import sense

        dev = torch.device(device)
        self.device = dev
        shapes = [tuple(c.ground_truth.shape) for c in cases]
        self.sb = StaticBatch(shapes, [g.n for g in inits], capacities, device=str(dev),
                              deterministic=deterministic, chunks=chunks)
        self.tv_weight, self.max_grad_norm = float(tv_weight), float(max_grad_norm)
        self.S = [c.sensitivity_maps.to(dev).to(torch.complex64).contiguous() for c in cases]
        self.mask = [c.mask.to(dev).float().contiguous() for c in cases]
        self.ku = [c.kspace_undersampled.to(dev).to(torch.complex64).contiguous() for c in cases]
        self.ws = sense.sense_workspace(dev)
        self.tv_grad = [torch.empty_like(v) for v in self.sb.volumes]
        self.data_loss = [torch.zeros((), device=dev) for _ in cases]
        self.tv_loss = [torch.zeros((), device=dev) for _ in cases]
        groups = [[] for _ in range(5)]
        self.leaves = []
        for i, gs in enumerate(inits):
            pos, scl, rot, dr, di = self.sb.params[i]
            pos.copy_(gs.positions.to(dev))
            rot.copy_(gs.rotations.to(dev))
            dr.copy_(gs.density_r.to(dev))
            di.copy_(gs.density_i.to(dev))
            log_s = torch.log(gs.scales.to(dev).clamp_min(1e-12))
            leaves = [torch.nn.Parameter(pos), torch.nn.Parameter(log_s), torch.nn.Parameter(rot),
                      torch.nn.Parameter(dr), torch.nn.Parameter(di)]
            gpos, gscl, grot, gdr, gdi = self.sb.grads[i]
            # the batched backward writes these buffers in place: they are the gradients
            leaves[0].grad, leaves[2].grad, leaves[3].grad, leaves[4].grad = gpos, grot, gdr, gdi
            leaves[1].grad = torch.zeros_like(log_s)
            for k, t in enumerate(leaves):
                groups[k].append(t)
            self.leaves.append(leaves)
        self.lrs = [torch.tensor(float(v), device=dev) for v in lrs]
        self.opt = torch.optim.Adam([{"params": g, "lr": lr} for g, lr in zip(groups, self.lrs)], fused=True,
                                    capturable=True)

    def step(self):
        sb = self.sb
        st = torch.cuda.current_stream(self.device).cuda_stream
        with torch.no_grad():
            for i, leaves in enumerate(self.leaves):
                torch.exp(leaves[1], out=sb.params[i][1])
            sb.bin()
            sb.forward()
            for i, vol in enumerate(sb.volumes):
                d, h, w = vol.shape
                nc = self.S[i].shape[0]
                X = torch.empty_like(self.S[i])
                check(lib.gsv_sense_expand(vol.data_ptr(), self.S[i].data_ptr(), nc, d, h, w, X.data_ptr(), st),
                      "gsv_sense_expand")
                K = torch.fft.fftn(X, dim=(-3, -2, -1), norm="ortho")
                check(lib.gsv_sense_residual(K.data_ptr(), self.mask[i].data_ptr(), self.ku[i].data_ptr(), nc, d,
                                             h, w, self.data_loss[i].data_ptr(), self.ws.data_ptr(), self.ws.numel(),
                                             st), "gsv_sense_residual")
                G = torch.fft.ifftn(K, dim=(-3, -2, -1), norm="ortho")
                gv = sb.grad_volumes[i]
                check(lib.gsv_sense_adjoint(G.data_ptr(), self.S[i].data_ptr(), nc, d, h, w, gv.data_ptr(), st),
                      "gsv_sense_adjoint")
                if self.tv_weight > 0:
                    check(lib.gsv_tv_magnitude(vol.data_ptr(), d, h, w, self.tv_loss[i].data_ptr(),
                                               self.tv_grad[i].data_ptr(), self.ws.data_ptr(), self.ws.numel(), st),
                          "gsv_tv_magnitude")
                    gv.add_(self.tv_grad[i], alpha=self.tv_weight)
            sb.backward()
            for i, leaves in enumerate(self.leaves):
                torch.mul(sb.grads[i][1], sb.params[i][1], out=leaves[1].grad)  # d/d log s = d/ds * s
                if self.max_grad_norm > 0:
                    torch.nn.utils.clip_grad_norm_(leaves, self.max_grad_norm, foreach=True)
        self.opt.step()

    def losses(self) -> List[float]:
        """Per-volume data + tv_weight * TV of the last step (synchronises)."""
        return [float(a) + self.tv_weight * float(b) for a, b in zip(self.data_loss, self.tv_loss)]
