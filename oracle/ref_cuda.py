"""The reference's CUDA voxelizer on the GPU -- TEST AND MEASUREMENT
INFRASTRUCTURE (the GPU cross-checks in tests/ and bench.py's reference-CUDA
baseline leg), never part of the product.

REF is the reference's own extension, compiled from its two source files
into oracle/_ref/ by oracle/build_ref.py (None where it was never built).
Around it this module restates the reference's glue so the extension runs
the way 3DGS/3dgsVC/gaussian/tile_voxelizer.py drives it: the torch
preprocess (:282-290), the torch binning with its host sync (:87-162), the
autograd wrapper (:165-207) and the complex volume of the caller
(trainers/trainer.py:231-235)."""
import torch

from oracle import build_ref, torch_port

REF = build_ref.load()


class RefFn(torch.autograd.Function):
    """_TileVoxelizeCUDA of tile_voxelizer.py:165-207 around REF."""

    @staticmethod
    def forward(ctx, center, cov_inv, dr, di, tr, pid, hs, ts, d, h, w):
        vr, vi = REF.forward(center.contiguous(), cov_inv.contiguous(), dr.contiguous(), di.contiguous(), tr, pid,
                             hs, ts, d, h, w)
        ctx.save_for_backward(center, cov_inv, dr, di, tr, pid, hs)
        ctx.dims = (ts, d, h, w)
        return vr, vi

    @staticmethod
    def backward(ctx, gr, gi):
        center, cov_inv, dr, di, tr, pid, hs = ctx.saved_tensors
        ts, d, h, w = ctx.dims
        gc, gm, gdr, gdi = REF.backward(center.contiguous(), cov_inv.contiguous(), dr.contiguous(), di.contiguous(),
                                        tr, pid, hs, gr.contiguous(), gi.contiguous(), ts, d, h, w)
        return gc, gm, gdr, gdi, None, None, None, None, None, None, None


def reference_step(params, shape, ts):
    """TileVoxelizer.forward of the reference (tile_voxelizer.py:279-309)
    with the CUDA extension: complex64 (D,H,W), differentiable in the five
    parameter tensors."""
    pos, scl, rot, dr, di = params
    center, cov_inv, half = torch_port.preprocess(pos, scl, rot, shape)
    with torch.no_grad():
        tr, pid = torch_port.build_tile_pairs_torch(center.detach(), torch_port.radius_vox(scl.detach(), half),
                                                    shape, ts)
    vr, vi = RefFn.apply(center, cov_inv, dr, di, tr, pid, half, ts, *shape)
    return torch.complex(vr, vi).view(*shape)


class RefVoxelizer:
    """Callable with TileVoxelizer's forward signature."""

    def __init__(self, shape, tile_size=8):
        self.shape, self.ts = tuple(shape), tile_size

    def __call__(self, positions, scales, rotations, density):
        return reference_step((positions, scales, rotations, density.real, density.imag), self.shape, self.ts)
