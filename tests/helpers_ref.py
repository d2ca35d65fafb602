"""The reference voxelizer on the GPU for A/B tests: its compiled CUDA
extension (oracle/_ref/, built by oracle/build_ref.py from its sources) with
its autograd glue (tile_voxelizer.py:165-207) and a torch restatement of its
preprocess and binning (tile_voxelizer.py:279-309)."""
import torch

from oracle import build_ref, torch_port

REF = build_ref.load()


class RefFn(torch.autograd.Function):
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
