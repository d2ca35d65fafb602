"""PyTorch-CPU port of the reference's own CPU voxelizer path -- test and
measurement infrastructure (bench.py's CPU-baseline leg and its
``--impl reference`` arm).

It restates, in FP32 torch on the host cores, what the reference runs when
its CUDA extension is unavailable (3DGS/3dgsVC/gaussian/tile_voxelizer.py):
the torch preprocess (:282-290, :77-84), then for every non-empty tile a
dense (voxels x listed Gaussians) evaluation -- distance normalised by the
half shape, Mahalanobis form via einsum, exp(-m/2) masked by m <= 9,
weighted density sum, scatter into the complex volume (:210-244) -- and
autograd for the backward.  The reference module itself cannot be shipped
with this repository, so this port is what the CPU baseline times.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch


def _rotation(q: torch.Tensor) -> torch.Tensor:
    q = q / (q.norm(dim=-1, keepdim=True) + 1e-8)
    w, x, y, z = q.unbind(-1)
    return torch.stack([
        torch.stack([1 - 2 * y * y - 2 * z * z, 2 * x * y - 2 * z * w, 2 * x * z + 2 * y * w], -1),
        torch.stack([2 * x * y + 2 * z * w, 1 - 2 * x * x - 2 * z * z, 2 * y * z - 2 * x * w], -1),
        torch.stack([2 * x * z - 2 * y * w, 2 * y * z + 2 * x * w, 1 - 2 * x * x - 2 * y * y], -1),
    ], -2)


def preprocess(positions, scales, rotations, shape):
    """center_vox, cov_inv, half_shape (tile_voxelizer.py:282-290)."""
    shape_t = torch.tensor(shape, dtype=torch.float32, device=positions.device)
    half = shape_t * 0.5
    center = (positions + 1.0) * 0.5 * shape_t - 0.5
    T = _rotation(rotations) * torch.reciprocal(scales + 1e-8).unsqueeze(1)
    return center, T @ T.transpose(1, 2), half


def radius_vox(scales, half):
    return (scales * half).max(dim=-1)[0] * 3.0


def tile_forward(center, cov_inv, density, half, tile_ranges, pair_ids, shape, tile_size, tiles):
    """Complex64 flat volume from the listed tiles (dense per-tile evaluation)."""
    d, h, w = shape
    n_th, n_tw = math.ceil(h / tile_size), math.ceil(w / tile_size)
    vol = torch.zeros(d * h * w, dtype=torch.complex64)
    for t in tiles:
        s, e = int(tile_ranges[t, 0]), int(tile_ranges[t, 1])
        if s >= e:
            continue
        gids = torch.from_numpy(pair_ids[s:e].astype(np.int64))
        td, rem = divmod(int(t), n_th * n_tw)
        th, tw = divmod(rem, n_tw)
        rd = torch.arange(td * tile_size, min(td * tile_size + tile_size, d), dtype=torch.float32)
        rh = torch.arange(th * tile_size, min(th * tile_size + tile_size, h), dtype=torch.float32)
        rw = torch.arange(tw * tile_size, min(tw * tile_size + tile_size, w), dtype=torch.float32)
        gd, gh, gw = torch.meshgrid(rd, rh, rw, indexing="ij")
        vox = torch.stack([gd, gh, gw], -1).reshape(-1, 3)
        diff = (vox.unsqueeze(1) - center[gids].unsqueeze(0)) / half
        mahal = torch.einsum("vgi,gij,vgj->vg", diff, cov_inv[gids], diff)
        wgt = torch.exp(-0.5 * mahal) * (mahal <= 9.0).float()
        contrib = (wgt.to(torch.complex64) * density[gids].unsqueeze(0)).sum(1)
        flat = (gd.reshape(-1).long() * h + gh.reshape(-1).long()) * w + gw.reshape(-1).long()
        vol = vol.index_add(0, flat, contrib)
    return vol


def time_fwd_bwd(params, shape, tile_size, tile_ranges, pair_ids, grad_vol, tiles):
    """Forward + autograd backward over `tiles`; returns seconds."""
    pos, scl, rot, dr, di = (torch.tensor(np.asarray(x), dtype=torch.float32).requires_grad_(True) for x in params)
    g = torch.tensor(np.asarray(grad_vol).reshape(-1), dtype=torch.complex64)
    t0 = time.perf_counter()
    center, cov_inv, half = preprocess(pos, scl, rot, shape)
    vol = tile_forward(center, cov_inv, torch.complex(dr, di), half, tile_ranges, pair_ids, shape, tile_size, tiles)
    loss = (vol.real * g.real + vol.imag * g.imag).sum()
    loss.backward()
    return time.perf_counter() - t0


def build_tile_pairs_torch(center_vox, radius_vox, shape, tile_size):
    """Torch restatement of the reference's binning (tile_voxelizer.py:87-162),
    runnable on CPU or GPU; includes the reference's host sync on the pair
    total.  Used to time the reference's full step on the GPU."""
    d, h, w = shape
    dev = center_vox.device
    n = center_vox.shape[0]
    ntd, nth, ntw = (math.ceil(s / tile_size) for s in shape)
    r3 = radius_vox.unsqueeze(1).expand(-1, 3)
    lo = (center_vox - r3).floor().int()
    hi = (center_vox + r3).ceil().int()
    size = torch.tensor([d, h, w], device=dev, dtype=torch.int32)
    nt = torch.tensor([ntd, nth, ntw], device=dev, dtype=torch.int32)
    lo = torch.minimum(torch.clamp(lo, min=0), size - 1)
    hi = torch.minimum(torch.clamp(hi, min=0), size - 1)
    tmin = torch.minimum(torch.clamp(lo // tile_size, min=0), nt - 1)
    tmax = torch.minimum(torch.clamp(hi // tile_size, min=0), nt - 1)
    n_per = tmax - tmin + 1
    cnt = n_per[:, 0] * n_per[:, 1] * n_per[:, 2]
    total = int(cnt.sum().item())
    ranges = torch.zeros(ntd * nth * ntw, 2, dtype=torch.int32, device=dev)
    if total == 0:
        return ranges, torch.zeros(0, dtype=torch.int32, device=dev)
    gid = torch.repeat_interleave(torch.arange(n, device=dev, dtype=torch.int32), cnt)
    start = torch.cumsum(cnt, 0) - cnt
    local = torch.arange(total, device=dev, dtype=torch.int64) - torch.repeat_interleave(start, cnt)
    nh = torch.repeat_interleave(n_per[:, 1], cnt)
    nw = torch.repeat_interleave(n_per[:, 2], cnt)
    ld, lr = local // (nh * nw), local % (nh * nw)
    lh, lw = lr // nw, lr % nw
    td = torch.repeat_interleave(tmin[:, 0], cnt) + ld.int()
    th = torch.repeat_interleave(tmin[:, 1], cnt) + lh.int()
    tw = torch.repeat_interleave(tmin[:, 2], cnt) + lw.int()
    tile = (td * nth * ntw + th * ntw + tw).int()
    order = torch.argsort(tile, stable=True)
    tile_s, gid_s = tile[order], gid[order]
    change = torch.ones(total, dtype=torch.bool, device=dev)
    change[1:] = tile_s[1:] != tile_s[:-1]
    pos = torch.nonzero(change, as_tuple=True)[0]
    ends = torch.cat([pos[1:], torch.tensor([total], device=dev)])
    ranges[tile_s[pos].long(), 0] = pos.int()
    ranges[tile_s[pos].long(), 1] = ends.int()
    return ranges, gid_s
