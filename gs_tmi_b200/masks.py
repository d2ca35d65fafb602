"""Variable-density Poisson-disc k-space masks on the GPU
(gsv_poisson_masks), for generating training data in bulk.

The reference (3DGS/3dgsVC/data/mask_generator.py) builds each (ky, kz)
phase-encode mask with a Python loop: the calibration square first, then one
pass of dart throwing over a random permutation of the pixels, where a pixel
is taken unless an already taken pixel lies within its exclusion radius
0.6 / sqrt(pdf), until ny*nz/accel pixels are set (:241-390).  The pdf and
the radius map are restated here in numpy, operation for operation
(gen_pdf, :22-63; sample_poisson_approx, :132-239).

The dart throwing itself runs on the device as an order-respecting parallel
greedy: a pixel is rejected as soon as an earlier taken pixel lies in its
disc and taken once no earlier pixel in its disc is undecided, so the result
equals the sequential pass exactly, and the first ny*nz/accel - |calibration|
taken pixels in visiting order are kept.  One CTA builds one mask; a batch of
masks runs in one launch.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Optional, Sequence, Tuple

import numpy as np
import torch

from ._lib import check, lib

RADIUS_SCALE = 0.6   # mask_generator.py:285 (s = 0.6)
PDF_FLOOR = 1e-4     # mask_generator.py:166


def gen_pdf(shape: Tuple[int, int], accel: float, calib_size: int, p: float = 2.0) -> np.ndarray:
    """mask_generator.py:22-63: polynomial variable-density pdf (1 - r)^p on
    the normalised polar radius, 1 in the calibration square, scaled to
    ny*nz/accel expected samples and clipped to [0, 1]; FP64."""
    ny, nz = shape
    y = np.linspace(-1, 1, ny)
    z = np.linspace(-1, 1, nz)
    yy, zz = np.meshgrid(y, z, indexing="ij")
    r = np.sqrt(yy ** 2 + zz ** 2)
    pdf = np.power(np.maximum(0, 1 - r), p)
    cy, cz = ny // 2, nz // 2
    h = calib_size // 2
    pdf[cy - h:cy + h, cz - h:cz + h] = 1.0
    target = int(ny * nz / accel)
    if pdf.sum() == 0:
        return np.ones(shape) / accel
    pdf = pdf / pdf.sum() * target
    return np.clip(pdf, 0, 1)


def exclusion_radius(shape: Tuple[int, int], accel: float, calib_size: int, p: float = 2.0) -> np.ndarray:
    """The per-pixel exclusion radius of the dart throwing
    (mask_generator.py:166-167, :285-298): 0.6 * (1 / sqrt(max(pdf, 1e-4)))."""
    pdf = gen_pdf(shape, accel, calib_size, p)
    return RADIUS_SCALE * (1.0 / np.sqrt(np.maximum(pdf, PDF_FLOOR)))


def target_points(shape: Tuple[int, int], accel: float) -> int:
    return int((shape[0] * shape[1]) / accel)


def poisson_masks(shape: Tuple[int, int], accel: float, calib_size: int = 24, orders=None,
                  seeds: Optional[Sequence[int]] = None, p: float = 2.0, device="cuda:0",
                  return_rounds: bool = False):
    """A batch of masks, int8 [B, ny, nz] on `device`.  The visiting orders
    are `orders` ([B, ny*nz] permutations) or, per seed,
    np.random.RandomState(seed).permutation(ny*nz) -- the order the
    reference draws after np.random.seed(seed)."""
    ny, nz = shape
    n = ny * nz
    dev = torch.device(device)
    if orders is None:
        if seeds is None:
            raise ValueError("give orders or seeds")
        orders = np.stack([np.random.RandomState(int(s)).permutation(n) for s in seeds])
    orders_t = torch.as_tensor(np.asarray(orders), dtype=torch.int32).reshape(-1, n).to(dev).contiguous()
    count = int(orders_t.shape[0])
    radius = torch.as_tensor(exclusion_radius(shape, accel, calib_size, p), dtype=torch.float64).to(dev)
    radius = radius.reshape(-1).contiguous()
    masks = torch.empty((count, n), dtype=torch.int8, device=dev)
    rounds = torch.empty(count, dtype=torch.int32, device=dev)
    ws = torch.empty(int(lib.gsv_poisson_workspace_bytes(ny, nz, count)), dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        check(lib.gsv_poisson_masks(ctypes.c_void_p(radius.data_ptr()), ctypes.c_void_p(orders_t.data_ptr()),
                                    ny, nz, int(calib_size), target_points(shape, accel), count,
                                    ctypes.c_void_p(masks.data_ptr()), ctypes.c_void_p(rounds.data_ptr()),
                                    ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                    ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
              "gsv_poisson_masks")
    if int(rounds.min()) < 0:  # one synchronisation; the kernel flags an order that is not a permutation
        raise ValueError("a visiting order is not a permutation of the ny*nz pixels")
    masks = masks.reshape(count, ny, nz)
    if return_rounds:
        return masks, rounds
    return masks


def gen_poisson_mask(shape: Tuple[int, int], accel: float, calib_size: int = 24, device="cuda:0") -> np.ndarray:
    """Drop-in for mask_generator.gen_poisson_mask (:392-400): draws the
    visiting order from numpy's global state as the reference does and
    returns the same int8 [ny, nz] numpy mask."""
    order = np.random.permutation(shape[0] * shape[1])
    return poisson_masks(shape, accel, calib_size, orders=order[None], device=device)[0].cpu().numpy()


def expand_phase_mask(mask_2d: torch.Tensor, shape: Tuple[int, int, int], phase_axes: Iterable[int]) -> torch.Tensor:
    """dataset.py:432-436: the (ky, kz) mask repeated along the readout axis."""
    axes = list(phase_axes)
    view = [1] * len(shape)
    view[axes[0]] = mask_2d.shape[0]
    view[axes[1]] = mask_2d.shape[1]
    return mask_2d.reshape(view).expand(*shape).clone()
