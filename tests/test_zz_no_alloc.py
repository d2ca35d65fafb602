"""gsv_build_tile_pairs_noalloc -- binning for callers that cannot allocate.

Some hosts cannot allocate device memory: their GPU memory is owned by
another allocator (a framework that reserves the device up front, a process
under a hard memory cap) or they run on a path with a fixed memory plan.
For them the library offers one binning entry point whose scratch lives in
a static device array; the caller supplies only the inputs (center_vox,
radius_vox) and the outputs (tile_ranges, pair_ids).

This file checks, through the C ABI, that it returns exactly what the
regular entry points (gsv_build_tile_pairs_count + _fill, which take a
caller workspace) return -- binning is compared bit for bit, as in every
other binning test -- on several calls in a row with different problems (the
static array keeps the previous call's contents, so a missing reset would
show), and that sizes beyond its stated limits are refused.  It is kept
last in collection order and needs nothing from the other test files.
"""
import ctypes

import numpy as np
import pytest
import torch

import gs_tmi_b200
from gs_tmi_b200 import synthetic
from gs_tmi_b200._lib import GSV_ERR_CAPACITY, GSV_ERR_EMPTY_BOX, GSV_ERR_INVALID_ARGUMENT, GSV_OK, GsvShape, lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_GAUSSIANS = 1 << 18
MAX_PAIRS = 1 << 21


def _noalloc(center, radius, shape, ts, capacity):
    dev = center.device
    ntiles = int(lib.gsv_num_tiles(GsvShape(*shape, ts)))
    tr = torch.full((ntiles, 2), -7, dtype=torch.int32, device=dev)  # stale garbage must be cleared
    pid = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device=dev)
    total = ctypes.c_int64(-1)
    rc = lib.gsv_build_tile_pairs_noalloc(
        ctypes.c_void_p(center.data_ptr()) if center.numel() else None,
        ctypes.c_void_p(radius.data_ptr()) if radius.numel() else None,
        int(center.shape[0]), GsvShape(*shape, ts), ctypes.c_void_p(tr.data_ptr()),
        ctypes.c_void_p(pid.data_ptr()), int(capacity), ctypes.byref(total),
        ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    torch.cuda.synchronize(dev)
    return rc, total.value, tr.cpu().numpy(), pid.cpu().numpy()


def _case(kind):
    if kind == "cube64":
        shape, ts = (64, 64, 64), 8
        gs = synthetic.random_gaussians(20000, shape, seed=0)
    elif kind == "ragged_ts4":
        shape, ts = (19, 13, 22), 4
        gs = synthetic.concat(synthetic.random_gaussians(300, shape, seed=81),
                              synthetic.edge_case_gaussians(shape, seed=82))
    else:  # "ragged_ts8"
        shape, ts = (37, 29, 45), 8
        gs = synthetic.random_gaussians(2500, shape, seed=83, log_scale_mean_vox=np.log(3.0))
    c, r, _ = O.preprocess_f32(gs.positions.numpy(), gs.scales.numpy(), gs.rotations.numpy(), shape)
    return shape, ts, c, r


def test_matches_regular_binning_on_calls_in_a_row(cuda_device):
    for kind in ("cube64", "ragged_ts4", "ragged_ts8", "cube64"):
        shape, ts, c, r = _case(kind)
        center = torch.tensor(c, device=cuda_device)
        radius = torch.tensor(r, device=cuda_device)
        ref_tr, ref_pid = gs_tmi_b200.build_tile_pairs(center, radius, shape, ts)  # workspace path
        ref_tr, ref_pid = ref_tr.cpu().numpy(), ref_pid.cpu().numpy()
        rc, total, tr, pid = _noalloc(center, radius, shape, ts, capacity=ref_pid.size + 17)
        assert rc == GSV_OK, kind
        assert total == ref_pid.size, kind
        assert np.array_equal(tr, ref_tr), kind
        assert np.array_equal(pid[:total], ref_pid), kind


def test_no_gaussians(cuda_device):
    empty = torch.zeros(0, 3, device=cuda_device)
    rc, total, tr, _ = _noalloc(empty, torch.zeros(0, device=cuda_device), (16, 16, 16), 8, capacity=0)
    assert rc == GSV_OK and total == 0 and not tr.any()


def test_limits_are_refused(cuda_device):
    # too many Gaussians: refused before any device work
    n = MAX_GAUSSIANS + 1
    big = torch.zeros(n, 3, device=cuda_device)
    rc, _, _, _ = _noalloc(big, torch.ones(n, device=cuda_device), (8, 8, 8), 8, capacity=n)
    assert rc == GSV_ERR_INVALID_ARGUMENT
    # pair total above the static maximum: two Gaussians covering all
    # 128^3 = 2,097,152 tiles of a 512^3 volume at tile edge 4
    shape = (512, 512, 512)
    center = torch.full((2, 3), 255.5, device=cuda_device)
    radius = torch.full((2,), 1000.0, device=cuda_device)
    rc, total, _, _ = _noalloc(center, radius, shape, 4, capacity=4 * MAX_PAIRS)
    assert rc == GSV_ERR_CAPACITY and total == 2 * 128 ** 3 > MAX_PAIRS
    # pair total above the caller's capacity: refused, total reported
    shape, ts, c, r = _case("ragged_ts4")
    rc, total, _, _ = _noalloc(torch.tensor(c, device=cuda_device), torch.tensor(r, device=cuda_device),
                               shape, ts, capacity=10)
    assert rc == GSV_ERR_CAPACITY and total > 10


def test_negative_radius_is_refused_and_the_next_call_is_clean(cuda_device):
    """A negative radius gives an empty tile box, which the reference's
    binning cannot handle either: the call returns GSV_ERR_EMPTY_BOX.  The
    flag lives in the shared array, so the following valid call must still
    match the regular binning."""
    shape, ts, c, r = _case("ragged_ts8")
    r_bad = r.copy()
    r_bad[5] = -50.0
    rc, _, _, _ = _noalloc(torch.tensor(c, device=cuda_device), torch.tensor(r_bad, device=cuda_device), shape, ts,
                           capacity=1 << 20)
    assert rc == GSV_ERR_EMPTY_BOX
    center, radius = torch.tensor(c, device=cuda_device), torch.tensor(r, device=cuda_device)
    ref_tr, ref_pid = gs_tmi_b200.build_tile_pairs(center, radius, shape, ts)
    rc, total, tr, pid = _noalloc(center, radius, shape, ts, capacity=ref_pid.numel())
    assert rc == GSV_OK and total == ref_pid.numel()
    assert np.array_equal(tr, ref_tr.cpu().numpy()) and np.array_equal(pid[:total], ref_pid.cpu().numpy())


def test_one_large_gaussian_is_spread_over_the_warp(cuda_device):
    """A single Gaussian whose box covers every tile of a 256^3 volume at
    tile edge 4 (262,144 pairs) next to small ones: the pairs of the large
    one are emitted by the whole warp, in the reference's raster order."""
    shape, ts = (256, 256, 256), 4
    gs = synthetic.random_gaussians(40, shape, seed=91)
    c, r, _ = O.preprocess_f32(gs.positions.numpy(), gs.scales.numpy(), gs.rotations.numpy(), shape)
    c[7] = 127.5
    r[7] = 400.0
    center, radius = torch.tensor(c, device=cuda_device), torch.tensor(r, device=cuda_device)
    ref_tr, ref_pid = gs_tmi_b200.build_tile_pairs(center, radius, shape, ts)
    rc, total, tr, pid = _noalloc(center, radius, shape, ts, capacity=ref_pid.numel())
    assert rc == GSV_OK and total == ref_pid.numel() >= 64 ** 3
    assert np.array_equal(tr, ref_tr.cpu().numpy()) and np.array_equal(pid[:total], ref_pid.cpu().numpy())
