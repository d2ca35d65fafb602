"""The two sorts of the binning give the same lists.

gsv_bin picks a counting sort over per-row tile counts when the tile grid is
small and an emit + radix sort + range pass otherwise (include/gsv.h,
gsv_bin_ex).  Here both run after one preprocess on the same workspace and
their tile ranges and pair ids are compared bit for bit: the benchmark
workloads, ragged volumes and tile edges 4/5/8/16, a Gaussian covering the
whole grid among small ones, parked rows (gsv_prepare_live), capacities
above and below the pair total, and a repeated bin after one preprocess.
The golden-vector and oracle tests check the lists themselves; these check
that the sort that did not run there agrees."""
import ctypes

import numpy as np
import pytest
import torch

from gs_tmi_b200 import _lib, synthetic
from gs_tmi_b200._lib import GsvParams, check, lib
from gs_tmi_b200.tile_voxelizer import BinPlan, _ptr, _shape, _stream

pytestmark = pytest.mark.gpu

RADIX, COUNTING = _lib.GSV_BIN_RADIX, _lib.GSV_BIN_COUNTING


def _prepare(params, shape, live=None):
    pos, scl, rot, dr, di = params
    dev = pos.device
    plan = BinPlan(shape, int(pos.shape[0]), dev)
    gp = GsvParams(pos.data_ptr(), scl.data_ptr(), rot.data_ptr(), dr.data_ptr(), di.data_ptr(), plan.n)
    total = ctypes.c_int64(0)
    if live is None:
        check(lib.gsv_prepare(ctypes.byref(gp), shape, _ptr(plan.ws_gauss), plan.gauss_bytes, ctypes.byref(total),
                              _stream(dev)), "gsv_prepare")
    else:
        check(lib.gsv_prepare_live(ctypes.byref(gp), _ptr(live), shape, _ptr(plan.ws_gauss), plan.gauss_bytes,
                                   ctypes.byref(total), _stream(dev)), "gsv_prepare_live")
    plan.total = int(total.value)
    return plan


def _bin(plan, mode, cap):
    """Bin into a fresh pair workspace of capacity `cap`; returns (ranges,
    the first min(total, cap) pair ids, flags)."""
    plan.alloc_pairs(cap)
    rc = lib.gsv_bin_ex(plan.shape, plan.n, _ptr(plan.ws_gauss), _ptr(plan.ws_pairs), plan.pair_bytes, cap, mode,
                        _stream(plan.device))
    if rc != 0:
        return rc
    _, flags = plan.read_status(_stream(plan.device))
    tr_ptr, pid_ptr = plan.views()
    t = int(lib.gsv_num_tiles(plan.shape))
    o1 = tr_ptr - plan.ws_gauss.data_ptr()
    o2 = pid_ptr - plan.ws_pairs.data_ptr()
    tr = plan.ws_gauss[o1:o1 + 8 * t].view(torch.int32).reshape(t, 2).cpu().numpy()
    k = min(plan.total, cap)
    pid = plan.ws_pairs[o2:o2 + 4 * k].view(torch.int32).cpu().numpy()
    return tr, pid, flags


def _params(gs, dev):
    return tuple(t.to(dev).float().contiguous() for t in gs.tensors())


def _same_lists(plan, cap=None):
    cap = plan.total if cap is None else cap
    a = _bin(plan, COUNTING, cap)
    assert not isinstance(a, int), f"counting sort refused: rc={a}"
    b = _bin(plan, RADIX, cap)
    c = _bin(plan, COUNTING, cap)  # again after one preprocess
    for x in (b, c):
        assert np.array_equal(a[0], x[0]), "tile ranges differ"
        assert np.array_equal(a[1], x[1]), "pair ids differ"
        assert a[2] == x[2]
    return a


CASES = [
    # (shape, tile, n, kind)
    ((64, 64, 64), 8, 20_000, "random"),
    ((37, 29, 45), 8, 3_000, "random"),
    ((37, 29, 45), 5, 3_000, "random"),
    ((40, 48, 32), 4, 5_000, "random"),
    ((33, 70, 21), 16, 2_000, "random"),
    ((64, 64, 64), 8, 1, "random"),
    ((64, 64, 64), 8, 257, "random"),
]


@pytest.mark.parametrize("shape,ts,n,kind", CASES)
def test_counting_and_radix_sorts_agree(shape, ts, n, kind, cuda_device):
    gs = synthetic.random_gaussians(n, shape, seed=n + ts)
    plan = _prepare(_params(gs, cuda_device), _shape(shape, ts))
    tr, pid, flags = _same_lists(plan)
    assert flags == 0
    assert pid.size == plan.total


def test_benchmark_workload_lists_agree(cuda_device):
    """128x128x96 with 50,000 intensity-seeded Gaussians (3,072 tiles)."""
    import bench

    gs, _ = bench.make_inputs("mri128x128x96_n50k")
    plan = _prepare(_params(gs, cuda_device), _shape((128, 128, 96), 8))
    _same_lists(plan)


def test_whole_grid_gaussian_among_small_ones(cuda_device):
    """One Gaussian whose box covers every tile (its pairs span all of a
    warp's strided passes) between thousands of small ones."""
    shape = (48, 40, 56)
    gs = synthetic.random_gaussians(4_000, shape, seed=5)
    gs.scales[1234] = torch.tensor([2.0, 2.0, 2.0])
    plan = _prepare(_params(gs, cuda_device), _shape(shape, 8))
    tr, pid, _ = _same_lists(plan)
    assert (pid == 1234).sum() == int(lib.gsv_num_tiles(_shape(shape, 8)))


def test_parked_rows(cuda_device):
    """gsv_prepare_live: rows past the live count have no tiles."""
    shape = (64, 64, 64)
    gs = synthetic.random_gaussians(6_000, shape, seed=9)
    live = torch.tensor([4_321], dtype=torch.int32, device=cuda_device)
    plan = _prepare(_params(gs, cuda_device), _shape(shape, 8), live=live)
    tr, pid, _ = _same_lists(plan)
    assert pid.max() < 4_321


def test_capacities_above_and_below_the_total(cuda_device):
    shape = (64, 64, 64)
    gs = synthetic.random_gaussians(20_000, shape, seed=0)
    plan = _prepare(_params(gs, cuda_device), _shape(shape, 8))
    total = plan.total
    # a static capacity above the total: the same lists, no flag
    tr, pid, flags = _same_lists(plan, cap=total + 1000)
    assert flags == 0 and pid.size == total
    # below the total: both flag the overflow and keep every range inside the buffer
    cap = total - 777
    for mode in (COUNTING, RADIX):
        tr, _, flags = _bin(plan, mode, cap)
        assert flags & _lib.GSV_FLAG_CAPACITY_OVERFLOW
        assert tr.min() >= 0 and tr.max() <= cap and np.all(tr[:, 0] <= tr[:, 1])


def test_counting_sort_refused_where_it_does_not_apply(cuda_device):
    """More than 3072 tiles (the 256x256x160 volume has 20,480): the
    counting mode is refused, the automatic mode takes the radix sort."""
    shape = (256, 256, 160)
    gs = synthetic.random_gaussians(2_000, shape, seed=1)
    plan = _prepare(_params(gs, cuda_device), _shape(shape, 8))
    assert _bin(plan, COUNTING, plan.total) == _lib.GSV_ERR_INVALID_ARGUMENT
    tr, pid, flags = _bin(plan, _lib.GSV_BIN_AUTO, plan.total)
    assert flags == 0 and pid.size == plan.total
