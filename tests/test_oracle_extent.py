"""The tile-8 kernels skip a Gaussian, or a 4x8x8 row slot of it, when its
conservative tight extent misses the CTA's voxels.  That is only correct if
no voxel the shared FP32 predicate includes lies outside the extent: checked
here on the CPU for every listed (voxel, Gaussian) pair of isotropic,
image-seeded, strongly anisotropic and edge-case sets."""
import numpy as np
import pytest
import torch

from gs_tmi_b200 import synthetic
from oracle import oracle as O


def _check(gs, shape):
    p = [t.numpy() for t in gs.tensors()]
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    tr, pid = O.build_tile_pairs(c, r, shape, 8)
    bad, stats = O.extent_check(*p[:3], shape, tr, pid)
    assert bad == 0
    assert stats["listed"] == pid.size
    return stats


def test_extent_cull_random_cube():
    stats = _check(synthetic.random_gaussians(20000, (64, 64, 64), seed=0), (64, 64, 64))
    # the isotropic 3-sigma box over-covers: about half the pairs are culled
    assert stats["kept"] < 0.6 * stats["listed"]


def test_extent_cull_edge_cases():
    shape = (40, 40, 40)
    _check(synthetic.edge_case_gaussians(shape), shape)
    _check(synthetic.edge_case_gaussians((13, 11, 9), seed=4), (13, 11, 9))


@pytest.mark.parametrize("spread", [0.5, 1.5, 3.0])
def test_extent_cull_anisotropic(spread):
    rng = np.random.default_rng(int(spread * 10))
    n, shape = 4000, (48, 40, 56)
    pos = torch.tensor(rng.uniform(-1.1, 1.1, (n, 3)), dtype=torch.float32)
    vox = np.exp(rng.normal(np.log(2.0), spread, (n, 3)))  # scale ratios up to ~1e4
    scl = torch.tensor(vox / (np.array(shape) / 2), dtype=torch.float32)
    q = torch.tensor(rng.normal(size=(n, 4)) * rng.uniform(0.01, 3, (n, 1)), dtype=torch.float32)
    _check(synthetic.GaussianSet(pos, scl, q, torch.zeros(n), torch.zeros(n)), shape)


def test_extent_cull_image_seeded():
    shape = (64, 64, 48)
    case = synthetic.mri_case(shape, n_coils=4, accel=4.0, calib=16, seed=3)
    _check(synthetic.from_image_init(case.zero_filled, 20000, seed=1), shape)
