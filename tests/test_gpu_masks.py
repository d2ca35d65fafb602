"""Poisson-disc k-space masks on the GPU (gsv_poisson_masks): the parallel
greedy equals the reference's sequential dart throwing bit for bit -- on the
golden masks made by the reference's own generator, and against the CPU
oracle on batches of random visiting orders -- plus the edge cases."""
import os

import numpy as np
import pytest
import torch

from gs_tmi_b200 import masks
from gs_tmi_b200._lib import GsvError
from oracle import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "poisson_masks.npz")


def _golden():
    g = np.load(GOLDEN)
    out = []
    for k in range(int(g["ncases"])):
        ny, nz, accel, calib, seed = g[f"case{k}_params"]
        ny, nz, calib, seed = int(ny), int(nz), int(calib), int(seed)
        mask = np.unpackbits(g[f"case{k}_mask"])[:ny * nz].reshape(ny, nz).astype(np.int8)
        out.append(((ny, nz), float(accel), calib, seed, mask))
    return out


@pytest.mark.parametrize("k", range(8))
def test_golden_reference_masks(k, cuda_device):
    shape, accel, calib, seed, ref = _golden()[k]
    m, rounds = masks.poisson_masks(shape, accel, calib, seeds=[seed], device=cuda_device, return_rounds=True)
    assert np.array_equal(m[0].cpu().numpy(), ref)
    assert 0 <= int(rounds[0]) < 64
    # the drop-in draws its order from numpy's global state, as the reference does
    np.random.seed(seed)
    assert np.array_equal(masks.gen_poisson_mask(shape, accel, calib, device=cuda_device), ref)


@pytest.mark.parametrize("shape,accel,calib,count", [((256, 256), 6.0, 24, 12), ((160, 128), 8.0, 20, 24),
                                                     ((64, 48), 4.0, 8, 64), ((512, 384), 10.0, 32, 3)])
def test_batches_match_the_oracle(shape, accel, calib, count, cuda_device):
    n = shape[0] * shape[1]
    rs = np.random.RandomState(n + count)
    orders = np.stack([rs.permutation(n) for _ in range(count)]).astype(np.int32)
    m, rounds = masks.poisson_masks(shape, accel, calib, orders=orders, device=cuda_device, return_rounds=True)
    m = m.cpu().numpy()
    radius = masks.exclusion_radius(shape, accel, calib)
    target = masks.target_points(shape, accel)
    for b in range(count):
        ref = oracle.poisson_mask(radius, orders[b], shape, calib, target)
        assert np.array_equal(m[b], ref), b
        assert int(m[b].sum()) == target
    assert int(rounds.max()) < 64


def test_edge_cases(cuda_device):
    # an order that is not a permutation is refused
    bad = np.arange(32 * 32, dtype=np.int32)
    bad[5] = 7
    with pytest.raises(ValueError):
        masks.poisson_masks((32, 32), 4.0, 8, orders=bad[None], device=cuda_device)
    # more pixels than the shared-memory state holds
    with pytest.raises(GsvError):
        masks.poisson_masks((512, 385), 4.0, 8, seeds=[0], device=cuda_device)
    # no calibration square, and a tiny plane
    for shape, calib in (((40, 30), 0), ((1, 7), 2), ((3, 3), 1)):
        order = np.random.RandomState(1).permutation(shape[0] * shape[1]).astype(np.int32)
        got = masks.poisson_masks(shape, 2.0, calib, orders=order[None], device=cuda_device)[0].cpu().numpy()
        ref = oracle.poisson_mask(masks.exclusion_radius(shape, 2.0, calib), order, shape, calib,
                                  masks.target_points(shape, 2.0))
        assert np.array_equal(got, ref)
    # expansion along the readout axis
    m2 = torch.tensor([[1, 0], [0, 1]], dtype=torch.float32)
    e = masks.expand_phase_mask(m2, (3, 2, 2), (1, 2))
    assert e.shape == (3, 2, 2) and torch.equal(e[1], m2)


def test_mri_case_with_the_reference_mask(cuda_device):
    """synthetic.mri_case(mask_kind="poisson"): the (ky, kz) plane is the
    reference generator's mask for the order RandomState(seed + 3) draws,
    repeated along the fully sampled readout axis."""
    from gs_tmi_b200 import synthetic

    shape, accel, calib, seed = (12, 48, 40), 6.0, 12, 5
    case = synthetic.mri_case(shape, n_coils=2, accel=accel, calib=calib, seed=seed, mask_kind="poisson")
    order = np.random.RandomState(seed + 3).permutation(48 * 40).astype(np.int32)
    ref = oracle.poisson_mask(masks.exclusion_radius((48, 40), accel, calib), order, (48, 40), calib,
                              masks.target_points((48, 40), accel))
    m = case.mask.numpy()
    assert m.shape == shape and all(np.array_equal(m[i], ref) for i in range(shape[0]))
