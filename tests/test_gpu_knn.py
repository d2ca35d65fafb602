"""Intensity-seeded initialisation on the GPU: the library's exact grid
3-NN (gsv_knn3_mean_distance) against scipy's cKDTree on the same seeds,
which is what the reference uses (gaussian_model.py:283-306): same seeds,
positions and densities, bit-identical scales (FP64 distances of the FP32
positions in the k-d tree's order, FP32 mean), on cubic and
non-cubic volumes, dense and sparse seeds, and 1-3 seeds."""
import pytest
import torch

from gs_tmi_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,n", [((32, 32, 32), 3000), ((40, 28, 20), 20_000), ((64, 48, 40), 300),
                                     ((16, 16, 16), 1), ((16, 16, 16), 2), ((16, 16, 16), 3),
                                     ((128, 128, 96), 50_000)])
def test_gpu_knn_init_matches_cktree(shape, n, cuda_device):
    img = synthetic.ellipsoid_phantom(shape, seed=n % 7)
    cpu = synthetic.from_image_init(img, n, seed=3)
    gpu = synthetic.from_image_init(img, n, seed=3, device=cuda_device)
    torch.cuda.synchronize()
    assert torch.equal(gpu.positions.cpu(), cpu.positions)
    assert torch.equal(gpu.density_r.cpu(), cpu.density_r) and torch.equal(gpu.density_i.cpu(), cpu.density_i)
    assert torch.equal(gpu.scales.cpu(), cpu.scales)


def test_importance_seeds_are_the_same_on_the_device(cuda_device):
    """The reference's importance seeding (voxels above the 90th magnitude
    percentile) gives the same seeds whether the percentile and the
    candidate search run on the host or on the device."""
    case = synthetic.mri_case((48, 40, 36), n_coils=4, accel=4.0, calib=12, seed=11)
    for n in (500, 6000, 10 ** 6):  # the last exceeds the candidates: every voxel is a candidate
        a = synthetic.seed_indices(case.zero_filled, n, 3, "importance")
        b = synthetic.seed_indices(case.zero_filled, n, 3, "importance", device=cuda_device)
        assert torch.equal(a, b)
