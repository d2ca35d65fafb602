"""The fused SENSE data term (gsv_sense_expand / residual / adjoint around
torch.fft) against the same term written op by op in torch: the loss value
and its gradient with respect to the volume, on even and odd volume sizes
(the FFT shifts are folded into the kernels' indexing).  FP32 sums in a
different order: relative error bar 1e-5."""
import pytest
import torch

from gs_tmi_b200 import sense, synthetic

pytestmark = pytest.mark.gpu


def _crand(shape, g, dev):
    return torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g)).to(dev)


@pytest.mark.parametrize("shape,nc", [((16, 12, 10), 3), ((13, 11, 9), 4), ((32, 32, 24), 8)])
def test_fused_data_term_matches_torch(shape, nc, cuda_device):
    g = torch.Generator().manual_seed(sum(shape) + nc)
    vol = _crand(shape, g, cuda_device)
    S = _crand((nc, *shape), g, cuda_device)
    mask = (torch.rand(shape, generator=g) < 0.4).float().to(cuda_device)
    ku = _crand((nc, *shape), g, cuda_device) * mask
    v1 = vol.clone().requires_grad_(True)
    l1 = sense.sense_data_term(v1, S, mask, ku)
    l1.backward()
    v2 = vol.clone().requires_grad_(True)
    l2 = sense.data_term_reference(v2, S, mask.unsqueeze(0), ku)
    l2.backward()
    assert abs(float(l1.detach()) - float(l2.detach())) <= 1e-5 * abs(float(l2.detach()))
    assert float((v1.grad - v2.grad).abs().norm() / v2.grad.abs().norm()) < 1e-5


def test_fused_data_term_in_a_fit(cuda_device):
    """Same fit (deterministic voxelizer, no densification) with the fused
    and the op-by-op data term: both improve on the start, and their NMSE
    after 60 iterations agrees to 2% (Adam amplifies the FP32 rounding
    differences of the two sum orders over the iterations)."""
    case = synthetic.mri_case((32, 32, 24), n_coils=4, accel=4.0, calib=8, seed=5)
    init = synthetic.from_image_init(case.zero_filled, 3000, seed=5)
    out = []
    for fused in (True, False):
        cfg = sense.FitConfig(iterations=60, eval_every=59, densify_from=10 ** 9, fused_sense=fused,
                              deterministic=True)
        r = sense.fit(case, init, cfg, device=str(cuda_device), eval_ssim=False)
        assert r.final_nmse < r.history[0]["nmse"]
        out.append(r.final_nmse)
    assert abs(out[0] - out[1]) <= 2e-2 * out[1]


@pytest.mark.parametrize("shape", [(16, 12, 10), (13, 11, 9), (1, 7, 5)])
def test_fused_tv_matches_torch(shape, cuda_device):
    g = torch.Generator().manual_seed(sum(shape))
    vol = _crand(shape, g, cuda_device)
    vol[0, 0, 0] = 0  # |x| = 0: zero gradient, as torch's abs backward
    v1 = vol.clone().requires_grad_(True)
    l1 = sense.magnitude_tv_fused(v1)
    (3 * l1).backward()
    v2 = vol.clone().requires_grad_(True)
    l2 = sense.magnitude_tv(v2)
    (3 * l2).backward()
    assert abs(float(l1.detach()) - float(l2.detach())) <= 1e-5 * abs(float(l2.detach()))
    assert float((v1.grad - v2.grad).abs().norm() / v2.grad.abs().norm()) < 1e-5
