"""Host-side checks of the warm start's training loss (no GPU).

The "dc" loss compares only the k-space that hard data consistency leaves in
place (``warmstart._unsampled``).  The training cases share one coil-map
tensor per shape because the synthetic maps of different seeds differ by a
constant phase per coil, which that map cancels."""
import torch

from gs_tmi_b200 import synthetic, warmstart


def _vol(shape, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g))


def test_unsampled_ignores_the_per_coil_phase():
    shape = (12, 16, 20)
    s1 = synthetic.ring_coils(shape, 4, seed=3)
    s2 = synthetic.ring_coils(shape, 4, seed=11)
    # the maps do differ (by a constant phase per coil) ...
    assert float((s1 - s2).abs().max()) > 0.1
    ratio = s2 / s1
    assert torch.allclose(ratio, ratio.reshape(4, -1)[:, :1].reshape(4, 1, 1, 1).expand_as(ratio), atol=1e-5)
    m = synthetic.variable_density_mask(shape, 4.0, calib=4, seed=5)
    v = _vol(shape, 0)
    a = warmstart._unsampled(v, s1, m)
    b = warmstart._unsampled(v, s2, m)
    # ... and the loss map does not
    assert float((a - b).abs().max()) <= 1e-5 * float(a.abs().max())


def test_unsampled_bool_mask_equals_float_mask():
    shape = (8, 12, 10)
    s = synthetic.ring_coils(shape, 3, seed=1)
    m = synthetic.variable_density_mask(shape, 3.0, calib=4, seed=2)
    v = _vol(shape, 1)
    assert torch.equal(warmstart._unsampled(v, s, m), warmstart._unsampled(v, s, m > 0.5))


def test_unsampled_is_zero_for_a_fully_sampled_mask():
    shape = (8, 8, 8)
    s = synthetic.ring_coils(shape, 2, seed=0)
    v = _vol(shape, 2)
    out = warmstart._unsampled(v, s, torch.ones(shape))
    assert float(out.abs().max()) == 0.0
