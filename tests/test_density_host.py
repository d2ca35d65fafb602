"""Host logic of the device density control (gs_tmi_b200.density) on the
CPU: the capacity-sized live rows, their growth, the optimizer-state view
handed to gsv_density_control, and the mask plane expansion.  No kernel is
launched here."""
import torch

from gs_tmi_b200 import density, masks, sense, synthetic


def _set(n, seed=0):
    return synthetic.random_gaussians(n, (16, 16, 16), seed=seed)


def test_live_rows_park_the_tail():
    gs = _set(10)
    p = density.LiveGaussianParams(gs, "cpu", 16)
    assert p.capacity == 16 and p.n == 10
    assert torch.equal(p.positions[:10], gs.positions)
    assert torch.allclose(torch.exp(p.log_scales[:10]), gs.scales, rtol=1e-6)
    assert not p.positions[10:].any() and not p.log_scales[10:].any()
    assert torch.equal(p.rotations[10:], torch.tensor([[1.0, 0, 0, 0]]).repeat(6, 1))
    assert not p.density_r[10:].any() and not p.density_i[10:].any()
    snap = p.snapshot()
    assert snap.positions.shape == (10, 3)


def test_live_rows_grow_in_place_order():
    p = density.LiveGaussianParams(_set(12, 1), "cpu", 12)
    q = p.grown(40)
    assert q.capacity == 40 and q.n == 12
    for a, b in zip(q.tensors(), p.tensors()):
        assert torch.equal(a[:12], b)
    assert torch.equal(q.rotations[12:, 0], torch.ones(28))


def test_rows_view_needs_full_adam_state():
    cfg = sense.FitConfig()
    p = density.LiveGaussianParams(_set(8, 2), "cpu", 32)
    dd = density.DeviceDensity(32, cfg, "cpu")
    opt = sense.make_optimizer(p, cfg, fused=False)
    r = dd.rows(p, opt)  # no Adam state yet: moments passed as NULL
    assert all(v is None for v in r.exp_avg) and r.capacity == 32
    for t in p.tensors():
        t.grad = torch.zeros_like(t)
    opt.step()
    r = dd.rows(p, opt)
    assert all(v for v in r.exp_avg) and all(v for v in r.exp_avg_sq)
    assert r.positions == p.positions.data_ptr()


def test_expand_phase_mask():
    m2 = torch.tensor([[1.0, 0.0, 1.0], [0.0, 1.0, 0.0]])
    e = masks.expand_phase_mask(m2, (4, 2, 3), (1, 2))
    assert e.shape == (4, 2, 3) and all(torch.equal(e[i], m2) for i in range(4))
    e = masks.expand_phase_mask(m2, (2, 5, 3), (0, 2))
    assert e.shape == (2, 5, 3) and all(torch.equal(e[:, j, :], m2) for j in range(5))
