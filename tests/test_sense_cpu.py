"""Host logic of the SENSE loop on the CPU: the loop, density control and
Adam-state transplant run with the CPU port of the reference voxelizer
(oracle/torch_port.py) standing in for the CUDA library."""
import numpy as np
import torch

from gs_tmi_b200 import sense, synthetic
from oracle import torch_port


def cpu_voxelizer(shape, ts=4):
    def vox(positions, scales, rotations, density):
        center, cov_inv, half = torch_port.preprocess(positions, scales, rotations, shape)
        with torch.no_grad():
            tr, pid = torch_port.build_tile_pairs_torch(center.detach(), torch_port.radius_vox(scales.detach(), half),
                                                        shape, ts)
        tiles = range(tr.shape[0])
        return torch_port.tile_forward(center, cov_inv, density, half, tr.numpy(), pid.numpy(), shape, ts,
                                       tiles).view(*shape)
    return vox


def test_fit_loop_and_density_control_on_cpu():
    shape = (16, 16, 12)
    case = synthetic.mri_case(shape, n_coils=2, accel=3.0, calib=6, seed=3)
    init = synthetic.from_image_init(case.zero_filled, 300, seed=4)
    cfg = sense.FitConfig(iterations=25, densify_from=5, densify_every=10, densify_until=25, eval_every=8,
                          grad_threshold=1e-4, scale_threshold=0.05, max_points=2000)
    rows = []
    res = sense.fit(case, init, cfg, voxelizer=cpu_voxelizer(shape), device="cpu", log=rows.append,
                    eval_ssim=True)
    assert len(rows) >= 3
    assert min(r["loss"] for r in rows[1:]) < rows[0]["loss"]
    assert all(np.isfinite(r["nmse"]) for r in rows)
    ns = [r["n_points"] for r in rows]
    assert max(ns) != 300 or min(ns) != 300  # density control fired
    p = res.params
    assert all(t.shape[0] == p.n for t in p.tensors())
    assert np.isfinite(res.final_nmse) and 0 < res.final_ssim <= 1


def test_transplant_keeps_moments_of_surviving_rows():
    shape = (8, 8, 8)
    gs = synthetic.random_gaussians(10, shape, seed=1)
    p = sense.GaussianParams(gs, "cpu")
    cfg = sense.FitConfig()
    opt = sense.make_optimizer(p, cfg, fused=False)
    for t in p.tensors():
        t.grad = torch.randn_like(t)
    opt.step()
    keep = torch.tensor([True, False] * 5)
    old = [opt.state[t]["exp_avg"].clone() for t in p.tensors()]
    p.replace([torch.cat([t[keep], t[:3]]) for t in p.tensors()])
    new_opt = sense.make_optimizer(p, cfg, fused=False)
    sense.transplant(opt, new_opt, keep, p.n)
    for o, t in zip(old, p.tensors()):
        st = new_opt.state[t]["exp_avg"]
        assert st.shape[0] == 8
        assert torch.equal(st[:5], o[keep]) and not st[5:].any()


def test_metrics():
    g = torch.Generator().manual_seed(0)
    x = torch.complex(torch.rand(12, 12, 12, generator=g), torch.rand(12, 12, 12, generator=g))
    assert sense.nmse(x, x) == 0.0
    assert abs(sense.ssim3d(x, x) - 1.0) < 1e-12
    y = x + 0.05 * torch.rand(12, 12, 12, generator=g)
    assert 0 < sense.ssim3d(y, x) < 1 and sense.nmse(y, x) > 0
    # SSIM against a direct evaluation of the definition at one window
    a, b = x.abs().double().numpy(), y.abs().double().numpy()
    L = b.max() - b.min()
    wa, wb = a[:7, :7, :7].ravel(), b[:7, :7, :7].ravel()
    c1, c2 = (0.01 * L) ** 2, (0.03 * L) ** 2
    s = ((2 * wa.mean() * wb.mean() + c1) * (2 * np.cov(wa, wb)[0, 1] + c2)) / (
        (wa.mean() ** 2 + wb.mean() ** 2 + c1) * (wa.var(ddof=1) + wb.var(ddof=1) + c2))
    import torch.nn.functional as F  # noqa: F401

    xa = torch.tensor(a)[None, None]
    yb = torch.tensor(b)[None, None]
    one = sense.ssim3d(torch.tensor(a[:7, :7, :7]).to(torch.complex128), torch.tensor(b[:7, :7, :7]).to(torch.complex128),
                       data_range=L)
    assert abs(one - s) < 1e-10
    del xa, yb


def _params(pos, scales, rot, dr, di):
    return sense.GaussianParams(synthetic.GaussianSet(torch.tensor(pos), torch.tensor(scales), torch.tensor(rot),
                                                      torch.tensor(dr), torch.tensor(di)), "cpu")


def test_long_axis_split_on_cpu():
    """gaussian_model.py:112-131: the longest axis halves, the others shrink
    by 0.85, the children sit at +/- child_scale along the rotated axis,
    densities x0.6; the survivors come first."""
    p = _params([[0.1, 0.2, 0.3], [0.0, 0.0, 0.0]], [[0.02, 0.05, 0.03], [0.02, 0.02, 0.02]],
                [[1.0, 0.0, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0]], [1.0, 2.0], [0.5, 1.0])
    cfg = sense.FitConfig(long_axis_split=True, use_cloning=False, grad_threshold=0.01, scale_threshold=0.03,
                          opacity_threshold=0.01, max_points=100)
    grad = torch.tensor([[0.02, 0.0, 0.0], [0.02, 0.0, 0.0]])
    events = sense.density_control(p, grad, cfg, None, lambda keep: None)
    assert events == 1 and p.n == 3
    assert torch.equal(p.positions[0], torch.tensor([0.0, 0.0, 0.0]))  # the survivor
    child = torch.tensor([0.02 * 0.85, 0.05 * 0.5, 0.03 * 0.85])
    for row, sign in ((1, 1.0), (2, -1.0)):
        assert torch.allclose(p.positions[row], torch.tensor([0.1, 0.2 + sign * 0.025, 0.3]), atol=1e-7)
        assert torch.allclose(torch.exp(p.log_scales[row]), child, rtol=1e-6)
        assert torch.allclose(p.density_r[row], torch.tensor(0.6)) and torch.allclose(p.density_i[row],
                                                                                      torch.tensor(0.3))


def test_split_noise_and_prune_on_cpu():
    """Children at parent + z * s / 2 with the given noise, scales s / 1.6;
    |rho| below the opacity threshold is pruned (complex magnitude)."""
    n = 120
    g = torch.Generator().manual_seed(0)
    pos = (torch.rand(n, 3, generator=g) * 2 - 1)
    scales = torch.full((n, 3), 0.005)
    scales[0] = 0.05                                   # the one split parent
    rot = torch.zeros(n, 4)
    rot[:, 0] = 1.0
    dr = torch.full((n,), 0.5)
    di = torch.zeros(n)
    dr[5], di[5] = 0.006, 0.008                         # |rho| = 0.01: kept (not < 0.01)
    dr[6], di[6] = 0.006, 0.007                         # |rho| < 0.01: pruned
    p = sense.GaussianParams(synthetic.GaussianSet(pos, scales, rot, dr, di), "cpu")
    grad = torch.zeros(n, 3)
    grad[0, 0] = 1.0
    noise = torch.randn(n, 6, generator=g)
    cfg = sense.FitConfig(max_points=10_000)
    keeps = []
    events = sense.density_control(p, grad, cfg, None, keeps.append, noise=noise)
    assert events == 2 and p.n == n + 1 - 1
    # after the split: rows 1..n-1, then the two children; then row 6 pruned
    s0 = torch.exp(torch.log(torch.tensor(0.05)))
    a = pos[0] + noise[0, :3] * s0 * 0.5
    b = pos[0] + noise[0, 3:] * s0 * 0.5
    assert torch.equal(p.positions[-2], a) and torch.equal(p.positions[-1], b)
    assert torch.allclose(torch.exp(p.log_scales[-1]), torch.full((3,), 0.05 / 1.6), rtol=1e-6)
    assert not torch.isclose(p.density_r, torch.tensor(0.006)).logical_and(
        torch.isclose(p.density_i, torch.tensor(0.007))).any()
    assert torch.isclose(p.density_i, torch.tensor(0.008)).sum() == 1


def test_density_control_branches_on_cpu():
    """The reference's branch order (trainer.py:300-352): nothing at
    max_points; split when it fits, else clone; clone halves the parent's
    density and appends a copy with log(scale + 1e-8); prune only when at
    least 100 rows survive."""
    n = 150
    g = torch.Generator().manual_seed(3)
    pos = torch.rand(n, 3, generator=g) * 2 - 1
    rot = torch.zeros(n, 4)
    rot[:, 0] = 1.0
    dr = torch.full((n,), 0.5)
    di = torch.full((n,), 0.1)
    grad = torch.zeros(n, 3)
    grad[:4, 0] = 1.0                      # four densify candidates
    small = torch.full((n, 3), 0.005)      # all below the scale threshold: clone
    cfg = sense.FitConfig(max_points=10_000)
    events = []
    p = sense.GaussianParams(synthetic.GaussianSet(pos, small, rot, dr, di), "cpu")
    assert sense.density_control(p, grad, cfg, None, events.append) == 1 and p.n == n + 4
    assert torch.equal(p.density_r[:4], torch.full((4,), 0.25)) and torch.equal(p.density_r[n:], p.density_r[:4])
    assert torch.equal(p.positions[n:], pos[:4])
    assert torch.allclose(p.log_scales[n:], torch.log(torch.full((4, 3), 0.005) + 1e-8))
    # at max_points nothing happens, not even a prune
    p = sense.GaussianParams(synthetic.GaussianSet(pos, small, rot, dr * 0, di * 0), "cpu")
    assert sense.density_control(p, grad, sense.FitConfig(max_points=n), None, events.append) == 0 and p.n == n
    # a split that would pass max_points falls back to clone; cloning off: nothing but the prune test
    big = torch.full((n, 3), 0.05)
    p = sense.GaussianParams(synthetic.GaussianSet(pos, big, rot, dr, di), "cpu")
    cfg2 = sense.FitConfig(max_points=n + 3, use_cloning=False)
    assert sense.density_control(p, grad, cfg2, None, events.append, noise=torch.zeros(n, 6)) == 0 and p.n == n
    # prune needs 100 survivors: 60 survivors -> no prune
    weak = dr.clone()
    weak[60:] = 0.001
    p = sense.GaussianParams(synthetic.GaussianSet(pos, big, rot, weak, di * 0), "cpu")
    assert sense.density_control(p, torch.zeros(n, 3), cfg, None, events.append) == 0 and p.n == n
    weak[110:] = 0.001
    weak[60:110] = 0.5
    p = sense.GaussianParams(synthetic.GaussianSet(pos, big, rot, weak, di * 0), "cpu")
    assert sense.density_control(p, torch.zeros(n, 3), cfg, None, events.append) == 1 and p.n == 110


def test_plateau_stop_follows_the_reference_rule():
    """V/metrics/metrics.py:166-195: an evaluation improves when some metric
    beats its best by more than its delta; `patience` evaluations in a row
    without improvement stop the fit, but not before `min_iterations`."""
    st = sense.PlateauStop(patience=2, min_iterations=100, min_delta={"psnr": 0.05, "ssim": 0.0005})
    seq = [(0, 20.0, 0.50), (50, 20.3, 0.51), (100, 20.33, 0.5103), (150, 20.34, 0.5104), (200, 20.2, 0.50)]
    out = [st.update(it, {"psnr": p, "ssim": s}) for it, p, s in seq]
    # 100 and 150: psnr +0.03 / +0.04 and ssim +0.0003 / +0.0004 stay within their deltas -> bad 1, 2: stop
    assert out == [False, False, False, True, True]
    # improvement resets the count; the minimum iteration holds the stop back
    st = sense.PlateauStop(patience=1, min_iterations=300)
    assert st.update(0, {"psnr": 10.0, "ssim": 0.1}) is False
    assert st.update(100, {"psnr": 10.0, "ssim": 0.1}) is False  # bad 1, but iteration < 300
    assert st.update(300, {"psnr": 10.2, "ssim": 0.1}) is False  # psnr improved: reset
    assert st.update(350, {"psnr": 10.2, "ssim": 0.1}) is True
