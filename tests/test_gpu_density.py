"""Device-side density control (gsv_density_control, gs_tmi_b200.density)
against the host-side restatement of the reference's split / clone / prune
and Adam-state transplant (sense.density_control + sense.transplant,
trainer.py:294-424, gaussian_model.py:85-222) on the same rows, moments and
split noise: same live count and row order; parameters equal to FP32
rounding of exp/log (rtol 1e-6), moments bitwise; vacated rows parked.
Then the live-row voxelizer, the Philox noise, and whole fits."""
import dataclasses

import pytest
import torch

from gs_tmi_b200 import density, sense, synthetic
from gs_tmi_b200._lib import (GSV_DENSITY_CLONE, GSV_DENSITY_PRUNE, GSV_DENSITY_ROW_OVERFLOW, GSV_DENSITY_SPLIT)

pytestmark = pytest.mark.gpu


def _rows(n, seed, dev, small_scales=False, few_prunes=False):
    """n Gaussians whose gradient norms, max scales and |rho| keep clear of
    the thresholds (0.01 / 0.01 / 0.01, max scale 0.5) by >= 2%."""
    g = torch.Generator().manual_seed(seed)
    pos = torch.rand(n, 3, generator=g) * 2 - 1
    lo, hi = (0.002, 0.0098) if small_scales else (0.002, 0.05)
    scales = lo + (hi - lo) * torch.rand(n, 3, generator=g)
    smax = scales.max(-1)[0]
    near = (smax > 0.0098) & (smax < 0.0102)
    scales[near] *= 1.05
    if not small_scales and not few_prunes:
        scales[torch.rand(n, generator=g) < 0.02] = 0.6  # over max_scale: pruned
    rot = torch.randn(n, 4, generator=g)
    mag = 0.001 + 0.2 * torch.rand(n, generator=g)
    if few_prunes:
        mag = 0.03 + 0.2 * torch.rand(n, generator=g)
    # |rho| of parents and of their children (x0.5, x0.6) clear of 0.01
    for edge in (0.01, 0.02, 0.01 / 0.6):
        mag[(mag > 0.98 * edge) & (mag < 1.02 * edge)] = 0.05
    ph = torch.rand(n, generator=g) * 6.283
    dr, di = mag * torch.cos(ph), mag * torch.sin(ph)
    gdir = torch.nn.functional.normalize(torch.randn(n, 3, generator=g), dim=-1)
    gmag = 0.03 * torch.rand(n, generator=g)
    gmag[(gmag > 0.0098) & (gmag < 0.0102)] = 0.02
    grad = gdir * gmag[:, None]
    gs = synthetic.GaussianSet(pos, scales, rot, dr, di)
    moments = [(torch.randn(n, w, generator=g).squeeze(-1), torch.rand(n, w, generator=g).squeeze(-1))
               for w in (3, 3, 4, 1, 1)]
    noise = torch.randn(n, 6, generator=g)
    return gs, grad, moments, noise


def _host(gs, grad, moments, noise, cfg, dev, with_state=True):
    p = sense.GaussianParams(gs, dev)
    opt = sense.make_optimizer(p, cfg, capturable=True)
    if with_state:
        for t, (m, v) in zip(p.tensors(), moments):
            opt.state[t] = {"step": torch.tensor(7.0, device=dev), "exp_avg": m.to(dev).reshape(t.shape).clone(),
                            "exp_avg_sq": v.to(dev).reshape(t.shape).clone()}
    holder = [opt]

    def rebuild(keep):
        new = sense.make_optimizer(p, cfg, capturable=True)
        sense.transplant(holder[0], new, keep, p.n)
        holder[0] = new

    events = sense.density_control(p, grad.to(dev), cfg, None, rebuild, noise=noise.to(dev))
    return p, holder[0], events


def _device(gs, grad, moments, noise, cfg, dev, cap, with_state=True):
    n = gs.positions.shape[0]
    p = density.LiveGaussianParams(gs, dev, cap)
    opt = sense.make_optimizer(p, cfg, capturable=True)
    if with_state:
        for t, (m, v) in zip(p.tensors(), moments):
            em, ev = torch.zeros_like(t), torch.zeros_like(t)
            em[:n] = m.to(dev).reshape(em[:n].shape)
            ev[:n] = v.to(dev).reshape(ev[:n].shape)
            opt.state[t] = {"step": torch.tensor(7.0, device=dev), "exp_avg": em, "exp_avg_sq": ev}
    dd = density.DeviceDensity(cap, cfg, dev)
    gpad = torch.zeros(cap, 3, device=dev)
    gpad[:n] = grad.to(dev)
    npad = torch.zeros(cap, 6, device=dev)
    npad[:n] = noise.to(dev)
    report = dd(p, opt if with_state else None, gpad, None if cfg.long_axis_split else npad)
    torch.cuda.synchronize()
    return p, opt, [int(v) for v in report.cpu()]


def _compare(ph, oh, pd, od, n_before, with_state=True, rtol=1e-6, atol=0.0):
    n = ph.n
    assert pd.n == n
    for a, b in zip(pd.tensors(), ph.tensors()):
        assert torch.allclose(a[:n], b, rtol=rtol, atol=atol), (a[:n] - b).abs().max()
    if with_state:
        for a, b in zip(pd.tensors(), ph.tensors()):
            for key in ("exp_avg", "exp_avg_sq"):
                assert torch.equal(od.state[a][key][:n], oh.state[b][key]), key
    # vacated rows are parked
    if n < n_before:
        assert not pd.positions[n:n_before].any() and not pd.density_r[n:n_before].any()
        assert torch.equal(pd.rotations[n:n_before, 0], torch.ones(n_before - n, device=pd.positions.device))
        if with_state:
            for a in pd.tensors():
                assert not od.state[a]["exp_avg"][n:n_before].any()


CASES = {
    # name: (n, cap, cfg overrides, _rows kwargs, expected flags)
    "split_and_prune": (6000, 16384, {}, {}, GSV_DENSITY_SPLIT | GSV_DENSITY_PRUNE),
    "clone_and_prune": (6000, 16384, {}, {"small_scales": True}, GSV_DENSITY_CLONE | GSV_DENSITY_PRUNE),
    "prune_only": (6000, 16384, {"use_cloning": False}, {"small_scales": True}, GSV_DENSITY_PRUNE),
    "at_max_points": (6000, 16384, {"max_points": 6000}, {}, 0),
    "split_over_max_falls_to_clone": (6000, 16384, {"max_points": 6100}, {},
                                      GSV_DENSITY_CLONE | GSV_DENSITY_PRUNE),
    "long_axis": (6000, 16384, {"long_axis_split": True, "use_cloning": False, "long_axis_offset_factor": 1.5}, {},
                  GSV_DENSITY_SPLIT | GSV_DENSITY_PRUNE),
    "min_keep": (150, 4096, {}, {}, GSV_DENSITY_SPLIT),
    "no_prune": (6000, 16384, {}, {"few_prunes": True}, GSV_DENSITY_SPLIT),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_density_matches_host(name, cuda_device):
    n, cap, over, kw, expect = CASES[name]
    dev = cuda_device
    gs, grad, moments, noise = _rows(n, seed=len(name), dev=dev, **kw)
    if name == "min_keep":  # most rows prunable: fewer than 100 survive, so nothing is pruned
        gs.density_r[:120] = 0.001
        gs.density_i[:120] = 0.0
    cfg = dataclasses.replace(sense.FitConfig(), **over)
    ph, oh, events = _host(gs, grad, moments, noise, cfg, dev)
    pd, od, rep = _device(gs, grad, moments, noise, cfg, dev, cap)
    assert rep[0] == expect, rep
    assert events == bin(expect & 7).count("1")
    if name == "long_axis":  # |q| and the rotated shift: torch reduction order, a few ulps
        _compare(ph, oh, pd, od, n + rep[1], rtol=2e-6, atol=1e-8)
    else:
        _compare(ph, oh, pd, od, n + rep[1] + rep[2])
    assert pd.n == n + rep[1] + rep[2] - rep[3]


def test_device_density_without_adam_state(cuda_device):
    gs, grad, moments, noise = _rows(5000, seed=11, dev=cuda_device)
    cfg = sense.FitConfig()
    ph, _, _ = _host(gs, grad, moments, noise, cfg, cuda_device, with_state=False)
    pd, _, rep = _device(gs, grad, moments, noise, cfg, cuda_device, 12288, with_state=False)
    assert rep[0] == GSV_DENSITY_SPLIT | GSV_DENSITY_PRUNE
    assert pd.n == ph.n
    for a, b in zip(pd.tensors(), ph.tensors()):
        assert torch.allclose(a[:ph.n], b, rtol=1e-6, atol=0)


def test_row_overflow_changes_nothing(cuda_device):
    gs, grad, moments, noise = _rows(6000, seed=3, dev=cuda_device)
    cfg = sense.FitConfig()
    pd, od, rep = _device(gs, grad, moments, noise, cfg, cuda_device, 6010)
    assert rep[0] == GSV_DENSITY_ROW_OVERFLOW and rep[1:] == [0, 0, 0]
    assert pd.n == 6000
    ref = density.LiveGaussianParams(gs, cuda_device, 6010)
    for a, b in zip(pd.tensors(), ref.tensors()):
        assert torch.equal(a, b)


def test_live_rows_voxelize_like_the_first_n(cuda_device):
    """Rows past the live count: no contribution, zero gradients; the
    volume and the live rows' gradients equal a plain n-row voxelizer's
    bitwise (deterministic backward)."""
    from gs_tmi_b200.tile_voxelizer import TileVoxelizer

    shape = (40, 36, 32)
    n, cap = 3000, 5000
    gs = synthetic.random_gaussians(cap, shape, seed=4)
    vox = TileVoxelizer(shape, device=str(cuda_device), deterministic=True)
    live = torch.tensor([n], dtype=torch.int32, device=cuda_device)
    full = [t.to(cuda_device).clone().requires_grad_(True) for t in
            (gs.positions, gs.scales, gs.rotations, gs.density_r, gs.density_i)]
    head = [t.detach()[:n].clone().requires_grad_(True) for t in full]
    cap_pairs = vox.count_pairs(full[0].detach(), full[1].detach()) + 1024
    sv = vox.static(cap, cap_pairs, live=live)
    v1 = sv(full[0], full[1], full[2], torch.complex(full[3], full[4]))
    v2 = vox(head[0], head[1], head[2], torch.complex(head[3], head[4]))
    assert torch.equal(v1, v2)
    g = torch.randn(v1.shape, dtype=torch.complex64, device=cuda_device)
    (v1 * g).real.sum().backward()
    (v2 * g).real.sum().backward()
    for a, b in zip(full, head):
        assert torch.equal(a.grad[:n], b.grad)
        assert not a.grad[n:].any()


def test_philox_normals(cuda_device):
    import ctypes

    from gs_tmi_b200._lib import check, lib

    counter = torch.zeros(1, dtype=torch.int64, device=cuda_device)
    count = 1_000_003
    out = [torch.empty(count, device=cuda_device) for _ in range(3)]

    def fill(t):
        check(lib.gsv_normal_fill(ctypes.c_void_p(t.data_ptr()), count, 1234, ctypes.c_void_p(counter.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "fill")

    fill(out[0])
    fill(out[1])
    counter.zero_()
    fill(out[2])
    torch.cuda.synchronize()
    assert int(counter) == 1
    assert torch.equal(out[0], out[2]) and not torch.equal(out[0], out[1])
    for t in out[:2]:
        assert torch.isfinite(t).all()
        assert abs(float(t.mean())) < 5e-3 and abs(float(t.std()) - 1) < 5e-3
        assert abs(float((t ** 3).mean())) < 2e-2 and abs(float((t ** 4).mean()) - 3) < 5e-2
    # the draw of row i does not depend on how many rows are drawn
    head = torch.empty(6 * 1000, device=cuda_device)
    counter.zero_()
    check(lib.gsv_normal_fill(ctypes.c_void_p(head.data_ptr()), head.numel(), 1234,
                              ctypes.c_void_p(counter.data_ptr()),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "fill")
    torch.cuda.synchronize()
    assert torch.equal(head, out[0][:6000])


def _small_fit():
    shape = (48, 48, 40)
    case = synthetic.mri_case(shape, n_coils=4, accel=4.0, calib=12, seed=5)
    init = synthetic.from_image_init(case.zero_filled, 4000, seed=6)
    cfg = sense.FitConfig(iterations=320, eval_every=50, max_points=40000, deterministic=True,
                          capturable_adam=True)
    return case, init, cfg


def test_live_fit_matches_host_density_fit(cuda_device):
    """Without gradient clipping (whose norm reduction depends on the row
    count) the graph-replayed live-row fit equals the eager fit with host
    density control and the same Philox split noise bitwise, through three
    densification steps, with two graph captures in all."""
    case, init, cfg = _small_fit()
    cfg.max_grad_norm = 0.0
    dev = str(cuda_device)
    eager = sense.fit(case, init, cfg, device=dev, eval_ssim=False,
                      split_noise=density.philox_noise(cfg.seed, cuda_device))
    st = {}
    live = density.fit_live(case, init, cfg, device=dev, eval_ssim=False, stats=st)
    assert st["row_growths"] == 0 and 2 <= st["captures"] <= 2 + 2 * st["overflows"]
    assert st["events"] >= 2
    n = eager.params.n
    assert live.params.n == n
    for a, b in zip(live.params.tensors(), eager.params.tensors()):
        assert torch.equal(a[:n], b)
    assert [r["n_points"] for r in live.history] == [r["n_points"] for r in eager.history]
    assert live.final_nmse == eager.final_nmse


def test_live_fit_with_clipping_and_growth(cuda_device):
    """With clipping, and with rows and pair capacity too small at the start
    (undo, grow, re-capture): the same trajectory as the host fit to float
    rounding (the clip norm's reduction order depends on the row count):
    final count within 2%, final NMSE within 1%."""
    case, init, cfg = _small_fit()
    dev = str(cuda_device)
    eager = sense.fit(case, init, cfg, device=dev, eval_ssim=False,
                      split_noise=density.philox_noise(cfg.seed, cuda_device))
    st = {}
    live = density.fit_live(case, init, cfg, device=dev, eval_ssim=False, stats=st, row_capacity=4001,
                            capacity_margin=0.6)
    assert st["overflows"] >= 1
    if max(r["n_points"] for r in eager.history) > 4001:
        assert st["row_growths"] >= 1
    assert abs(live.params.n - eager.params.n) <= 0.02 * eager.params.n
    assert abs(live.final_nmse - eager.final_nmse) <= 0.01 * eager.final_nmse
