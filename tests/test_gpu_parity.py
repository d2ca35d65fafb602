"""GPU parity: the sm_100a kernels (through the C ABI) against the FP64 oracle
and the reference's golden outputs.

Bars: binning bit-exact; forward relative L2 <= 1e-5 (FWD_TOL); every
gradient relative L2 <= 1e-4 (GRAD_TOL); deterministic mode bitwise
reproducible."""
import numpy as np
import pytest
import torch

import gs_tmi_b200
from gs_tmi_b200 import synthetic
from gs_tmi_b200.tile_voxelizer import _shape, prepare_and_bin
from oracle import oracle as O
from tests.helpers import FWD_TOL, GRAD_KEYS, GRAD_TOL, SMALL_CASES, load, params_of, rel

pytestmark = pytest.mark.gpu


def gpu_run(params, shape, ts, gv, deterministic=False, dev="cuda:0"):
    ts_ = [torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=dev, requires_grad=True)
           for x in params]
    vol = gs_tmi_b200.voxelize(*ts_, shape, ts, deterministic=deterministic)
    g = torch.tensor(np.asarray(gv), dtype=torch.complex64, device=dev)
    loss = (vol.real * g.real + vol.imag * g.imag).sum()
    loss.backward()
    torch.cuda.synchronize()
    return vol.detach().cpu().numpy(), [t.grad.detach().cpu().numpy() for t in ts_]


def plan_lists(plan):
    """Copy the tile ranges / pair ids out of a BinPlan's workspaces."""
    tr_ptr, pid_ptr = plan.views()
    t = gs_tmi_b200.num_tiles((plan.shape.d, plan.shape.h, plan.shape.w), plan.shape.tile_size)
    o1 = tr_ptr - plan.ws_gauss.data_ptr()
    o2 = pid_ptr - plan.ws_pairs.data_ptr()
    tr = plan.ws_gauss[o1:o1 + 8 * t].view(torch.int32).reshape(t, 2).cpu().numpy()
    pid = plan.ws_pairs[o2:o2 + 4 * plan.total].view(torch.int32).cpu().numpy()
    return tr, pid


@pytest.mark.parametrize("name", SMALL_CASES)
def test_binning_bit_exact(name, cuda_device):
    z = load(name)
    shape, ts = tuple(int(x) for x in z["shape"]), int(z["tile_size"])
    # reference-signature device binning from the reference's own center/radius
    tr, pid = gs_tmi_b200.build_tile_pairs(torch.tensor(z["center"], device=cuda_device),
                                           torch.tensor(z["radius"], device=cuda_device), shape, ts)
    assert np.array_equal(tr.cpu().numpy(), z["tile_ranges"])
    assert np.array_equal(pid.cpu().numpy(), z["pair_ids"])
    # fused path: preprocess + binning from the raw parameters
    params = tuple(torch.tensor(x, device=cuda_device) for x in params_of(z))
    plan = prepare_and_bin(params, _shape(shape, ts))
    tr2, pid2 = plan_lists(plan)
    assert np.array_equal(tr2, z["tile_ranges"]) and np.array_equal(pid2, z["pair_ids"])


@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("name", SMALL_CASES)
def test_forward_backward_vs_oracle(name, deterministic, cuda_device):
    z = load(name)
    shape, ts = tuple(int(x) for x in z["shape"]), int(z["tile_size"])
    p = params_of(z)
    vol, grads = gpu_run(p, shape, ts, z["grad_vol"], deterministic)
    ovol, _ = O.forward(p, shape, ts, z["tile_ranges"], z["pair_ids"])
    assert rel(vol, ovol) < FWD_TOL
    ograds = O.backward(p, shape, ts, z["tile_ranges"], z["pair_ids"], z["grad_vol"])
    for k, a, b in zip(GRAD_KEYS, grads, ograds):
        assert rel(a, b) < GRAD_TOL, k
    # and against the reference's own FP32 output away from the cutoff boundary
    bnd = O.boundary_voxels(*p[:3], shape, ts, z["tile_ranges"], z["pair_ids"], tol=1e-4)
    assert rel(vol[~bnd], z["vol"][~bnd]) < 1e-5


def test_deterministic_mode_is_bitwise_reproducible(cuda_device):
    shape, ts = (40, 40, 40), 8
    gs = synthetic.random_gaussians(6000, shape, seed=5)
    gv = synthetic.upstream_grad(shape, seed=6).numpy()
    p = tuple(t.numpy() for t in gs.tensors())
    _, g1 = gpu_run(p, shape, ts, gv, deterministic=True)
    _, g2 = gpu_run(p, shape, ts, gv, deterministic=True)
    for a, b in zip(g1, g2):
        assert np.array_equal(a.view(np.int32), b.view(np.int32))


def test_repeated_backward_after_one_preprocess(cuda_device):
    """The atomic backward's moment accumulators start from zero on every
    call: the preprocess clears them and k_finalize clears them after
    reading, so a second backward on the same binning gives the first's
    gradients (to atomic-order rounding), not their sum."""
    from gs_tmi_b200.tile_voxelizer import backward_into

    shape, ts = (48, 40, 56), 8
    gs = synthetic.random_gaussians(5000, shape, seed=21)
    params = tuple(t.to(cuda_device).contiguous() for t in gs.tensors())
    g = synthetic.upstream_grad(shape, seed=22).to(cuda_device)
    plan = prepare_and_bin(params, _shape(shape, ts))
    first = [torch.empty_like(t) for t in params]
    second = [torch.empty_like(t) for t in params]
    backward_into(plan, params, g, first)
    backward_into(plan, params, g, second)
    torch.cuda.synchronize()
    for k, a, b in zip(GRAD_KEYS, first, second):
        assert rel(b.cpu().numpy(), a.cpu().numpy()) < 1e-5, k


def test_64cube_n20000(cuda_device):
    """The 64^3 / N=20,000 micro-benchmark workload at full size."""
    shape, ts = (64, 64, 64), 8
    gs = synthetic.random_gaussians(20000, shape, seed=0)
    gv = synthetic.upstream_grad(shape, seed=1).numpy()
    p = tuple(t.numpy() for t in gs.tensors())
    z = load("cfg_64cube_n20000")
    plan = prepare_and_bin(tuple(t.to(cuda_device) for t in gs.tensors()), _shape(shape, ts))
    tr, pid = plan_lists(plan)
    assert plan.total == int(z["n_pairs"])
    assert np.array_equal(tr, z["tile_ranges"])
    ctr, cpid = O.build_tile_pairs(*O.preprocess_f32(*p[:3], shape)[:2], shape, ts)
    assert np.array_equal(pid, cpid)
    for det in (False, True):
        vol, grads = gpu_run(p, shape, ts, gv, deterministic=det)
        ovol, _ = O.forward(p, shape, ts, tr, pid)
        assert rel(vol, ovol) < FWD_TOL
        for k, a, b in zip(GRAD_KEYS, grads, O.backward(p, shape, ts, tr, pid, gv)):
            assert rel(a, b) < GRAD_TOL, k


@pytest.mark.parametrize("ts", [4, 5, 8, 16])
def test_tile_sizes_and_ragged_volume(ts, cuda_device):
    shape = (19, 13, 22)
    gs = synthetic.concat(synthetic.random_gaussians(300, shape, seed=70 + ts),
                          synthetic.edge_case_gaussians(shape, seed=71))
    gv = synthetic.upstream_grad(shape, seed=72).numpy()
    p = tuple(t.numpy() for t in gs.tensors())
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    tr, pid = O.build_tile_pairs(c, r, shape, ts)
    gtr, gpid = gs_tmi_b200.build_tile_pairs(torch.tensor(c, device=cuda_device),
                                             torch.tensor(r, device=cuda_device), shape, ts)
    assert np.array_equal(gtr.cpu().numpy(), tr) and np.array_equal(gpid.cpu().numpy(), pid)
    for det in (False, True):
        vol, grads = gpu_run(p, shape, ts, gv, deterministic=det)
        assert rel(vol, O.forward(p, shape, ts, tr, pid)[0]) < FWD_TOL
        for k, a, b in zip(GRAD_KEYS, grads, O.backward(p, shape, ts, tr, pid, gv)):
            assert rel(a, b) < GRAD_TOL, (k, det)


def test_empty_and_outside(cuda_device):
    shape, ts = (16, 16, 16), 8
    # no Gaussians at all
    empty = [np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), np.zeros((0, 4), np.float32),
             np.zeros(0, np.float32), np.zeros(0, np.float32)]
    vol, grads = gpu_run(empty, shape, ts, np.ones(shape, np.complex64))
    assert not vol.any() and all(g.size == 0 for g in grads)
    tr, pid = gs_tmi_b200.build_tile_pairs(torch.zeros(0, 3, device=cuda_device),
                                           torch.zeros(0, device=cuda_device), shape, ts)
    assert tr.shape == (8, 2) and not tr.any() and pid.numel() == 0
    # every Gaussian far outside: clamped into the border tiles, contributes ~0
    gs = synthetic.random_gaussians(50, shape, seed=9)
    gs.positions[:] = gs.positions.sign() * 3.0
    p = tuple(t.numpy() for t in gs.tensors())
    gv = synthetic.upstream_grad(shape, seed=10).numpy()
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    tr, pid = O.build_tile_pairs(c, r, shape, ts)
    vol, grads = gpu_run(p, shape, ts, gv)
    ovol, _ = O.forward(p, shape, ts, tr, pid)
    assert np.abs(vol - ovol).max() < 1e-6


def _nan_close(a, b, tol):
    """Same NaN positions, finite parts within `tol` (relative L2)."""
    a, b = np.asarray(a), np.asarray(b)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    f = ~np.isnan(b)
    return rel(a[f], b[f]) < tol if f.any() else True


@pytest.mark.parametrize("deterministic", [False, True])
def test_nan_parameters(deterministic, cuda_device):
    """NaN in a position, a scale, a quaternion or a density (the reference's
    GPU path semantics: float -> int conversion maps NaN to 0 in the tile
    boxes, and "m <= 9" is false for NaN m): binning stays bit-exact, a
    NaN-geometry Gaussian contributes nothing, a NaN density poisons exactly
    the voxels it covers, and NaN stays inside the gradients of the NaN
    Gaussians."""
    shape, ts = (24, 20, 16), 8
    gs = synthetic.random_gaussians(400, shape, seed=41)
    gs.positions[0] = float("nan")
    gs.scales[1, 0] = float("nan")
    gs.rotations[2] = float("nan")
    gs.density_r[3] = float("nan")
    p = tuple(t.numpy() for t in gs.tensors())
    gv = synthetic.upstream_grad(shape, seed=42).numpy()
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    tr, pid = O.build_tile_pairs(c, r, shape, ts)
    plan = prepare_and_bin(tuple(torch.tensor(x, device=cuda_device) for x in p), _shape(shape, ts))
    gtr, gpid = plan_lists(plan)
    assert np.array_equal(gtr, tr) and np.array_equal(gpid, pid)
    vol, grads = gpu_run(p, shape, ts, gv, deterministic=deterministic)
    ovol, _ = O.forward(p, shape, ts, tr, pid)
    assert _nan_close(vol, ovol, FWD_TOL) and np.isnan(vol).any()
    og = O.backward(p, shape, ts, tr, pid, gv)
    for a, b in zip(grads, og):
        assert _nan_close(a, b, GRAD_TOL)
        bad = np.isnan(a).reshape(a.shape[0], -1).any(1)
        assert not bad[4:].any()  # only the NaN Gaussians


def test_negative_radius_is_rejected(cuda_device):
    """Only negative scales can make a tile box empty; the reference fails in
    repeat_interleave on such input, this build raises ValueError."""
    shape = (32, 32, 32)
    gs = synthetic.random_gaussians(4, shape, seed=1)
    gs.positions[1] = 0.0
    gs.scales[1] = -0.5
    with pytest.raises(ValueError):
        gs_tmi_b200.voxelize(*(t.to(cuda_device) for t in gs.tensors()), shape, 4)


def _cov_inv_f32(scales, rotations):
    q = rotations / (rotations.norm(dim=-1, keepdim=True) + 1e-8)
    w, x, y, z = q.unbind(-1)
    R = torch.stack([
        torch.stack([1 - 2 * y * y - 2 * z * z, 2 * x * y - 2 * z * w, 2 * x * z + 2 * y * w], -1),
        torch.stack([2 * x * y + 2 * z * w, 1 - 2 * x * x - 2 * z * z, 2 * y * z - 2 * x * w], -1),
        torch.stack([2 * x * z - 2 * y * w, 2 * y * z + 2 * x * w, 1 - 2 * x * x - 2 * y * y], -1),
    ], -2)
    T = R * torch.reciprocal(scales + 1e-8).unsqueeze(1)
    return T @ T.transpose(1, 2)


@pytest.mark.parametrize("name", ["edge_20x12x16_ts8", "cube_16_ts4", "odd_13x11x9_ts5"])
def test_reference_signature_kernels(name, cuda_device):
    """_TileVoxelizeCUDA / gsv_tile_forward / gsv_tile_backward with the
    reference extension's arguments, against the oracle's compat mode."""
    z = load(name)
    shape, ts = tuple(int(x) for x in z["shape"]), int(z["tile_size"])
    d, h, w = shape
    M = _cov_inv_f32(torch.tensor(z["scales"]), torch.tensor(z["rotations"])).numpy().reshape(-1, 9)
    hs = np.array([d * 0.5, h * 0.5, w * 0.5], np.float32)
    c = z["center"]
    dev = cuda_device
    tc = torch.tensor(c, device=dev, requires_grad=True)
    tm = torch.tensor(M.reshape(-1, 3, 3), device=dev, requires_grad=True)
    tdr = torch.tensor(z["density_r"], device=dev, requires_grad=True)
    tdi = torch.tensor(z["density_i"], device=dev, requires_grad=True)
    tr = torch.tensor(z["tile_ranges"], device=dev)
    pid = torch.tensor(z["pair_ids"], device=dev)
    vr, vi = gs_tmi_b200._TileVoxelizeCUDA.apply(tc, tm, tdr, tdi, tr, pid, torch.tensor(hs, device=dev), ts,
                                                 d, h, w)
    gv = z["grad_vol"].reshape(-1)
    loss = (vr * torch.tensor(gv.real, device=dev)).sum() + (vi * torch.tensor(gv.imag, device=dev)).sum()
    loss.backward()
    cp = (c, M, None, z["density_r"], z["density_i"])
    ovol, _ = O.forward(cp, shape, ts, z["tile_ranges"], z["pair_ids"], compat=True, half_shape=hs)
    vol = (vr + 1j * vi).detach().cpu().numpy().reshape(shape)
    assert rel(vol, ovol) < FWD_TOL
    og = O.backward(cp, shape, ts, z["tile_ranges"], z["pair_ids"], z["grad_vol"], compat=True, half_shape=hs)
    for name_, a, b in (("center", tc.grad, og[0]), ("cov", tm.grad, og[1]), ("dr", tdr.grad, og[3]),
                        ("di", tdi.grad, og[4])):
        assert rel(a.cpu().numpy(), b) < GRAD_TOL, name_


def test_module_autograd_like_the_trainer(cuda_device):
    """TileVoxelizer as GaussianTrainer._get_volume calls it: scales =
    exp(log-scale parameter), density = complex(re, im) parameters
    (trainers/trainer.py:223-229, gaussian_model.py:63-68)."""
    shape, ts = (24, 20, 16), 8
    gs = synthetic.random_gaussians(400, shape, seed=77)
    dev = cuda_device
    pos = torch.nn.Parameter(gs.positions.to(dev))
    log_s = torch.nn.Parameter(torch.log(gs.scales).to(dev))
    rot = torch.nn.Parameter(gs.rotations.to(dev))
    dr = torch.nn.Parameter(gs.density_r.to(dev))
    di = torch.nn.Parameter(gs.density_i.to(dev))
    vox = gs_tmi_b200.TileVoxelizer(shape, tile_size=ts, device=str(dev))
    assert vox.backend == "tile_cuda"
    vol = vox(positions=pos, scales=torch.exp(log_s), rotations=rot, density=torch.complex(dr, di))
    assert vol.dtype == torch.complex64 and tuple(vol.shape) == shape
    g = synthetic.upstream_grad(shape, seed=78).to(dev)
    (vol.real * g.real + vol.imag * g.imag).sum().backward()
    p = tuple(t.numpy() for t in gs.tensors())
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    tr, pid = O.build_tile_pairs(c, r, shape, ts)
    og = O.backward(p, shape, ts, tr, pid, g.cpu().numpy())
    assert rel(pos.grad.cpu().numpy(), og[0]) < GRAD_TOL
    assert rel(log_s.grad.cpu().numpy(), og[1] * gs.scales.numpy()) < GRAD_TOL
    assert rel(rot.grad.cpu().numpy(), og[2]) < GRAD_TOL
    assert rel(dr.grad.cpu().numpy(), og[3]) < GRAD_TOL
    assert rel(di.grad.cpu().numpy(), og[4]) < GRAD_TOL
