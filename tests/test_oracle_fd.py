"""FP64 central finite differences against the oracle's analytic backward.

The FP32 parameters fix the inclusion set, the FP64 copy is perturbed, so
the loss L = sum Re(conj(g) vol) is smooth and the difference converges at
O(h^2).  This checks the chain rule through cov_inv -> (scale, quaternion)
and center -> position that the CUDA finalize kernel implements."""
import numpy as np
import pytest

from oracle import oracle as O
from gs_tmi_b200 import synthetic


def _case(seed, shape=(12, 10, 14), ts=4, n=6):
    gs = synthetic.random_gaussians(n, shape, seed=seed, log_scale_mean_vox=np.log(2.0))
    rng = np.random.default_rng(seed)
    gs.rotations[:] = gs.rotations * 1.7  # unnormalised quaternions
    p = tuple(t.numpy().copy() for t in gs.tensors())
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    tr, pid = O.build_tile_pairs(c, r, shape, ts)
    g = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)
    return p, shape, ts, tr, pid, g


@pytest.mark.parametrize("seed", [0, 1])
def test_params_mode_fd(seed):
    p, shape, ts, tr, pid, g = _case(seed)
    grads = O.backward(p, shape, ts, tr, pid, g)
    names = ("a", "b", "c", "dr", "di")
    rng = np.random.default_rng(100 + seed)
    for which, an in zip(names, grads):
        flat = an.reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            base = float(np.asarray(p[names.index(which)], np.float64).reshape(-1)[idx])
            h = 1e-6 * max(1.0, abs(base))
            fd = O.fd_gradient(p, shape, ts, tr, pid, g, which, int(idx), h=h)
            assert abs(fd - flat[idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7, (which, idx, fd, flat[idx])


def test_compat_mode_fd():
    """Gradients w.r.t. (center_vox, cov_inv, density) of the reference
    extension's parameterisation (tile_voxelize_cuda_kernel.cu:233-252)."""
    p, shape, ts, tr, pid, g = _case(7)
    c, _, _ = O.preprocess_f32(*p[:3], shape)
    # FP64 cov_inv from the same parameters, rounded to FP32 like the reference
    import torch

    q = torch.tensor(p[2], dtype=torch.float64)
    q = q / (q.norm(dim=-1, keepdim=True) + 1e-8)
    w, x, y, z = q.unbind(-1)
    R = torch.stack([
        torch.stack([1 - 2 * y * y - 2 * z * z, 2 * x * y - 2 * z * w, 2 * x * z + 2 * y * w], -1),
        torch.stack([2 * x * y + 2 * z * w, 1 - 2 * x * x - 2 * z * z, 2 * y * z - 2 * x * w], -1),
        torch.stack([2 * x * z - 2 * y * w, 2 * y * z + 2 * x * w, 1 - 2 * x * x - 2 * y * y], -1),
    ], -2)
    T = R / (torch.tensor(p[1], dtype=torch.float64) + 1e-8).unsqueeze(1)
    M = (T @ T.transpose(1, 2)).float().numpy().reshape(-1, 9)
    hs = np.array([s * 0.5 for s in shape], np.float32)
    cp = (c, M, None, p[3], p[4])
    gc, gm, _, gdr, gdi = O.backward(cp, shape, ts, tr, pid, g, compat=True, half_shape=hs)
    rng = np.random.default_rng(5)
    for which, an in (("a", gc), ("b", gm), ("dr", gdr), ("di", gdi)):
        flat = an.reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            arr = {"a": c, "b": M, "dr": p[3], "di": p[4]}[which]
            base = float(np.asarray(arr, np.float64).reshape(-1)[idx])
            h = 1e-6 * max(1.0, abs(base))
            fd = O.fd_gradient(cp, shape, ts, tr, pid, g, which, int(idx), h=h, compat=True, half_shape=hs)
            assert abs(fd - flat[idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7, (which, idx, fd, flat[idx])
