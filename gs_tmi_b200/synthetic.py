"""Seeded synthetic inputs for the voxelizer workloads.

The reference ships no datasets (its clinical ``.mat`` k-space files are not
public), so every workload here is a seeded synthetic stand-in with the
shapes, sizes and value distributions of the stated configuration.
All draws use a CPU ``torch.Generator`` so inputs are identical on every
machine; callers move them to the device themselves.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch


@dataclass
class GaussianSet:
    positions: torch.Tensor   # [N,3] normalised to [-1,1], axis order (d,h,w)
    scales: torch.Tensor      # [N,3] fraction of the half extent (exp of the log-scale param)
    rotations: torch.Tensor   # [N,4] (w,x,y,z) quaternion, unnormalised
    density_r: torch.Tensor   # [N]
    density_i: torch.Tensor   # [N]

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])

    def to(self, device) -> "GaussianSet":
        return GaussianSet(*(t.to(device) for t in self.tensors()))

    def tensors(self):
        return (self.positions, self.scales, self.rotations, self.density_r, self.density_i)

    @property
    def density(self) -> torch.Tensor:
        return torch.complex(self.density_r, self.density_i)


def random_gaussians(n: int, shape, seed: int = 0, log_scale_mean_vox: float = math.log(1.5),
                     log_scale_std: float = 0.3, density_std: float = 0.1) -> GaussianSet:
    """Uniform means in the volume, per-axis log-normal scales in voxels,
    uniformly random unit quaternions and N(0, std) complex density.

    This is the 64^3 / N=20,000 voxelizer micro-benchmark distribution
    (means uniform, log-scale ~ N(ln 1.5 voxels, 0.3), density ~ N(0, 0.1))."""
    g = torch.Generator().manual_seed(seed)
    half = torch.tensor([s * 0.5 for s in shape], dtype=torch.float32)
    positions = torch.rand(n, 3, generator=g) * 2 - 1
    log_vox = torch.randn(n, 3, generator=g) * log_scale_std + log_scale_mean_vox
    scales = torch.exp(log_vox) / half
    quat = torch.randn(n, 4, generator=g)
    quat = quat / quat.norm(dim=-1, keepdim=True).clamp_min(1e-12)
    dr = torch.randn(n, generator=g) * density_std
    di = torch.randn(n, generator=g) * density_std
    return GaussianSet(positions.float(), scales.float(), quat.float(), dr.float(), di.float())


def upstream_grad(shape, seed: int = 1) -> torch.Tensor:
    """Complex standard-normal upstream volume gradient, complex64 [d,h,w]."""
    g = torch.Generator().manual_seed(seed)
    re = torch.randn(*shape, generator=g)
    im = torch.randn(*shape, generator=g)
    return torch.complex(re, im) / math.sqrt(2.0)


def edge_case_gaussians(shape, seed: int = 3) -> GaussianSet:
    """A handful of Gaussians that exercise the binning edges: outside the
    volume, on a face, huge, tiny, strongly anisotropic, unnormalised and
    zero quaternions."""
    g = torch.Generator().manual_seed(seed)
    half = torch.tensor([s * 0.5 for s in shape], dtype=torch.float32)
    pos = torch.tensor([
        [0.0, 0.0, 0.0],       # centre
        [1.3, 0.2, -0.1],      # outside along d
        [-1.0, -1.0, -1.0],    # corner
        [0.999, 0.5, 0.999],   # near the far faces
        [0.1, -0.2, 0.3],      # huge
        [0.2, 0.2, 0.2],       # tiny
        [-0.4, 0.3, 0.1],      # needle
        [0.5, -0.5, 0.0],      # pancake
        [0.05, 0.6, -0.7],     # unnormalised quaternion
        [-0.3, -0.6, 0.45],    # zero quaternion
    ], dtype=torch.float32)
    vox = torch.tensor([
        [2.0, 2.0, 2.0],
        [3.0, 2.0, 2.5],
        [2.5, 2.5, 2.5],
        [1.5, 3.0, 1.0],
        [40.0, 35.0, 50.0],
        [0.05, 0.08, 0.04],
        [8.0, 0.4, 0.4],
        [5.0, 5.0, 0.3],
        [2.0, 1.0, 3.0],
        [1.5, 1.5, 1.5],
    ], dtype=torch.float32)
    scales = vox / half
    rot = torch.randn(pos.shape[0], 4, generator=g)
    rot[8] = rot[8] * 7.5
    rot[9] = 0.0
    dr = torch.randn(pos.shape[0], generator=g) * 0.1
    di = torch.randn(pos.shape[0], generator=g) * 0.1
    return GaussianSet(pos, scales, rot, dr, di)


def concat(*sets: GaussianSet) -> GaussianSet:
    return GaussianSet(*(torch.cat(ts, 0) for ts in zip(*(s.tensors() for s in sets))))


# ---------------------------------------------------------------------------
# Synthetic MRI case: phantom, coils, sampling mask, k-space, zero-filled.
# Stand-ins for the reference's private clinical .mat data.
# ---------------------------------------------------------------------------

def fft3c(x: torch.Tensor) -> torch.Tensor:
    """Centred orthonormal 3-D FFT over the last three axes."""
    dims = (-3, -2, -1)
    return torch.fft.fftshift(torch.fft.fftn(torch.fft.ifftshift(x, dim=dims), dim=dims, norm="ortho"), dim=dims)


def ifft3c(k: torch.Tensor) -> torch.Tensor:
    dims = (-3, -2, -1)
    return torch.fft.fftshift(torch.fft.ifftn(torch.fft.ifftshift(k, dim=dims), dim=dims, norm="ortho"), dim=dims)


def _grid(shape):
    axes = [torch.linspace(-1.0, 1.0, s) for s in shape]
    return torch.meshgrid(*axes, indexing="ij")


def ellipsoid_phantom(shape, n_ellipsoids: int = 10, seed: int = 0) -> torch.Tensor:
    """Sum of random rotated ellipsoids times a smooth low-order polynomial
    phase; complex64 (D,H,W), magnitude roughly in [0, 1]."""
    g = torch.Generator().manual_seed(seed)
    zz, yy, xx = _grid(shape)
    pts = torch.stack([zz, yy, xx], -1)
    mag = torch.zeros(shape)
    for _ in range(n_ellipsoids):
        c = (torch.rand(3, generator=g) - 0.5) * 0.9
        ax = 0.12 + torch.rand(3, generator=g) * 0.33
        q = torch.randn(4, generator=g)
        q = q / q.norm()
        w, x, y, z = q
        R = torch.tensor([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                          [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                          [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        local = (pts - c) @ R
        inside = ((local / ax) ** 2).sum(-1) <= 1.0
        mag = mag + inside.float() * (0.2 + 0.8 * torch.rand((), generator=g))
    mag = mag / mag.max().clamp_min(1e-6)
    coef = torch.randn(10, generator=g) * 0.6
    phase = (coef[0] + coef[1] * zz + coef[2] * yy + coef[3] * xx + coef[4] * zz * zz + coef[5] * yy * yy
             + coef[6] * xx * xx + coef[7] * zz * yy + coef[8] * yy * xx + coef[9] * zz * xx)
    return torch.polar(mag, phase).to(torch.complex64)


def ring_coils(shape, n_coils: int = 8, seed: int = 0) -> torch.Tensor:
    """Gaussian-profile coil sensitivities on a ring around the (h,w) plane
    with a per-coil smooth phase, normalised to unit sum-of-squares."""
    g = torch.Generator().manual_seed(seed)
    zz, yy, xx = _grid(shape)
    maps = []
    for k in range(n_coils):
        a = 2 * math.pi * k / n_coils
        cy, cx = 1.3 * math.cos(a), 1.3 * math.sin(a)
        prof = torch.exp(-((yy - cy) ** 2 + (xx - cx) ** 2 + 0.5 * zz ** 2) / (2 * 0.9 ** 2))
        ph = float(torch.rand((), generator=g)) * 2 * math.pi + 0.5 * (yy * math.sin(a) - xx * math.cos(a))
        maps.append(torch.polar(prof, ph))
    S = torch.stack(maps, 0)
    sos = torch.sqrt((S.abs() ** 2).sum(0, keepdim=True)).clamp_min(1e-8)
    return (S / sos).to(torch.complex64)


def variable_density_mask(shape, accel: float, calib: int = 24, seed: int = 0) -> torch.Tensor:
    """Readout (axis 0) fully sampled; (ky,kz) variable-density Poisson-disc
    style pattern: candidate points drawn with a polynomial density and
    thinned by a density-scaled minimum distance, plus a fully sampled
    calib x calib centre.  Returns float32 (D,H,W) of 0/1 at about 1/accel."""
    _, ny, nz = shape
    rng = torch.Generator().manual_seed(seed)
    y = torch.linspace(-1, 1, ny)
    z = torch.linspace(-1, 1, nz)
    yy, zz = torch.meshgrid(y, z, indexing="ij")
    r = torch.sqrt(yy ** 2 + zz ** 2)
    pdf = (1 - r / r.max()).clamp_min(0) ** 2 + 0.02
    target = int(ny * nz / accel)
    mask = torch.zeros(ny, nz, dtype=torch.bool)
    cy, cz, h = ny // 2, nz // 2, calib // 2
    mask[max(cy - h, 0):cy + h, max(cz - h, 0):cz + h] = True
    order = torch.multinomial(pdf.reshape(-1), ny * nz, replacement=False, generator=rng)
    # minimum spacing (in samples) grows where the density is low
    base = 0.5 * math.sqrt(accel)
    taken = mask.clone()
    count = int(mask.sum())
    for idx in order.tolist():
        if count >= target:
            break
        iy, iz = divmod(idx, nz)
        if taken[iy, iz]:
            continue
        rad = base * float(pdf.max() / pdf[iy, iz]) ** 0.5 * 0.5
        ri = int(math.floor(rad))
        if ri >= 1:
            y0, y1 = max(iy - ri, 0), min(iy + ri + 1, ny)
            z0, z1 = max(iz - ri, 0), min(iz + ri + 1, nz)
            if mask[y0:y1, z0:z1].any():
                continue
        mask[iy, iz] = True
        taken[iy, iz] = True
        count += 1
    return mask.float().unsqueeze(0).expand(shape[0], ny, nz).contiguous()


@dataclass
class MRICase:
    ground_truth: torch.Tensor      # complex64 (D,H,W)
    sensitivity_maps: torch.Tensor  # complex64 (C,D,H,W)
    mask: torch.Tensor              # float32 (D,H,W)
    kspace_undersampled: torch.Tensor  # complex64 (C,D,H,W)
    zero_filled: torch.Tensor       # complex64 (D,H,W), coil-combined


def mri_case(shape, n_coils: int = 8, accel: float = 6.0, calib: int = 24, noise_rel: float = 1e-3,
             seed: int = 0, device=None, mask_kind: str = "vd") -> MRICase:
    """Synthetic multi-coil acquisition: phantom x coils -> fft3c -> mask +
    complex noise sigma = noise_rel * max|k| -> SENSE-combined zero-filled.
    `device`: where the FFTs and the noise are computed (and the case lives);
    the default, the CPU, is the reference generator of all seeded cases.
    `mask_kind`: "vd" (variable_density_mask, any device) or "poisson" (the
    reference's own Poisson-disc generator, mask_generator.py:241-400, on
    the GPU through gs_tmi_b200.masks; visiting order drawn with seed + 3)."""
    dev = torch.device(device) if device is not None else torch.device("cpu")
    x = ellipsoid_phantom(shape, seed=seed).to(dev)
    S = ring_coils(shape, n_coils, seed=seed + 1).to(dev)
    k = fft3c(S * x.unsqueeze(0))
    g = torch.Generator(device=dev).manual_seed(seed + 2)
    sigma = noise_rel * float(k.abs().max())
    noise = torch.complex(torch.randn(k.shape, generator=g, device=dev),
                          torch.randn(k.shape, generator=g, device=dev)) * sigma
    if mask_kind == "poisson":
        from . import masks

        plane = masks.poisson_masks(tuple(shape[1:]), accel, calib, seeds=[seed + 3],
                                    device=dev if dev.type == "cuda" else "cuda")[0]
        m = masks.expand_phase_mask(plane.float().to(dev), tuple(shape), (1, 2))
    elif mask_kind == "vd":
        m = variable_density_mask(shape, accel, calib, seed=seed + 3).to(dev)
    else:
        raise ValueError(f"unknown mask kind {mask_kind!r}")
    ku = (k + noise) * m.unsqueeze(0)
    zf = (torch.conj(S) * ifft3c(ku)).sum(0)
    return MRICase(x, S, m, ku.to(torch.complex64), zf.to(torch.complex64))


def seed_indices(image: torch.Tensor, num_points: int, seed: int, mode: str = "random",
                 device=None) -> torch.Tensor:
    """Seed voxels (flat indices, CPU) of the intensity-seeded init, as
    GaussianModel3D.from_image draws them (gaussian_model.py:320-335):
    "random" -- a random permutation of all voxels; "importance" -- a random
    permutation of the voxels whose magnitude exceeds the 90th percentile
    (all voxels when there are fewer of those than seeds).  The permutation
    always comes from a CPU generator seeded with `seed`; `device` (CUDA)
    only moves the percentile and the candidate search there, which gives
    the same candidates (a sort-based quantile either way) in a fraction of
    the CPU's time."""
    total = image.numel()
    g = torch.Generator().manual_seed(seed)
    n = min(num_points, total)
    if mode == "random" or num_points >= total:
        return torch.randperm(total, generator=g)[:n]
    if mode != "importance":
        raise ValueError(f"unknown seeding mode {mode!r}")
    dev = torch.device(device) if device is not None else torch.device("cpu")
    mag = image.detach().to(dev).abs().reshape(-1).float()
    thr = torch.quantile(mag, 0.90)
    cand = torch.nonzero(mag > thr, as_tuple=False).squeeze(-1).cpu()
    if cand.numel() < n:
        cand = torch.arange(total)
    return cand[torch.randperm(cand.numel(), generator=g)[:n]]


def from_image_init(image: torch.Tensor, num_points: int, density_scale_k: float = 0.2,
                    seed: int = 0, device=None, mode: str = "random") -> GaussianSet:
    """Intensity-seeded initialisation in the manner of the reference's
    GaussianModel3D.from_image (gaussian_model.py:308-355, random mode):
    random voxel centres, isotropic scale = mean distance to the 3 nearest
    other centres (normalised units), identity rotation, density =
    k * zero-filled value at the centre.

    `device` (a CUDA device): the 3-NN distances come from the library's
    exact grid search (gsv_knn3_mean_distance) instead of scipy's cKDTree and
    the set is returned on that device; the seed voxels are the same.
    `mode`: the seed draw, "random" (the reference's paper profile) or
    "importance" (its other mode), see `seed_indices`."""
    d, h, w = image.shape
    if device is not None and torch.device(device).type == "cuda":
        return _from_image_init_gpu(image, num_points, density_scale_k, seed, torch.device(device), mode)
    from scipy.spatial import cKDTree

    idx = seed_indices(image, num_points, seed, mode)
    n = idx.numel()
    z = idx // (h * w)
    rem = idx % (h * w)
    y = rem // w
    x = rem % w
    pos = torch.stack([((z.float() + 0.5) / d) * 2 - 1, ((y.float() + 0.5) / h) * 2 - 1,
                       ((x.float() + 0.5) / w) * 2 - 1], -1)
    pts = pos.numpy().astype("float32")
    k = min(4, n)
    if n > 1:
        dist, _ = cKDTree(pts).query(pts, k=k, workers=-1)
        nd = torch.from_numpy(dist[:, 1:].astype("float32"))
        if nd.ndim == 1:
            nd = nd[:, None]
        if nd.shape[1] < 3:  # fewer than 3 other seeds: the last distance repeats (:297-299)
            nd = torch.cat([nd, nd[:, -1:].repeat(1, 3 - nd.shape[1])], 1)
        mean = nd[:, :3].mean(1, keepdim=True).clamp_min(1e-6)
    else:
        mean = torch.full((n, 1), 1e-3)
    scales = mean.repeat(1, 3)
    rot = torch.zeros(n, 4)
    rot[:, 0] = 1.0
    flat = image.reshape(-1)[idx]
    return GaussianSet(pos.float(), scales.float(), rot, (flat.real * density_scale_k).float(),
                       (flat.imag * density_scale_k).float())


def _from_image_init_gpu(image, num_points, density_scale_k, seed, dev, mode="random") -> GaussianSet:
    import ctypes

    from ._lib import check, lib

    d, h, w = image.shape
    total = d * h * w
    idx_cpu = seed_indices(image, num_points, seed, mode, device=dev)
    n = idx_cpu.numel()
    z = idx_cpu // (h * w)
    rem = idx_cpu % (h * w)
    y = rem // w
    x = rem % w
    # positions exactly as the CPU path rounds them
    pos = torch.stack([((z.float() + 0.5) / d) * 2 - 1, ((y.float() + 0.5) / h) * 2 - 1,
                       ((x.float() + 0.5) / w) * 2 - 1], -1).to(dev).contiguous()
    idx = idx_cpu.to(dev)
    mean = torch.empty(n, dtype=torch.float32, device=dev)
    grid = torch.empty(total, dtype=torch.int32, device=dev)
    check(lib.gsv_knn3_mean_distance(ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(pos.data_ptr()), n, d, h, w,
                                     ctypes.c_void_p(grid.data_ptr()),
                                     ctypes.c_void_p(mean.data_ptr()),
                                     ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
          "gsv_knn3_mean_distance")
    scales = mean[:, None].repeat(1, 3)
    rot = torch.zeros(n, 4, device=dev)
    rot[:, 0] = 1.0
    flat = image.to(dev).reshape(-1)[idx]
    return GaussianSet(pos.float().contiguous(), scales.contiguous(), rot, (flat.real * density_scale_k).float(),
                       (flat.imag * density_scale_k).float())
