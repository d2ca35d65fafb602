"""The reference's own trainer driving either voxelizer (helper of
tests/test_gpu_reference_trainer.py).

The reference's Python package (V = 3DGS/3dgsVC: trainers/trainer.py,
data/dataset.py, gaussian/, losses/, metrics/, configs/) is staged
unchanged into the git-ignored baseline/_ref/3dgsVC by
oracle/build_ref.py.  Two things it imports are not installed here and are
stood in for before it is imported:

* ``skimage.metrics.structural_similarity`` (V/metrics/metrics.py:10):
  restated from the published SSIM definition (Wang et al. 2004) with the
  defaults V/metrics/metrics.py:43-67 relies on -- uniform window of
  ``win_size`` voxels per axis, K1 = 0.01, K2 = 0.03, sample covariance,
  the mean over the voxels whose window lies inside the volume;
* nothing else: torch.utils.tensorboard, tqdm, yaml and scipy.io import.

The voxelizer is chosen the way a user of this library switches:
``gaussian.TileVoxelizer`` rebound to ``gs_tmi_b200.TileVoxelizer`` (the
one-line change in V/gaussian/__init__.py), or the reference's own
TileVoxelizer on its CUDA extension (compiled from its sources into
oracle/_ref/, handed to V/gaussian/tile_voxelizer.py's extension cache
instead of its JIT build).  The seeded synthetic acquisition is written as
the k-space / coil-map / mask .mat files V/data/dataset.py reads, and the
trainer runs its own ``train()`` loop (V/trainers/trainer.py:527-604)."""
from __future__ import annotations

import copy
import os
import random
import sys
import types

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STAGED = os.path.join(ROOT, "baseline", "_ref", "3dgsVC")


def structural_similarity(im1, im2, *, data_range=None, win_size=7, channel_axis=None, **_):
    """Mean SSIM of two real arrays (Wang et al. 2004), uniform window."""
    from scipy.ndimage import uniform_filter

    x = np.asarray(im1, np.float64)
    y = np.asarray(im2, np.float64)
    if data_range is None:
        data_range = float(y.max() - y.min())
    npix = win_size ** x.ndim
    cov = npix / (npix - 1.0)
    ux, uy = uniform_filter(x, win_size), uniform_filter(y, win_size)
    vx = cov * (uniform_filter(x * x, win_size) - ux * ux)
    vy = cov * (uniform_filter(y * y, win_size) - uy * uy)
    vxy = cov * (uniform_filter(x * y, win_size) - ux * uy)
    c1, c2 = (0.01 * data_range) ** 2, (0.03 * data_range) ** 2
    s = ((2 * ux * uy + c1) * (2 * vxy + c2)) / ((ux * ux + uy * uy + c1) * (vx + vy + c2))
    pad = (win_size - 1) // 2
    return float(s[tuple(slice(pad, n - pad) for n in s.shape)].mean())


def available() -> bool:
    return os.path.isdir(os.path.join(STAGED, "trainers"))


def _import_reference():
    if "skimage.metrics" not in sys.modules:
        sk = types.ModuleType("skimage")
        skm = types.ModuleType("skimage.metrics")
        skm.structural_similarity = structural_similarity
        sk.metrics = skm
        sys.modules["skimage"], sys.modules["skimage.metrics"] = sk, skm
    if STAGED not in sys.path:
        sys.path.insert(0, STAGED)
    import gaussian  # noqa: F401  (the reference's package)
    import gaussian.tile_voxelizer as ref_tv
    import trainers.trainer as ref_trainer
    import yaml

    with open(os.path.join(STAGED, "configs", "default.yaml")) as f:
        default = yaml.safe_load(f)
    return ref_tv, ref_trainer, default


def write_case(case, path):
    """The acquisition as V/data/dataset.py reads it: fully sampled
    multi-coil k-space (coils first; the loader masks it), the coil maps and
    the sampling mask (the reference adds no noise; the case's complex noise
    is already in its samples)."""
    from scipy.io import savemat

    from gs_tmi_b200.synthetic import fft3c

    os.makedirs(path, exist_ok=True)
    k_full = fft3c(case.sensitivity_maps.cpu() * case.ground_truth.cpu().unsqueeze(0))
    # the case's noisy samples where the mask samples, the clean spectrum elsewhere: after the
    # loader applies the mask the trainer sees exactly the case's undersampled k-space
    m = case.mask.cpu().unsqueeze(0)
    k_full = (k_full * (1 - m) + case.kspace_undersampled.cpu()).to(torch.complex64)
    files = {"kspace": os.path.join(path, "kspace.mat"), "csm": os.path.join(path, "csm.mat"),
             "mask": os.path.join(path, "mask.mat")}
    savemat(files["kspace"], {"kspace": k_full.numpy().astype(np.complex64)})
    savemat(files["csm"], {"csm": case.sensitivity_maps.cpu().numpy().astype(np.complex64)})
    savemat(files["mask"], {"mask": case.mask.cpu().numpy().astype(np.float32)})
    return files


def _seed(seed):
    random.seed(seed)
    np.random.seed(seed)
    torch.manual_seed(seed)
    torch.cuda.manual_seed_all(seed)


def run(voxelizer: str, files: dict, out_dir: str, *, accel: float, iterations: int, eval_every: int,
        num_points: int, seed: int = 42, device="cuda:0") -> dict:
    """One run of the reference's GaussianTrainer.train() with
    ``voxelizer`` = "this_build", "reference_cuda" or "reference_cpu" (the
    reference's PyTorch path, for checking the harness on a CPU).  Returns the total
    loss of every iteration, the metrics of every evaluation and the wall
    time of train()."""
    import time

    ref_tv, ref_trainer, default = _import_reference()
    if voxelizer == "this_build":
        import gs_tmi_b200

        vox_cls = gs_tmi_b200.TileVoxelizer
    elif voxelizer == "reference_cpu":  # the reference's PyTorch tile path (harness check without a GPU)
        vox_cls = ref_tv.TileVoxelizer
    elif voxelizer == "reference_cuda":
        from oracle.ref_cuda import REF

        if REF is None:
            raise RuntimeError("reference extension not built (oracle/build_ref.py)")
        ref_tv._cuda_ext = REF  # the extension the reference would JIT-build from the same sources
        vox_cls = ref_tv.TileVoxelizer
    else:
        raise ValueError(voxelizer)
    ref_trainer.TileVoxelizer = vox_cls  # what `from gaussian import TileVoxelizer` binds

    cfg = copy.deepcopy(default)
    cfg["data"].update(data_path=files["kspace"], csm_path=files["csm"], mask_path=files["mask"],
                       acceleration_factor=accel, readout_axis=0, phase_axes=[1, 2], acs_lines=24)
    cfg["gaussian"].update(initial_num_points=num_points)
    cfg["training"].update(max_iterations=iterations, eval_every=eval_every, log_every=10 ** 9,
                           save_every=10 ** 9, seed=seed)
    cfg["stopping"]["enable_metric_plateau"] = False
    cfg["output"].update(output_dir=out_dir, use_tensorboard=False, save_nii=False, save_npy=False)
    cfg["voxelizer"]["type"] = "tile" if voxelizer == "reference_cpu" else "tile_cuda"
    if voxelizer == "reference_cpu":
        cfg["mode"]["strict_cuda"] = False
    _seed(seed)
    trainer = ref_trainer.GaussianTrainer(cfg, device=torch.device(device))
    assert isinstance(trainer.voxelizer, vox_cls)
    losses, evals = [], []
    step, evaluate = trainer.train_step, trainer.evaluate

    def train_step():
        d = step()
        losses.append(d["total_loss"])
        return d

    def evaluate_():
        m = evaluate()
        evals.append(dict(m, iteration=trainer.current_iteration))
        return m

    trainer.train_step, trainer.evaluate = train_step, evaluate_
    sync = torch.cuda.synchronize if torch.device(device).type == "cuda" else (lambda: None)
    sync()
    t0 = time.perf_counter()
    best = trainer.train()
    sync()
    return {"voxelizer": voxelizer, "backend": getattr(trainer.voxelizer, "backend", None), "losses": losses,
            "evals": evals, "best": best, "seconds": time.perf_counter() - t0,
            "n_points": int(trainer.gaussian_model.num_points)}
