"""Learned warm start for the plain 3DGSMR fit.

A small MLP maps the zero-filled image around a seed voxel (a 5^3 complex
patch = 250 values, plus the sampling density of the acquisition and the
seed's intensity-seeded scale; padded to 256) to the initial parameters of
the Gaussian at that seed: centre offset (3), log-scale (3), quaternion (4)
and complex density (2); padded to 16 outputs.

Network 256 -> 256 (GELU, tanh form) -> 256 (GELU) -> 16 with BF16 weights and FP32
accumulation.  Every matrix product of inference and training -- X W^T with
the bias + GELU epilogue, dY W with the GELU' epilogue, and the split-K
weight gradients dZ^T X -- runs on the hand-written tcgen05 kernel
(``gsv_mlp_gemm``); FP32 master weights take Adam steps and are rounded to
BF16 for the next step.

Training data come from plain fits the method itself produces on synthetic
phantoms (``training_case``): the target is the volume the plain fit
reconstructs.  A training step renders the MLP's Gaussians with this
package's voxelizer and back-propagates the relative L2 distance to that
volume through the voxelizer's backward kernels, the decoding and the MLP's
tcgen05 backward (``render_step``).  The intensity-seeded initialisation of
the reference (``synthetic.from_image_init``) stays as the fallback -- an
untrained network reproduces it exactly -- and as the yardstick: the warm
start is scored by the final NMSE against the fully sampled phantom.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import time
from dataclasses import dataclass
from typing import List, Optional, Tuple

import torch

from . import sense, synthetic
from ._lib import check, lib

IN, HID, OUT = 256, 256, 16
N_TARGET = 12
PATCH = 5
EPI_F32, EPI_BIAS_GELU, EPI_GELU_GRAD, EPI_ATOMIC_F32 = 0, 1, 2, 3


def _p(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def gemm(a, a_strides, b, b_strides, M, N, K, epi, out_f32=None, out_bf16=None, z=None, bias=None,
         c_strides=None, splits=1, err=None, col_sum=None):
    """C = A B^T on the tcgen05 kernel (see include/gsv.h, gsv_mlp_gemm)."""
    if err is None:
        err = torch.zeros(1, dtype=torch.int32, device=a.device)
    c_sm, c_sn = c_strides if c_strides else (N, 1)
    check(lib.gsv_mlp_gemm(_p(a), a_strides[0], a_strides[1], _p(b), b_strides[0], b_strides[1], M, N, K, splits,
                           _p(bias), _p(out_f32), _p(out_bf16), _p(z), c_sm, c_sn, epi, _p(col_sum), _p(err),
                           ctypes.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)), "gsv_mlp_gemm")
    return err


# ---------------------------------------------------------------------------
# features and decoding
# ---------------------------------------------------------------------------

def image_scale(zero_filled: torch.Tensor) -> float:
    return float(torch.quantile(zero_filled.abs().reshape(-1)[::7].float(), 0.999).clamp_min(1e-6))


def patch_features(zero_filled: torch.Tensor, voxels: torch.Tensor, sampling_density: float,
                   scale: float, log_base_scale: torch.Tensor) -> torch.Tensor:
    """[N, 256] BF16 features: the 5^3 complex patch around each seed voxel
    (zero outside the volume), real then imaginary parts, divided by `scale`;
    then the sampling density of the acquisition and the log of the seed's
    intensity-seeded scale (voxels); then zeros."""
    dev = zero_filled.device
    r = PATCH // 2
    pad = torch.nn.functional.pad(zero_filled.real.unsqueeze(0).unsqueeze(0), (r,) * 6).squeeze()
    padi = torch.nn.functional.pad(zero_filled.imag.unsqueeze(0).unsqueeze(0), (r,) * 6).squeeze()
    off = torch.arange(PATCH, device=dev)
    od, oh, ow = torch.meshgrid(off, off, off, indexing="ij")
    d = voxels[:, 0:1] + od.reshape(1, -1)
    h = voxels[:, 1:2] + oh.reshape(1, -1)
    w = voxels[:, 2:3] + ow.reshape(1, -1)
    feats = torch.zeros(voxels.shape[0], IN, device=dev, dtype=torch.float32)
    feats[:, :125] = pad[d, h, w] / scale
    feats[:, 125:250] = padi[d, h, w] / scale
    feats[:, 250] = sampling_density
    feats[:, 251] = log_base_scale
    return feats.bfloat16()


def seed_voxels(init: synthetic.GaussianSet, shape) -> torch.Tensor:
    """Voxel index of each seed position (from_image places seeds at voxel centres)."""
    s = torch.tensor(shape, dtype=torch.float32, device=init.positions.device)
    cv = (init.positions + 1.0) * 0.5 * s - 0.5
    return torch.minimum(torch.clamp(torch.round(cv), min=0), s - 1).long()


def decode(out: torch.Tensor, seed_vox: torch.Tensor, base: synthetic.GaussianSet, shape, scale: float):
    """Network outputs -> (positions, scales, rotations, density_r, density_i),
    differentiable.  Every output is a correction of the intensity-seeded
    Gaussian (zero output = the plain init): offsets bounded to half a voxel,
    log-scale corrections bounded to +-1, a quaternion correction of the
    identity, a density correction in units of the image scale."""
    s = torch.tensor(shape, dtype=torch.float32, device=out.device)
    cv = seed_vox.float() + 0.5 * torch.tanh(out[:, 0:3])
    pos = (cv + 0.5) / s * 2 - 1
    scales = base.scales * torch.exp(torch.tanh(out[:, 3:6]))
    q = out[:, 6:10] * 0.25
    q = torch.cat([1.0 + q[:, :1], q[:, 1:]], 1)
    q = q / q.norm(dim=-1, keepdim=True)
    return pos, scales, q, base.density_r + out[:, 10] * scale, base.density_i + out[:, 11] * scale


# ---------------------------------------------------------------------------
# the network
# ---------------------------------------------------------------------------

class WarmStartMLP:
    def __init__(self, device="cuda:0", seed: int = 0, lr: float = 1e-3):
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)

        def lin(o, i):
            return (torch.randn(o, i, generator=g) * math.sqrt(2.0 / i)).to(self.device)

        self.w = [lin(HID, IN), lin(HID, HID), lin(OUT, HID) * 0.1]
        self.b = [torch.zeros(HID, device=self.device), torch.zeros(HID, device=self.device),
                  torch.zeros(OUT, device=self.device)]
        for t in self.w + self.b:
            t.requires_grad_(False)
        self.params = [torch.nn.Parameter(t) for t in self.w + self.b]
        self.opt = torch.optim.Adam(self.params, lr=lr)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._sync_bf16()

    def _sync_bf16(self):
        self.wb = [p.detach().bfloat16().contiguous() for p in self.params[:3]]

    def forward(self, x: torch.Tensor):
        """x: [B, 256] BF16 -> standardized outputs [B, 16] FP32 and the cache."""
        B = x.shape[0]
        dev = x.device
        z1 = torch.empty(B, HID, device=dev)
        y1 = torch.empty(B, HID, device=dev, dtype=torch.bfloat16)
        gemm(x, (IN, 1), self.wb[0], (IN, 1), B, HID, IN, EPI_BIAS_GELU, out_bf16=y1, z=z1,
             bias=self.params[3].detach(), err=self.err)
        z2 = torch.empty(B, HID, device=dev)
        y2 = torch.empty(B, HID, device=dev, dtype=torch.bfloat16)
        gemm(y1, (HID, 1), self.wb[1], (HID, 1), B, HID, HID, EPI_BIAS_GELU, out_bf16=y2, z=z2,
             bias=self.params[4].detach(), err=self.err)
        out = torch.empty(B, OUT, device=dev)
        gemm(y2, (HID, 1), self.wb[2], (HID, 1), B, OUT, HID, EPI_F32, out_f32=out, bias=self.params[5].detach(),
             err=self.err)
        return out, (x, z1, y1, z2, y2)

    def backward(self, cache, dout: torch.Tensor) -> List[torch.Tensor]:
        """Gradients of (W1, W2, W3, b1, b2, b3) for upstream dout [B, 16] FP32."""
        x, z1, y1, z2, y2 = cache
        B = x.shape[0]
        dev = x.device
        splits = max(1, min(64, B // 256))
        dob = dout.bfloat16().contiguous()
        dW3 = torch.zeros(OUT, HID, device=dev)
        gemm(y2, (1, HID), dob, (1, OUT), HID, OUT, B, EPI_ATOMIC_F32, out_f32=dW3, c_strides=(1, HID),
             splits=splits, err=self.err)
        dz2 = torch.empty(B, HID, device=dev, dtype=torch.bfloat16)
        db2 = torch.zeros(HID, device=dev)
        gemm(dob, (OUT, 1), self.wb[2], (1, HID), B, HID, OUT, EPI_GELU_GRAD, out_bf16=dz2, z=z2, err=self.err,
             col_sum=db2)
        dW2 = torch.zeros(HID, HID, device=dev)
        gemm(dz2, (1, HID), y1, (1, HID), HID, HID, B, EPI_ATOMIC_F32, out_f32=dW2, splits=splits, err=self.err)
        dz1 = torch.empty(B, HID, device=dev, dtype=torch.bfloat16)
        db1 = torch.zeros(HID, device=dev)
        gemm(dz2, (HID, 1), self.wb[1], (1, HID), B, HID, HID, EPI_GELU_GRAD, out_bf16=dz1, z=z1, err=self.err,
             col_sum=db1)
        dW1 = torch.zeros(HID, IN, device=dev)
        gemm(dz1, (1, HID), x, (1, IN), HID, IN, B, EPI_ATOMIC_F32, out_f32=dW1, splits=splits, err=self.err)
        return [dW1, dW2, dW3, db1, db2, dout.sum(0)]

    def check_ok(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("tcgen05 GEMM wait timed out")

    @torch.no_grad()
    def predict(self, x: torch.Tensor) -> torch.Tensor:
        out, _ = self.forward(x)
        self.check_ok()
        return out

    def apply_grads(self, grads: List[torch.Tensor]):
        for p, g in zip(self.params, grads):
            p.grad = g
        self.opt.step()
        self._sync_bf16()

    def state_dict(self):
        return {"params": [p.detach().cpu() for p in self.params]}

    def load_state_dict(self, sd):
        for p, t in zip(self.params, sd["params"]):
            p.data.copy_(t.to(self.device))
        self._sync_bf16()


# ---------------------------------------------------------------------------
# training data from plain fits, training through the voxelizer, warm init
# ---------------------------------------------------------------------------

@dataclass
class WarmConfig:
    shape: Tuple[int, int, int] = (96, 96, 96)
    n_coils: int = 8
    accel: float = 6.0
    calib: int = 24
    points_per_voxel: float = 50_000 / (128 * 128 * 96)
    mask_kind: str = "vd"  # "poisson": the reference's Poisson-disc (ky, kz) sampling (synthetic.mri_case)
    fit_iterations: int = 1000
    # the training target: "best" = the plain fit's best-PSNR evaluation under the reference
    # trainer's metric-plateau stop (what the reference reports); "last" = its last iterate
    target: str = "best"
    # MLP seeds per training phantom relative to the plain method's count: the network sets up
    # the larger Gaussian set the plain method only reaches through densification
    seed_factor: float = 3.0
    # training loss: "volume" = relative L2 of the rendered volume to the target volume;
    # "dc" = the same after hard data consistency of both (only the unsampled k-space, which the
    # measured samples do not fix, is compared)
    loss: str = "dc"
    # seed draw of the warm start: "random" (the reference's paper profile) or "importance"
    # (its other mode: voxels above the 90th magnitude percentile); the plain fits that make
    # the targets always seed as the paper profile does
    seed_mode: str = "importance"
    # learning-rate factor of the fit that starts from the warm start (every parameter group):
    # the warm start sits close to a good fit, and the plain method's step sizes kick it away
    fit_lr_scale: float = 0.5

    def fit_overrides(self) -> dict:
        """FitConfig fields the warm-started fit overrides (the plain method's schedule otherwise)."""
        if self.fit_lr_scale == 1.0:
            return {}
        base = sense.FitConfig()
        f = self.fit_lr_scale
        return {"position_lr": base.position_lr * f, "scale_lr": base.scale_lr * f,
                "rotation_lr": base.rotation_lr * f, "density_lr": base.density_lr * f}


@dataclass
class TrainingCase:
    shape: Tuple[int, int, int]
    features: torch.Tensor        # [N, 256] BF16
    seed_vox: torch.Tensor        # [N, 3]
    base: synthetic.GaussianSet   # intensity-seeded Gaussians (the plain init)
    scale: float
    target: torch.Tensor          # complex64 volume of the plain fit
    coils: Optional[torch.Tensor] = None  # (C,D,H,W) complex64, for the "dc" loss (shared, _shared_coils)
    mask: Optional[torch.Tensor] = None   # (D,H,W) bool sampling mask, for the "dc" loss


def case_inputs(case: synthetic.MRICase, num_points: int, seed: int, device, mode: str = "random"):
    dev = torch.device(device)
    base = synthetic.from_image_init(case.zero_filled, num_points, seed=seed, device=dev, mode=mode).to(dev)
    shape = tuple(case.ground_truth.shape)
    zf = case.zero_filled.to(dev)
    scale = image_scale(zf)
    vox = seed_voxels(base, shape)
    s = torch.tensor(shape, dtype=torch.float32, device=dev)
    log_base = torch.log(base.scales[:, 0] * s.max() * 0.5)
    x = patch_features(zf, vox, float(case.mask.mean()), scale, log_base)
    return x, vox, base, scale


_COILS = {}


def _shared_coils(case: synthetic.MRICase, device) -> torch.Tensor:
    """One coil-map tensor per (shape, coil count, device) for the "dc" loss
    of every training case.  The synthetic maps (``synthetic.ring_coils``)
    of two seeds differ only by a constant phase per coil, and
    ``_unsampled`` is invariant to it: conj(S e^{ip}) F^-1((1-m) F(S e^{ip} v))
    = conj(S) F^-1((1-m) F(S v)).  Sharing the first case's maps therefore
    gives every case its own loss and keeps 57 MB per 96^3 case off the
    device (``tests/test_warmstart_cpu.py`` checks the invariance)."""
    key = (tuple(case.sensitivity_maps.shape), str(device))
    if key not in _COILS:
        _COILS[key] = case.sensitivity_maps.to(device).to(torch.complex64)
    return _COILS[key]


def synthetic_case(seed: int, wc: WarmConfig) -> synthetic.MRICase:
    """The seeded training acquisition of ``training_case`` (host-generated)."""
    return synthetic.mri_case(wc.shape, n_coils=wc.n_coils, accel=wc.accel, calib=wc.calib, seed=seed,
                              mask_kind=wc.mask_kind)


def training_case(seed: int, wc: WarmConfig, device="cuda:0",
                  case: Optional[synthetic.MRICase] = None) -> TrainingCase:
    """A synthetic phantom, its intensity-seeded Gaussians and the volume the
    plain method reconstructs from them (the training target).  `case`:
    ``synthetic_case(seed, wc)`` when the caller made it already."""
    if case is None:
        case = synthetic_case(seed, wc)
    n = int(round(wc.points_per_voxel * math.prod(wc.shape)))
    _, _, plain_base, _ = case_inputs(case, n, seed + 1, device)
    if wc.seed_factor == 1.0 and wc.seed_mode == "random":
        x, vox, base, scale = case_inputs(case, n, seed + 1, device)
    else:
        x, vox, base, scale = case_inputs(case, int(round(n * wc.seed_factor)), seed + 2, device, wc.seed_mode)
    if wc.target == "best":
        cfg = sense.FitConfig(iterations=wc.fit_iterations, eval_every=50, plateau_stop=True, keep_best=True)
    else:
        cfg = sense.FitConfig(iterations=wc.fit_iterations, eval_every=10 ** 9)
    res = sense.fit(case, plain_base, cfg, device=device, eval_ssim=False)
    from .tile_voxelizer import TileVoxelizer

    vz = TileVoxelizer(wc.shape, device=device)
    g = res.best_params if wc.target == "best" else res.params.snapshot()
    with torch.no_grad():
        target = vz(g.positions, g.scales, g.rotations, torch.complex(g.density_r, g.density_i))
    dev = torch.device(device)
    coils = _shared_coils(case, dev) if wc.loss == "dc" else None
    mask = (case.mask.to(dev) > 0.5) if wc.loss == "dc" else None
    return TrainingCase(wc.shape, x, vox, base, scale, target.detach(), coils, mask)


def training_cases(seeds, wc: WarmConfig, device="cuda:0") -> List[TrainingCase]:
    """``training_case`` for every seed, with each next acquisition generated
    on a host thread while the device fits the current one (same cases as
    one ``training_case`` call per seed)."""
    from concurrent.futures import ThreadPoolExecutor

    seeds = list(seeds)
    out = []
    with ThreadPoolExecutor(max_workers=1) as pool:
        nxt = pool.submit(synthetic_case, seeds[0], wc) if seeds else None
        for i, s in enumerate(seeds):
            case = nxt.result()
            nxt = pool.submit(synthetic_case, seeds[i + 1], wc) if i + 1 < len(seeds) else None
            out.append(training_case(s, wc, device, case=case))
    return out


def _unsampled(vol: torch.Tensor, coils: torch.Tensor, mask: torch.Tensor) -> torch.Tensor:
    """The part of `vol` hard data consistency leaves in place: the coil
    images' k-space outside the sampling mask, combined back with the coils
    (the difference of two hard-DC volumes is this map of their difference)."""
    k = synthetic.fft3c(coils * vol.unsqueeze(0)) * (~mask if mask.dtype == torch.bool else 1.0 - mask).unsqueeze(0)
    return (torch.conj(coils) * synthetic.ifft3c(k)).sum(0)


def render_step(mlp: WarmStartMLP, tc: TrainingCase, vox) -> float:
    """One training step: MLP -> decode -> voxelize -> relative L2 to the
    plain fit's volume; gradients back through the voxelizer's backward and
    the MLP's tcgen05 backward."""
    out, cache = mlp.forward(tc.features)
    out = out.requires_grad_(True)
    pos, scl, rot, dr, di = decode(out, tc.seed_vox, tc.base, tc.shape, tc.scale)
    vol = vox(pos, scl, rot, torch.complex(dr, di))
    diff = vol - tc.target
    if tc.coils is not None:  # "dc" loss: compare what hard data consistency keeps
        diff = _unsampled(diff, tc.coils, tc.mask)
    loss = (diff.real.square().sum() + diff.imag.square().sum()) / tc.target.abs().square().sum()
    loss.backward()
    mlp.apply_grads(mlp.backward(cache, out.grad))
    return float(loss.detach())


def train(mlp: WarmStartMLP, cases: List[TrainingCase], steps: int = 1500, seed: int = 0, log=None) -> List[float]:
    from .tile_voxelizer import TileVoxelizer

    voxes = {}
    g = torch.Generator().manual_seed(seed)
    losses = []
    for i in range(steps):
        tc = cases[int(torch.randint(0, len(cases), (1,), generator=g))]
        if tc.shape not in voxes:
            voxes[tc.shape] = TileVoxelizer(tc.shape, device=str(mlp.device))
        losses.append(render_step(mlp, tc, voxes[tc.shape]))
        if log and (i % 100 == 0 or i == steps - 1):
            log({"step": i, "loss": losses[-1]})
    mlp.check_ok()
    return losses


@torch.no_grad()
def warm_init(mlp: WarmStartMLP, case: synthetic.MRICase, num_points: int, seed: int = 0,
              device="cuda:0", mode: str = "random") -> synthetic.GaussianSet:
    """Seeds exactly as the intensity-seeded init (same seed and mode ->
    same voxels and scales), parameters from the MLP."""
    x, vox, base, scale = case_inputs(case, num_points, seed, device, mode)
    out = mlp.predict(x)
    pos, scl, rot, dr, di = decode(out, vox, base, tuple(case.ground_truth.shape), scale)
    return synthetic.GaussianSet(pos.contiguous(), scl.contiguous(), rot.contiguous(), dr.contiguous(),
                                 di.contiguous())


def warm_start(mlp: WarmStartMLP, case: synthetic.MRICase, plain_points: int, wc: WarmConfig, seed: int = 0,
               device="cuda:0") -> synthetic.GaussianSet:
    """The warm start for an acquisition whose plain fit seeds `plain_points`
    Gaussians: `wc.seed_factor` times as many seeds, drawn as `wc.seed_mode`,
    with their parameters from the network."""
    return warm_init(mlp, case, int(round(plain_points * wc.seed_factor)), seed=seed, device=device,
                     mode=wc.seed_mode)


def time_to_target(mlp: Optional[WarmStartMLP], case: synthetic.MRICase, num_points: int, seed: int = 0,
                   device="cuda:0", cadence: int = 10, max_iterations: int = 2000,
                   warm_points: Optional[int] = None, ablation: bool = False, warm_mode: str = "random",
                   warm_schedule: Optional[dict] = None) -> dict:
    """Warm start against the plain method on one acquisition.

    The plain method runs as the reference trainer runs it (evaluation
    every 50 iterations, metric-plateau stop, best evaluation by PSNR); its
    best NMSE is the target.  Then the plain fit and the warm-started fit
    each run from their initialisation until their hard-data-consistency
    NMSE first reaches the target, evaluated every `cadence` iterations.
    Times are wall seconds of initialisation plus fitting (evaluations
    excluded); all fits use the deterministic backward, so the plain rerun
    retraces the first run exactly.  `mlp` None: the warm arm is skipped.
    `warm_points`, `warm_mode`: seed count and seed draw of the warm start
    (default: the plain method's); `warm_schedule`: FitConfig fields the
    warm-started fit overrides (default none: the plain method's schedule);
    `ablation`: also time intensity seeding with the warm start's seeds,
    draw and schedule but no network, which separates what the network adds
    from what the seeding and schedule add."""
    dev = torch.device(device)
    shape = tuple(case.ground_truth.shape)
    rule = sense.FitConfig(iterations=max_iterations, eval_every=50, plateau_stop=True, deterministic=True)

    def timed_init(fn):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize(dev)
        return out, time.perf_counter() - t0

    plain_init, t_plain_init = timed_init(
        lambda: synthetic.from_image_init(case.zero_filled, num_points, seed=seed, device=dev))
    ref = sense.fit(case, plain_init, rule, device=device, eval_ssim=False)
    target = ref.best["nmse"]
    to_target = sense.FitConfig(iterations=max_iterations, eval_every=cadence, deterministic=True)

    def first_hit(res):
        hit = [h for h in res.history if h["nmse"] <= target]
        return (hit[0]["iteration"], hit[0]["seconds"]) if hit else (None, None)

    plain = sense.fit(case, plain_init, to_target, device=device, stop_nmse=target, eval_ssim=False)
    p_it, p_s = first_hit(plain)
    row = {"target_nmse": target, "plain_best_iteration": ref.best["iteration"],
           "plain_stopped_at": ref.history[-1]["iteration"], "plain_nmse_at_0": plain.history[0]["nmse"],
           "plain_iterations_to_target": p_it, "plain_init_seconds": t_plain_init,
           "plain_seconds_to_target": None if p_s is None else p_s + t_plain_init}
    if mlp is None:
        return row
    nw = warm_points or num_points
    warm_cfg = dataclasses.replace(to_target, **(warm_schedule or {}))
    warm, t_warm_init = timed_init(lambda: warm_init(mlp, case, nw, seed=seed, device=device, mode=warm_mode))
    w = sense.fit(case, warm, warm_cfg, device=device, stop_nmse=target, eval_ssim=False)
    w_it, w_s = first_hit(w)
    row.update({"warm_points": nw, "warm_nmse_at_0": w.history[0]["nmse"], "warm_iterations_to_target": w_it,
                "warm_init_seconds": t_warm_init,
                "warm_seconds_to_target": None if w_s is None else w_s + t_warm_init})
    if w_s is not None and p_s:
        row["wall_ratio"] = row["warm_seconds_to_target"] / row["plain_seconds_to_target"]
    if ablation:
        seeded, t_seed = timed_init(
            lambda: synthetic.from_image_init(case.zero_filled, nw, seed=seed, device=dev, mode=warm_mode))
        a = sense.fit(case, seeded, warm_cfg, device=device, stop_nmse=target, eval_ssim=False)
        a_it, a_s = first_hit(a)
        row.update({"seeded_nmse_at_0": a.history[0]["nmse"], "seeded_iterations_to_target": a_it,
                    "seeded_seconds_to_target": None if a_s is None else a_s + t_seed})
    return row


def time_training_pass(batch: int = 65536, iters: int = 5, device="cuda:0", seed: int = 0) -> dict:
    """CUDA-event time of one MLP forward + backward (8 tcgen05 GEMMs) on a
    random BF16 batch, with the bytes those GEMMs must move at least: every
    operand read once, every output written once."""
    mlp = WarmStartMLP(device, seed=seed)
    g = torch.Generator(device=device).manual_seed(seed)
    x = torch.randn(batch, IN, device=device, generator=g).bfloat16()
    dout = torch.randn(batch, OUT, device=device, generator=g) / batch
    for _ in range(2):
        mlp.backward(mlp.forward(x)[1], dout)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        mlp.backward(mlp.forward(x)[1], dout)
    e1.record()
    torch.cuda.synchronize(device)
    mlp.check_ok()
    ms = e0.elapsed_time(e1) / iters
    b = batch
    # forward: x, y1, y2 read (bf16); z1, z2 (f32) + y1, y2 (bf16) + out (f32) written
    fwd = 2 * b * (IN + 2 * HID) + b * (4 + 2) * 2 * HID + 4 * b * OUT
    bwd = (2 * b * (HID + OUT)                        # dW3: y2, dout
           + 2 * b * OUT + 4 * b * HID + 2 * b * HID  # dz2: dout, z2 -> dz2
           + 4 * b * HID                              # dW2: dz2, y1
           + 2 * b * HID + 4 * b * HID + 2 * b * HID  # dz1: dz2, z1 -> dz1
           + 2 * b * (HID + IN))                      # dW1: dz1, x
    flops = 2 * b * (IN * HID + HID * HID + HID * OUT) * 3
    return {"batch": batch, "ms": ms, "min_bytes": fwd + bwd, "gbs": (fwd + bwd) / (ms * 1e-3) / 1e9,
            "tflops": flops / (ms * 1e-3) / 1e12}


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="time one warm-start MLP training pass on the tcgen05 GEMMs")
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--iters", type=int, default=5)
    a = ap.parse_args()
    print(json.dumps(time_training_pass(a.batch, a.iters)))
