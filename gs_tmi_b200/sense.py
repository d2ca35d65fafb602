"""The SENSE data-consistency loop that calls the voxelizer (plain 3DGSMR fit).

A compact restatement of the reference trainer's plain method, used as the
caller of the voxelizer for reconstruction runs, parity runs against the
reference kernels and the warm-start evaluation.  Reference (V = 3DGS/3dgsVC):

* loss (``V/trainers/trainer.py:256-283``, ``V/losses/losses.py:18-26``):
  || mask * fft3c(S x) - y ||^2 + tv_weight * TV(|x|)
* optimiser (``trainer.py:167-183``, ``V/gaussian/gaussian_model.py:76-83``):
  Adam with per-tensor learning rates, ExponentialLR(gamma), grad-norm clip
  (``trainer.py:426-439``)
* adaptive density control (``trainer.py:294-352``,
  ``gaussian_model.py:85-222``): split (two children drawn around the parent,
  scales / 1.6, density x 0.5), clone (density halved and duplicated), prune
  (|rho| < opacity threshold or max scale > limit), Adam moments transplanted
  for surviving rows (``trainer.py:355-424``)
* evaluation (``trainer.py:237-243``, ``V/metrics/metrics.py:70-77``):
  hard data consistency, then magnitude NMSE; SSIM follows the published
  definition (Wang et al. 2004) with a uniform 7^3 window, K1=0.01, K2=0.03,
  sample covariance.

The voxelizer is any callable (positions, scales, rotations, density) ->
complex64 volume; the default is this package's ``TileVoxelizer``.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import torch
import torch.nn as nn
import torch.nn.functional as F

from .synthetic import GaussianSet, MRICase, fft3c, ifft3c


@dataclass
class FitConfig:
    iterations: int = 2000
    position_lr: float = 1e-3
    scale_lr: float = 5e-3
    rotation_lr: float = 1e-3
    density_lr: float = 1e-2
    gamma: float = 0.999
    max_grad_norm: float = 1.0
    tv_weight: float = 0.1
    densify_from: int = 100
    densify_every: int = 100
    densify_until: int = 2500
    grad_threshold: float = 0.01
    scale_threshold: float = 0.01
    opacity_threshold: float = 0.01
    max_scale: float = 0.5
    max_points: int = 500_000
    use_cloning: bool = True
    long_axis_split: bool = False        # "long_axis" strategy: deterministic children (gaussian_model.py:112-131)
    long_axis_offset_factor: float = 1.0
    tile_size: int = 8
    deterministic: bool = False
    eval_every: int = 100
    seed: int = 0
    capturable_adam: bool = False  # device-side LR/bias correction (what fit_graph uses)
    fused_sense: bool = True       # data term through the fused SENSE kernels (sense_data_term)
    # the reference trainer's early stop on ground-truth metrics (PlateauStop; V/configs/default.yaml
    # `stopping`: enable_metric_plateau, min_iterations_before_stop, patience_evals, metric_min_delta)
    plateau_stop: bool = False
    plateau_patience: int = 4
    plateau_min_iterations: int = 200
    plateau_min_delta_psnr: float = 0.05
    plateau_min_delta_ssim: float = 0.0005
    keep_best: bool = False  # snapshot the parameters at the best-PSNR evaluation (the reference's best.pth)


@dataclass
class PlateauStop:
    """The reference trainer's early stop on ground-truth metrics
    (V/metrics/metrics.py:166-195, driven by V/trainers/trainer.py:571-590).
    After each evaluation a metric counts as improved when it beats its best
    so far by more than its minimum delta; any improved metric resets the
    count of evaluations without improvement, and the fit stops once the
    iteration is at least `min_iterations` and `patience` evaluations in a
    row improved nothing."""
    patience: int = 4
    min_iterations: int = 200
    min_delta: Dict[str, float] = field(default_factory=lambda: {"psnr": 0.05, "ssim": 0.0005})
    best: Dict[str, float] = field(default_factory=dict)
    bad: int = 0

    def update(self, iteration: int, metrics: Dict[str, float]) -> bool:
        improved = False
        for name, value in metrics.items():
            if value is None:
                continue
            if name not in self.best or value > self.best[name] + self.min_delta.get(name, 0.0):
                self.best[name] = value
                improved = True
        self.bad = 0 if improved else self.bad + 1
        return iteration >= self.min_iterations and self.bad >= self.patience


# ---------------------------------------------------------------------------
# metrics / losses
# ---------------------------------------------------------------------------

def magnitude_tv(vol: torch.Tensor) -> torch.Tensor:
    m = vol.abs()
    return ((m[1:] - m[:-1]).abs().sum() + (m[:, 1:] - m[:, :-1]).abs().sum()
            + (m[:, :, 1:] - m[:, :, :-1]).abs().sum())


def nmse(pred: torch.Tensor, target: torch.Tensor) -> float:
    p, t = pred.abs().double(), target.abs().double()
    den = float((t * t).sum())
    return float(((p - t) ** 2).sum()) / den if den > 0 else float("inf")


def psnr(pred: torch.Tensor, target: torch.Tensor) -> float:
    p, t = pred.abs().double(), target.abs().double()
    mse = float(((p - t) ** 2).mean())
    peak = float(t.max())
    return 10 * math.log10(peak * peak / mse) if mse > 0 else float("inf")


def ssim3d(pred: torch.Tensor, target: torch.Tensor, data_range: Optional[float] = None, win: int = 7) -> float:
    x = pred.abs().double()[None, None]
    y = target.abs().double()[None, None]
    if data_range is None:
        data_range = float(y.max() - y.min()) or 1.0
    c1, c2 = (0.01 * data_range) ** 2, (0.03 * data_range) ** 2
    n = win ** 3
    mu = lambda a: F.avg_pool3d(a, win, stride=1)
    mx, my = mu(x), mu(y)
    cov = n / (n - 1)
    sxx = (mu(x * x) - mx * mx) * cov
    syy = (mu(y * y) - my * my) * cov
    sxy = (mu(x * y) - mx * my) * cov
    s = ((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))
    return float(s.mean())


class _SenseDataTerm(torch.autograd.Function):
    """sum_c || M * fft3c(S_c x) - y_c ||^2 with the coil product, the FFT
    shifts, the mask, the residual, its square sum and the adjoint coil sum
    in the library's fused kernels (gsv_sense_*) and the FFTs in torch.fft."""

    @staticmethod
    def forward(ctx, vol, S, mask, ku, ws):
        from ._lib import check, lib

        nc, (d, h, w) = S.shape[0], vol.shape
        st = torch.cuda.current_stream(vol.device).cuda_stream
        X = torch.empty_like(S)
        check(lib.gsv_sense_expand(vol.data_ptr(), S.data_ptr(), nc, d, h, w, X.data_ptr(), st), "gsv_sense_expand")
        K = torch.fft.fftn(X, dim=(-3, -2, -1), norm="ortho")
        loss = torch.empty((), device=vol.device)
        check(lib.gsv_sense_residual(K.data_ptr(), mask.data_ptr(), ku.data_ptr(), nc, d, h, w, loss.data_ptr(),
                                     ws.data_ptr(), ws.numel(), st), "gsv_sense_residual")
        ctx.save_for_backward(K, S)  # K now holds dL/dK = 2 M R
        return loss

    @staticmethod
    def backward(ctx, gout):
        from ._lib import check, lib

        K, S = ctx.saved_tensors
        nc, (d, h, w) = S.shape[0], S.shape[1:]
        with torch.cuda.device(K.device):  # the autograd thread may have no current context
            G = torch.fft.ifftn(K, dim=(-3, -2, -1), norm="ortho")
            vg = torch.empty((d, h, w), dtype=torch.complex64, device=K.device)
            check(lib.gsv_sense_adjoint(G.data_ptr(), S.data_ptr(), nc, d, h, w, vg.data_ptr(),
                                        torch.cuda.current_stream(K.device).cuda_stream), "gsv_sense_adjoint")
            return vg * gout, None, None, None, None


class _MagnitudeTV(torch.autograd.Function):
    """TV(|x|) (losses.py:18-26) with its gradient from the same pass of the
    library kernel (gsv_tv_magnitude)."""

    @staticmethod
    def forward(ctx, vol, ws):
        from ._lib import check, lib

        d, h, w = vol.shape
        loss = torch.empty((), device=vol.device)
        grad = torch.empty_like(vol)
        check(lib.gsv_tv_magnitude(vol.data_ptr(), d, h, w, loss.data_ptr(), grad.data_ptr(), ws.data_ptr(),
                                   ws.numel(), torch.cuda.current_stream(vol.device).cuda_stream), "gsv_tv_magnitude")
        ctx.save_for_backward(grad)
        return loss

    @staticmethod
    def backward(ctx, gout):
        (grad,) = ctx.saved_tensors
        return grad * gout, None


def magnitude_tv_fused(vol: torch.Tensor, ws: Optional[torch.Tensor] = None) -> torch.Tensor:
    """magnitude_tv on the GPU in one kernel (value and gradient)."""
    if ws is None:
        ws = sense_workspace(vol.device)
    return _MagnitudeTV.apply(vol.contiguous(), ws)


def sense_workspace(device) -> torch.Tensor:
    from ._lib import lib

    return torch.empty(int(lib.gsv_sense_workspace_bytes()), dtype=torch.uint8, device=device)


def sense_data_term(vol: torch.Tensor, S: torch.Tensor, mask: torch.Tensor, ku: torch.Tensor,
                    ws: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Scalar data term of the plain loss (trainer.py:256-268), differentiable
    in `vol` (complex64 [d,h,w]); S, ku complex64 [C,d,h,w], mask float32
    [d,h,w], all contiguous on the same GPU."""
    if ws is None:
        ws = sense_workspace(vol.device)
    return _SenseDataTerm.apply(vol.contiguous(), S, mask, ku, ws)


def data_term_reference(vol, S, mask_c, ku):
    """The same data term op by op in torch (the reference's formulation)."""
    diff = fft3c(vol.unsqueeze(0) * S) * mask_c - ku
    return diff.real.square().sum() + diff.imag.square().sum()


def hard_data_consistency(vol, S, mask, ku):
    """Replace the measured k-space samples (trainer.py:237-243)."""
    k = fft3c(vol.unsqueeze(0) * S)
    k = k * (1.0 - mask.unsqueeze(0)) + ku
    return (torch.conj(S) * ifft3c(k)).sum(0)


# ---------------------------------------------------------------------------
# parameters, optimiser, density control
# ---------------------------------------------------------------------------

class GaussianParams(nn.Module):
    """positions [N,3], log-scales [N,3], rotations [N,4], density re/im [N]
    as nn.Parameters (the layout of gaussian_model.py:38-68)."""

    def __init__(self, init: GaussianSet, device):
        super().__init__()
        self.positions = nn.Parameter(init.positions.to(device).clone())
        self.log_scales = nn.Parameter(torch.log(init.scales.to(device).clamp_min(1e-8)))
        self.rotations = nn.Parameter(init.rotations.to(device).clone())
        self.density_r = nn.Parameter(init.density_r.to(device).clone())
        self.density_i = nn.Parameter(init.density_i.to(device).clone())

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])

    def tensors(self):
        return [self.positions, self.log_scales, self.rotations, self.density_r, self.density_i]

    def replace(self, new: List[torch.Tensor]):
        for name, t in zip(("positions", "log_scales", "rotations", "density_r", "density_i"), new):
            setattr(self, name, nn.Parameter(t.detach().contiguous()))

    def snapshot(self) -> GaussianSet:
        return GaussianSet(self.positions.detach().clone(), torch.exp(self.log_scales.detach()),
                           self.rotations.detach().clone(), self.density_r.detach().clone(),
                           self.density_i.detach().clone())


def make_optimizer(p: GaussianParams, cfg: FitConfig, lrs=None, fused: Optional[bool] = None,
                   capturable: bool = False):
    lr = lrs or [cfg.position_lr, cfg.scale_lr, cfg.rotation_lr, cfg.density_lr, cfg.density_lr]
    groups = [{"params": [t], "lr": l} for t, l in zip(p.tensors(), lr)]
    kw = {}
    if fused is None:
        fused = p.positions.is_cuda
    if fused:
        kw["fused"] = True
    if capturable:
        kw["capturable"] = True
    return torch.optim.Adam(groups, **kw)


def transplant(old_opt, new_opt, keep: torch.Tensor, n_new: int):
    """Adam moments of surviving rows move to the new tensors; appended rows
    start at zero (trainer.py:355-389)."""
    for og, ng in zip(old_opt.param_groups, new_opt.param_groups):
        op, np_ = og["params"][0], ng["params"][0]
        st = old_opt.state.get(op)
        if not st or "exp_avg" not in st:
            continue
        new_state = {}
        for key in ("exp_avg", "exp_avg_sq"):
            kept = st[key][keep]
            pad = np_.shape[0] - kept.shape[0]
            if pad > 0:
                kept = torch.cat([kept, kept.new_zeros((pad,) + tuple(kept.shape[1:]))], 0)
            new_state[key] = kept.contiguous()
        new_state["step"] = st["step"].clone() if torch.is_tensor(st["step"]) else st["step"]
        new_opt.state[np_] = new_state


def _quat_rotation(q: torch.Tensor) -> torch.Tensor:
    """quaternion_to_rotation_matrix (gaussian_model.py:12-19)."""
    q = q / (q.norm(dim=-1, keepdim=True) + 1e-8)
    w, x, y, z = q.unbind(-1)
    return torch.stack([torch.stack([1 - 2 * y * y - 2 * z * z, 2 * x * y - 2 * z * w, 2 * x * z + 2 * y * w], -1),
                        torch.stack([2 * x * y + 2 * z * w, 1 - 2 * x * x - 2 * z * z, 2 * y * z - 2 * x * w], -1),
                        torch.stack([2 * x * z - 2 * y * w, 2 * y * z + 2 * x * w, 1 - 2 * x * x - 2 * y * y], -1)],
                       -2)


@torch.no_grad()
def density_control(p: GaussianParams, pos_grad: torch.Tensor, cfg: FitConfig, gen: Optional[torch.Generator],
                    on_event: Callable[[torch.Tensor], None], noise: Optional[torch.Tensor] = None):
    """Split, clone, prune (trainer.py:294-352, gaussian_model.py:85-186).
    After every change of the parameter tensors ``on_event(keep_mask)`` runs
    (the optimiser rebuild of trainer.py:391-424); returns the event count.
    ``noise`` [N,6]: the standard normals of the two children of each row
    (columns 0-2 and 3-5) instead of draws from ``gen``."""
    events = 0
    if p.n >= cfg.max_points:
        return events
    gnorm = pos_grad.norm(dim=-1)
    scales = torch.exp(p.log_scales)
    smax = scales.max(-1)[0]
    high = gnorm > cfg.grad_threshold
    split = high & (smax > cfg.scale_threshold)
    n_split = int(split.sum())
    did_split_branch = False
    if n_split > 0 and p.n + n_split <= cfg.max_points:
        did_split_branch = True
        par_pos = p.positions[split]
        par_s = scales[split]
        keep = ~split
        if cfg.long_axis_split:
            # gaussian_model.py:112-131
            axis = par_s.argmax(dim=-1)
            rows = torch.arange(n_split, device=par_s.device)
            child = par_s.clone()
            child[rows, axis] *= 0.5
            other = torch.ones_like(child, dtype=torch.bool)
            other[rows, axis] = False
            child[other] *= 0.85
            local = torch.zeros_like(par_pos)
            local[rows, axis] = child[rows, axis] * cfg.long_axis_offset_factor
            shift = torch.bmm(_quat_rotation(p.rotations[split]), local.unsqueeze(-1)).squeeze(-1)
            pos_new = [par_pos + shift, par_pos - shift]
            ls_new = torch.log(child + 1e-8).repeat(2, 1)
            dfac = 0.6
        else:
            if noise is not None:
                za, zb = noise[split, :3], noise[split, 3:]
            else:
                za = torch.randn(par_pos.shape, device=par_pos.device, generator=gen)
                zb = torch.randn(par_pos.shape, device=par_pos.device, generator=gen)
            pos_new = [par_pos + za * par_s * 0.5, par_pos + zb * par_s * 0.5]
            ls_new = torch.log(par_s / 1.6 + 1e-8).repeat(2, 1)
            dfac = 0.5
        new = [torch.cat([p.positions[keep], *pos_new]),
               torch.cat([p.log_scales[keep], ls_new]),
               torch.cat([p.rotations[keep], p.rotations[split].repeat(2, 1)]),
               torch.cat([p.density_r[keep], (p.density_r[split] * dfac).repeat(2)]),
               torch.cat([p.density_i[keep], (p.density_i[split] * dfac).repeat(2)])]
        p.replace(new)
        on_event(keep)
        events += 1
    if cfg.use_cloning and not did_split_branch:
        clone = high & (smax <= cfg.scale_threshold)
        n_clone = int(clone.sum())
        if n_clone > 0 and p.n + n_clone <= cfg.max_points:
            dr = p.density_r.detach().clone()
            di = p.density_i.detach().clone()
            dr[clone] *= 0.5
            di[clone] *= 0.5
            keep = torch.ones(p.n, dtype=torch.bool, device=dr.device)
            new = [torch.cat([p.positions, p.positions[clone]]),
                   torch.cat([p.log_scales, torch.log(scales[clone] + 1e-8)]),
                   torch.cat([p.rotations, p.rotations[clone]]),
                   torch.cat([dr, dr[clone]]), torch.cat([di, di[clone]])]
            p.replace(new)
            on_event(keep)
            events += 1
    scales = torch.exp(p.log_scales)
    smax = scales.max(-1)[0]
    mag = torch.abs(torch.complex(p.density_r, p.density_i))
    prune = (mag < cfg.opacity_threshold) | (smax > cfg.max_scale)
    keep = ~prune
    if int(keep.sum()) >= 100 and int(prune.sum()) > 0:
        p.replace([t[keep] for t in p.tensors()])
        on_event(keep)
        events += 1
    return events


# ---------------------------------------------------------------------------
# the fit
# ---------------------------------------------------------------------------

def _sync(dev: torch.device):
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)

@dataclass
class FitResult:
    params: GaussianParams
    history: List[Dict] = field(default_factory=list)
    seconds: float = 0.0
    final_nmse: float = float("nan")
    final_ssim: float = float("nan")
    final_psnr: float = float("nan")
    # the best evaluation by PSNR, as the reference trainer keeps it (trainer.py:455-471)
    best: Dict = field(default_factory=dict)
    best_params: Optional[GaussianSet] = None
    stopped_early: bool = False


def fit(case: MRICase, init: GaussianSet, cfg: FitConfig, voxelizer: Optional[Callable] = None,
        device="cuda:0", stop_nmse: Optional[float] = None, log: Optional[Callable] = None,
        eval_ssim: bool = True, split_noise: Optional[Callable[[int], torch.Tensor]] = None) -> FitResult:
    """Plain 3DGSMR fit of `case` from `init`.  Wall time excludes the
    evaluations; `stop_nmse` ends the fit at the first evaluation at or below
    that hard-DC NMSE (time-to-NMSE runs).  `split_noise(n)`, called once
    per densifying iteration, gives the [n,6] split noise instead of draws
    from the fit's generator.  With `cfg.plateau_stop` every evaluation also
    scores PSNR and SSIM and the fit ends as the reference trainer's metric
    plateau stop ends it; `res.best` is the best evaluation by PSNR either
    way (with `cfg.keep_best`, `res.best_params` its parameters)."""
    dev = torch.device(device)
    shape = tuple(case.ground_truth.shape)
    if voxelizer is None:
        from .tile_voxelizer import TileVoxelizer

        voxelizer = TileVoxelizer(shape, tile_size=cfg.tile_size, device=str(dev), deterministic=cfg.deterministic)
    S = case.sensitivity_maps.to(dev)
    mask = case.mask.to(dev).float().contiguous()
    ku = case.kspace_undersampled.to(dev).to(torch.complex64).contiguous()
    S = S.to(torch.complex64).contiguous()
    fused = cfg.fused_sense and dev.type == "cuda"
    ws = sense_workspace(dev) if fused else None
    ws_tv = sense_workspace(dev) if fused else None
    gt = case.ground_truth.to(dev)
    p = GaussianParams(init, dev)
    lrs = [cfg.position_lr, cfg.scale_lr, cfg.rotation_lr, cfg.density_lr, cfg.density_lr]
    if cfg.capturable_adam:
        lrs = [torch.tensor(v, device=dev) for v in lrs]
    opt = make_optimizer(p, cfg, lrs, capturable=cfg.capturable_adam)
    gen = torch.Generator(device=dev).manual_seed(cfg.seed)
    res = FitResult(params=p)
    stopper = (PlateauStop(cfg.plateau_patience, cfg.plateau_min_iterations,
                           {"psnr": cfg.plateau_min_delta_psnr, "ssim": cfg.plateau_min_delta_ssim})
               if cfg.plateau_stop else None)
    mask_c = mask.unsqueeze(0)
    skip_sched = False
    wall = 0.0
    _sync(dev)
    t0 = time.perf_counter()
    for it in range(cfg.iterations):
        opt.zero_grad(set_to_none=True)
        vol = voxelizer(p.positions, torch.exp(p.log_scales), p.rotations, torch.complex(p.density_r, p.density_i))
        if isinstance(vol, tuple):
            vol = torch.complex(vol[0], vol[1])
        loss = sense_data_term(vol, S, mask, ku, ws) if fused else data_term_reference(vol, S, mask_c, ku)
        if cfg.tv_weight > 0:
            loss = loss + cfg.tv_weight * (magnitude_tv_fused(vol, ws_tv) if fused else magnitude_tv(vol))
        loss.backward()
        pos_grad = p.positions.grad.detach().clone()
        if cfg.max_grad_norm > 0:
            torch.nn.utils.clip_grad_norm_(p.tensors(), cfg.max_grad_norm)
        opt.step()
        if (cfg.densify_from <= it <= cfg.densify_until and it % cfg.densify_every == 0):
            holder = [opt]
            lrs = [g["lr"] for g in opt.param_groups]

            def rebuild(keep, holder=holder, lrs=lrs):
                new_opt = make_optimizer(p, cfg, lrs, capturable=cfg.capturable_adam)
                transplant(holder[0], new_opt, keep, p.n)
                holder[0] = new_opt

            noise = split_noise(p.n) if split_noise is not None else None
            if density_control(p, pos_grad, cfg, gen, rebuild, noise=noise):
                opt = holder[0]
                skip_sched = True
        if skip_sched:
            skip_sched = False
        elif cfg.capturable_adam:
            torch._foreach_mul_([g["lr"] for g in opt.param_groups], cfg.gamma)
        else:
            for g in opt.param_groups:
                g["lr"] *= cfg.gamma
        last = it == cfg.iterations - 1
        if (it % cfg.eval_every == 0) or last:
            _sync(dev)
            wall += time.perf_counter() - t0
            with torch.no_grad():
                v = voxelizer(p.positions, torch.exp(p.log_scales), p.rotations,
                              torch.complex(p.density_r, p.density_i))
                if isinstance(v, tuple):
                    v = torch.complex(v[0], v[1])
                rec = hard_data_consistency(v, S, mask, ku)
                e = nmse(rec, gt)
                row = {"iteration": it, "loss": float(loss.detach()), "nmse": e, "n_points": p.n, "seconds": wall,
                       "psnr": psnr(rec, gt)}
                if stopper is not None:
                    row["ssim"] = ssim3d(rec, gt)
                if not res.best or row["psnr"] > res.best["psnr"]:
                    res.best = dict(row)
                    if cfg.keep_best:
                        res.best_params = p.snapshot()
            res.history.append(row)
            if log:
                log(row)
            done = stop_nmse is not None and e <= stop_nmse
            if stopper is not None and stopper.update(it, {"psnr": row["psnr"], "ssim": row["ssim"]}):
                done = True
                res.stopped_early = not last
            if last or done:
                res.final_nmse = e
                res.final_psnr = psnr(rec, gt)
                if eval_ssim:
                    res.final_ssim = ssim3d(rec, gt)
                if done:
                    break
            _sync(dev)
            t0 = time.perf_counter()
    res.seconds = wall
    return res


# ---------------------------------------------------------------------------
# the same fit with each iteration replayed from a CUDA graph
# ---------------------------------------------------------------------------

class _GraphedStep:
    """One training iteration (voxelize -> coils -> FFT -> mask -> loss ->
    backward -> clip -> Adam) captured in a CUDA graph for a fixed Gaussian
    count.  The graph first snapshots parameters and Adam state, so an
    iteration whose tile pairs overflowed the static capacity can be undone
    and re-run with a larger capacity."""

    def __init__(self, p, opt, vox, S, mask_c, ku, cfg, capacity):
        self.p, self.opt, self.cfg = p, opt, cfg
        self.svox = vox.static(p.n, capacity)
        self.capacity = capacity
        dev = p.positions.device
        for t in p.tensors():
            t.grad = torch.zeros_like(t)
        self.pos_grad = torch.zeros_like(p.positions)
        self.loss = torch.zeros((), device=dev)
        self.flags_host = torch.zeros(1, dtype=torch.int32).pin_memory()
        self.state_tensors = []
        for t in p.tensors():
            st = opt.state.get(t, {})
            self.state_tensors += [st[k] for k in ("exp_avg", "exp_avg_sq", "step") if k in st]
        # Adam creates its state lazily at the first step: an undo before that
        # must drop the state again
        self.had_state = bool(self.state_tensors)
        self.live = p.tensors() + self.state_tensors
        self.snap = [torch.empty_like(t) for t in self.live]
        self.S, self.mask_c, self.ku = S, mask_c, ku
        self.ws = sense_workspace(dev) if cfg.fused_sense else None
        self.ws_tv = sense_workspace(dev) if cfg.fused_sense else None
        self.graph = None
        self.stream = torch.cuda.Stream(dev)

    def _body(self):
        torch._foreach_copy_(self.snap, self.live)
        for t in self.p.tensors():
            t.grad.zero_()
        p = self.p
        vol = self.svox(p.positions, torch.exp(p.log_scales), p.rotations, torch.complex(p.density_r, p.density_i))
        if self.cfg.fused_sense:
            loss = sense_data_term(vol, self.S, self.mask_c[0], self.ku, self.ws)
        else:
            loss = data_term_reference(vol, self.S, self.mask_c, self.ku)
        if self.cfg.tv_weight > 0:
            tv = magnitude_tv_fused(vol, self.ws_tv) if self.cfg.fused_sense else magnitude_tv(vol)
            loss = loss + self.cfg.tv_weight * tv
        loss.backward()
        self.pos_grad.copy_(p.positions.grad)
        if self.cfg.max_grad_norm > 0:
            torch.nn.utils.clip_grad_norm_(p.tensors(), self.cfg.max_grad_norm)
        self.opt.step()
        self.loss.copy_(loss.detach())
        self.flags_host.copy_(self.svox.plan.flags_dev, non_blocking=True)

    def eager(self):
        """Run one real iteration outside the graph (also the capture warm-up),
        on the stream the capture will use."""
        dev = self.p.positions.device
        self.stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(self.stream):
            self._body()
        torch.cuda.current_stream(dev).wait_stream(self.stream)

    def capture(self, pool=None):
        """Capture the iteration.  capture_begin/end directly: torch.cuda.graph()
        would empty the device and pinned-host allocator caches on every
        (re)capture.  `pool` = the previous graph's memory pool: most large
        buffers (volumes, k-space) do not depend on the Gaussian count and
        are reused; the previous graph is never replayed again."""
        dev = self.p.positions.device
        self.graph = torch.cuda.CUDAGraph()
        self.stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(self.stream):
            if pool is None:
                self.graph.capture_begin()
            else:
                self.graph.capture_begin(pool=pool)
            try:
                self._body()
            finally:
                self.graph.capture_end()
        torch.cuda.current_stream(dev).wait_stream(self.stream)

    def replay(self):
        self.graph.replay()

    def overflowed(self) -> bool:
        torch.cuda.current_stream(self.p.positions.device).synchronize()
        return bool(int(self.flags_host[0]) & 1)

    @torch.no_grad()
    def undo(self):
        torch._foreach_copy_(self.live, self.snap)
        if not self.had_state:
            for t in self.p.tensors():
                self.opt.state.pop(t, None)


def fit_graph(case: MRICase, init: GaussianSet, cfg: FitConfig, device="cuda:0", stop_nmse: Optional[float] = None,
              log: Optional[Callable] = None, eval_ssim: bool = True, capacity_margin: float = 1.25,
              stats: Optional[Dict] = None) -> FitResult:
    """`fit` with every iteration replayed from a CUDA graph.  The graph is
    (re)captured after the first iteration and after every density-control
    change; the voxelizer inside runs on a fixed pair capacity (the current
    pair count x `capacity_margin`), and an overflowing iteration is undone
    and re-run after re-sizing."""
    from .tile_voxelizer import TileVoxelizer

    dev = torch.device(device)
    shape = tuple(case.ground_truth.shape)
    vox = TileVoxelizer(shape, tile_size=cfg.tile_size, device=str(dev), deterministic=cfg.deterministic)
    S = case.sensitivity_maps.to(dev).to(torch.complex64).contiguous()
    mask = case.mask.to(dev).float().contiguous()
    ku = case.kspace_undersampled.to(dev).to(torch.complex64).contiguous()
    gt = case.ground_truth.to(dev)
    mask_c = mask.unsqueeze(0)
    p = GaussianParams(init, dev)
    lrs = [torch.tensor(v, device=dev) for v in (cfg.position_lr, cfg.scale_lr, cfg.rotation_lr, cfg.density_lr,
                                                   cfg.density_lr)]
    opt = make_optimizer(p, cfg, lrs=lrs, capturable=True)
    gen = torch.Generator(device=dev).manual_seed(cfg.seed)
    res = FitResult(params=p)
    st = stats if stats is not None else {}
    st.setdefault("captures", 0)
    st.setdefault("overflows", 0)
    st.setdefault("capture_seconds", 0.0)

    def new_step():
        cap = int(vox.count_pairs(p.positions.detach(), torch.exp(p.log_scales.detach())) * capacity_margin) + 4096
        return _GraphedStep(p, opt, vox, S, mask_c, ku, cfg, cap)

    step = None
    prev_graph = None  # kept alive until the next capture has reused its pool
    wall = 0.0
    _sync(dev)
    t0 = time.perf_counter()
    for it in range(cfg.iterations):
        while True:
            if step is None or step.graph is None:
                tc = time.perf_counter()
                if step is None:
                    step = new_step()
                step.eager()
                if step.overflowed():
                    step.undo()
                    st["overflows"] += 1
                    step = _GraphedStep(p, opt, vox, S, mask_c, ku, cfg, step.capacity * 2)
                    continue
                step.capture(pool=prev_graph.pool() if prev_graph is not None else None)
                prev_graph = step.graph
                st["captures"] += 1
                st["capture_seconds"] += time.perf_counter() - tc
                break
            step.replay()
            if not step.overflowed():
                break
            step.undo()
            st["overflows"] += 1
            step = _GraphedStep(p, opt, vox, S, mask_c, ku, cfg, step.capacity * 2)
            step.graph = None
        skip_sched = False
        if cfg.densify_from <= it <= cfg.densify_until and it % cfg.densify_every == 0:
            holder = [opt]
            cur_lrs = [g["lr"] for g in opt.param_groups]

            def rebuild(keep, holder=holder, cur_lrs=cur_lrs):
                new_opt = make_optimizer(p, cfg, cur_lrs, capturable=True)
                transplant(holder[0], new_opt, keep, p.n)
                holder[0] = new_opt

            if density_control(p, step.pos_grad, cfg, gen, rebuild):
                opt = holder[0]
                skip_sched = True
                step = None
        if not skip_sched:
            torch._foreach_mul_(lrs, cfg.gamma)
        last = it == cfg.iterations - 1
        if (it % cfg.eval_every == 0) or last:
            _sync(dev)
            wall += time.perf_counter() - t0
            with torch.no_grad():
                v = vox(p.positions, torch.exp(p.log_scales), p.rotations, torch.complex(p.density_r, p.density_i))
                rec = hard_data_consistency(v, S, mask, ku)
                e = nmse(rec, gt)
            lossv = float(step.loss) if step is not None else float("nan")
            row = {"iteration": it, "loss": lossv, "nmse": e, "n_points": p.n, "seconds": wall}
            res.history.append(row)
            if log:
                log(row)
            done = stop_nmse is not None and e <= stop_nmse
            if last or done:
                res.final_nmse = e
                res.final_psnr = psnr(rec, gt)
                if eval_ssim:
                    res.final_ssim = ssim3d(rec, gt)
                if done:
                    break
            _sync(dev)
            t0 = time.perf_counter()
    res.seconds = wall
    res.params = p
    return res
