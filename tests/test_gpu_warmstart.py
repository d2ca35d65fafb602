"""Learned warm start: the MLP's tcgen05 forward/backward against a CPU
reference, training, and what the trained network gains over the
intensity-seeded initialisation.

GSV_WARM_FULL=1 runs the full evaluation (training phantoms at 96^3, held-out
128x128x96 R=6 phantoms, iterations and wall time to the plain method's final
NMSE) and writes $GSV_REPORT_DIR/warmstart_eval.json."""
import json
import math
import os
import time

import pytest
import torch

import gs_tmi_b200
from gs_tmi_b200 import sense, synthetic, warmstart

pytestmark = pytest.mark.gpu


def _cpu_reference(mlp, x, dout):
    """FP64 CPU forward/backward of the same network, with the BF16 roundings
    the GPU path applies to operands (activations, upstream gradients)."""
    bf = lambda t: t.to(torch.bfloat16).double()
    W = [bf(w.detach().cpu()) for w in mlp.params[:3]]
    b = [p.detach().cpu().double() for p in mlp.params[3:]]
    xc = bf(x.cpu())
    c0, c1 = math.sqrt(2 / math.pi), math.sqrt(2 / math.pi) * 0.044715  # GELU, tanh form
    g = lambda z: 0.5 * z * (1 + torch.tanh(z * (c0 + c1 * z * z)))
    gp = lambda z: (0.5 * (1 + torch.tanh(z * (c0 + c1 * z * z)))
                    + 0.5 * z * (1 - torch.tanh(z * (c0 + c1 * z * z)) ** 2) * (c0 + 3 * c1 * z * z))
    z1 = xc @ W[0].t() + b[0]
    y1 = bf(g(z1))
    z2 = y1 @ W[1].t() + b[1]
    y2 = bf(g(z2))
    out = y2 @ W[2].t() + b[2]
    do = bf(dout.cpu())
    dW3 = do.t() @ y2
    dz2 = bf((do @ W[2]) * gp(z2))
    dW2 = dz2.t() @ y1
    dz1 = bf((dz2 @ W[1]) * gp(z1))
    dW1 = dz1.t() @ xc
    return out, [dW1, dW2, dW3, dz1.sum(0), dz2.sum(0), dout.cpu().double().sum(0)]


def rel(a, b):
    return float((a.double().cpu() - b).norm() / b.norm().clamp_min(1e-30))


@pytest.mark.parametrize("B", [1536, 28125, 50000])
def test_mlp_forward_backward_vs_cpu(B, cuda_device):
    """B = 1536: every split-K slice fits the 4-stage ring; 28,125 (a 96^3
    training phantom's seed count, 7 k-tiles per slice) and 50,000 (13 per
    slice): the ring refills its stages, with partial row and K tiles."""
    mlp = warmstart.WarmStartMLP(str(cuda_device), seed=1)
    g = torch.Generator(device=cuda_device).manual_seed(2)
    x = torch.randn(B, 256, device=cuda_device, generator=g).bfloat16()
    dout = torch.randn(B, 16, device=cuda_device, generator=g) / B
    out, cache = mlp.forward(x)
    grads = mlp.backward(cache, dout)
    torch.cuda.synchronize()
    mlp.check_ok()
    ro, rg = _cpu_reference(mlp, x, dout)
    assert rel(out, ro) < 5e-3
    for name, a, b in zip(("dW1", "dW2", "dW3", "db1", "db2", "db3"), grads, rg):
        assert rel(a, b) < 2e-2, name


def test_mlp_regression_training(cuda_device):
    """The MLP's own forward/backward kernels fit a smooth regression target."""
    mlp = warmstart.WarmStartMLP(str(cuda_device), seed=3, lr=2e-3)
    g = torch.Generator(device=cuda_device).manual_seed(4)
    x = torch.randn(8192, 256, device=cuda_device, generator=g)
    proj = torch.randn(256, 16, device=cuda_device, generator=g) / 16
    t = torch.tanh(x @ proj)
    xb = x.bfloat16()
    losses = []
    for i in range(300):
        idx = torch.randint(0, 8192, (2048,), device=cuda_device, generator=g)
        out, cache = mlp.forward(xb[idx])
        diff = out - t[idx]
        losses.append(float((diff * diff).mean()))
        mlp.apply_grads(mlp.backward(cache, 2 * diff / diff.numel()))
    mlp.check_ok()
    assert sum(losses[-20:]) / 20 < 0.25 * sum(losses[:5]) / 5


def _small_warm_setup(device):
    wc = warmstart.WarmConfig(shape=(40, 40, 40), n_coils=4, accel=4.0, calib=12, fit_iterations=300)
    cases = [warmstart.training_case(100 + 10 * s, wc, device=device) for s in range(6)]
    mlp = warmstart.WarmStartMLP(device, seed=0)
    losses = warmstart.train(mlp, cases, steps=1000)
    return wc, mlp, losses


def test_warm_start_gains_over_intensity_seeding(cuda_device):
    """Held-out phantom: the trained network's Gaussians (the warm start's
    seeding: three times the seeds, drawn where the zero-filled image is
    bright) start closer to the target than the intensity-seeded ones and
    stay ahead over the first iterations of the same fit."""
    dev = str(cuda_device)
    wc, mlp, losses = _small_warm_setup(dev)
    assert sum(losses[-20:]) / 20 < 0.8 * sum(losses[:5]) / 5
    case = synthetic.mri_case(wc.shape, n_coils=wc.n_coils, accel=wc.accel, calib=wc.calib, seed=999)
    n = int(round(wc.points_per_voxel * math.prod(wc.shape)))
    plain_init = synthetic.from_image_init(case.zero_filled, n, seed=7)
    warm = warmstart.warm_start(mlp, case, n, wc, seed=7, device=dev)
    gt = case.ground_truth.to(cuda_device)
    vox = gs_tmi_b200.TileVoxelizer(wc.shape, device=dev)
    S, m, ku = (t.to(cuda_device) for t in (case.sensitivity_maps, case.mask, case.kspace_undersampled))
    dc = {}
    for name, gs in (("plain", plain_init.to(cuda_device)), ("warm", warm)):
        v = vox(gs.positions, gs.scales, gs.rotations, torch.complex(gs.density_r, gs.density_i))
        # scored after hard data consistency, as the fits score themselves (the network is
        # trained on the part of the volume that data consistency keeps)
        dc[name] = sense.nmse(sense.hard_data_consistency(v, S.to(torch.complex64), m.float(),
                                                          ku.to(torch.complex64)), gt)
    assert dc["warm"] < 0.85 * dc["plain"]
    cfg = sense.FitConfig(iterations=101, eval_every=50, densify_from=10 ** 9)
    p = sense.fit(case, plain_init, cfg, device=dev, eval_ssim=False)
    w = sense.fit(case, warm, cfg, device=dev, eval_ssim=False)
    assert w.history[0]["nmse"] < p.history[0]["nmse"]
    assert w.history[-1]["nmse"] < p.history[-1]["nmse"]


def _time_to_target_eval(dev, n_train, n_eval, steps, mask_kind="poisson", report_name=None, ablations=3):
    """Train on `n_train` plain fits of 96^3 phantoms (the reference's
    stopping rule picks each fit's best iterate as the target), then time
    warm start and plain method to the plain method's final NMSE on
    `n_eval` held-out 128x128x96, 8-coil, R=6 acquisitions.  The first
    `ablations` acquisitions also time the warm start's seeding without the
    network."""
    wc = warmstart.WarmConfig(mask_kind=mask_kind)
    t0 = time.perf_counter()
    cases = warmstart.training_cases([1000 + 17 * s for s in range(n_train)], wc, device=dev)
    t_data = time.perf_counter() - t0
    n_examples = int(sum(c.features.shape[0] for c in cases))
    mlp = warmstart.WarmStartMLP(dev, seed=0)
    t0 = time.perf_counter()
    losses = warmstart.train(mlp, cases, steps=steps)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del cases
    torch.cuda.empty_cache()
    shape = (128, 128, 96)
    rows = []

    def summary():
        ratios = sorted(r["wall_ratio"] for r in rows if r.get("wall_ratio") is not None)
        return {"mask": mask_kind, "train_phantoms": n_train, "eval_phantoms": n_eval, "train_steps": steps,
                "seed_factor": wc.seed_factor, "seed_mode": wc.seed_mode, "loss": wc.loss,
                "fit_lr_scale": wc.fit_lr_scale,
                "train_examples": n_examples, "data_seconds": t_data,
                "train_seconds": t_train, "first_train_loss": losses[0], "final_train_loss": losses[-1],
                "evaluated": len(rows),
                "median_wall_ratio": ratios[len(ratios) // 2] if ratios else None,
                "reached": sum(r.get("warm_iterations_to_target") is not None for r in rows),
                "warm_starts_lower": sum(r["warm_nmse_at_0"] < r["plain_nmse_at_0"] for r in rows),
                "seeding_alone_reached": sum(r.get("seeded_iterations_to_target") is not None
                                             for r in rows if "seeded_nmse_at_0" in r),
                "eval": rows}

    def write(report):
        out = os.environ.get("GSV_REPORT_DIR")
        if out and report_name:
            os.makedirs(out, exist_ok=True)
            with open(os.path.join(out, report_name), "w") as f:
                json.dump(report, f, indent=1)

    # One untimed pass of each initialisation at the evaluation size, so that costs a process
    # pays once (lazy loading of kernels first used at this size, the caching allocator
    # growing again after the training set was freed) are not charged to the first
    # acquisition's wall time; the plain method's own initialisation is covered the same way.
    warm_case = synthetic.mri_case(shape, n_coils=8, accel=6.0, calib=24, seed=49_999, mask_kind=mask_kind)
    synthetic.from_image_init(warm_case.zero_filled, 50_000, seed=0, device=torch.device(dev))
    synthetic.from_image_init(warm_case.zero_filled, int(round(50_000 * wc.seed_factor)), seed=0,
                              device=torch.device(dev), mode=wc.seed_mode)
    warmstart.warm_init(mlp, warm_case, int(round(50_000 * wc.seed_factor)), seed=0, device=dev, mode=wc.seed_mode)
    torch.cuda.synchronize()
    del warm_case
    for e in range(n_eval):
        case = synthetic.mri_case(shape, n_coils=8, accel=6.0, calib=24, seed=50_000 + e, mask_kind=mask_kind)
        rows.append(dict(warmstart.time_to_target(mlp, case, 50_000, seed=e, device=dev,
                                                  warm_points=int(round(50_000 * wc.seed_factor)),
                                                  warm_mode=wc.seed_mode, warm_schedule=wc.fit_overrides(),
                                                  ablation=e < ablations), phantom=e))
        write(summary())  # the report so far, after every acquisition
    report = summary()
    print(json.dumps({k: v for k, v in report.items() if k != "eval"}), json.dumps(rows))
    return report


def test_time_to_target_small(cuda_device):
    """Reduced config-5 evaluation that every GPU test run performs: 16
    training phantoms, 2 held-out acquisitions on the reference's
    Poisson-disc sampling.  The warm start must reach the plain method's
    final NMSE on both, in at most 0.7x the plain method's wall time (the
    full evaluation's bar is 0.5x); its seeding without the network is timed
    beside it."""
    rep = _time_to_target_eval(str(cuda_device), n_train=16, n_eval=2, steps=1000,
                               report_name="warmstart_time_to_target_small.json", ablations=2)
    assert rep["reached"] == rep["eval_phantoms"]
    assert rep["median_wall_ratio"] <= 0.7


@pytest.mark.skipif(os.environ.get("GSV_WARM_FULL") != "1", reason="set GSV_WARM_FULL=1")
def test_full_time_to_nmse(cuda_device):
    """Config 5: GSV_WARM_TRAIN_PHANTOMS (default 2000) training phantoms,
    GSV_WARM_EVAL_PHANTOMS (default 50) held-out acquisitions; the median
    warm/plain wall ratio to the plain method's final NMSE must be <= 0.5."""
    rep = _time_to_target_eval(str(cuda_device), n_train=int(os.environ.get("GSV_WARM_TRAIN_PHANTOMS", "2000")),
                               n_eval=int(os.environ.get("GSV_WARM_EVAL_PHANTOMS", "50")),
                               steps=int(os.environ.get("GSV_WARM_STEPS", "6000")),
                               mask_kind=os.environ.get("GSV_WARM_MASK", "poisson"),
                               report_name="warmstart_eval.json")
    assert rep["reached"] == rep["eval_phantoms"]
    assert rep["median_wall_ratio"] <= 0.5
