"""The drop-in, run inside the reference's own trainer: GaussianTrainer
(V/trainers/trainer.py, unchanged, staged into baseline/_ref by
oracle/build_ref.py) on the seeded 128x128x96, 8-coil, R=6 Poisson-disc
acquisition with 50,000 intensity-seeded Gaussians, once with this build's
TileVoxelizer rebound as gaussian.TileVoxelizer and once with the
reference's TileVoxelizer on its own CUDA extension.  Same seed, same data,
same config (the reference's default.yaml with the data paths, the point
count and the iteration budget set).

Bars over the first 50 iterations: the hard-data-consistency NMSE of every
evaluation (every 10 iterations, the trainer's own evaluate()) within 0.1%,
and the total loss of every iteration within 0.5%.  A second run with the
reference's extension gives the reference's own run-to-run scatter (its
backward sums FP32 atomics in a different order each run), reported beside
the two builds' difference.

Set GSV_REPORT_DIR to write both trajectories as JSON."""
import json
import os

import pytest

from tests import reference_trainer as RT

pytestmark = pytest.mark.gpu

ITERS, EVAL_EVERY = 50, 10


@pytest.mark.skipif(not RT.available(), reason="reference package not staged (oracle/build_ref.py)")
def test_reference_trainer_with_this_voxelizer(cuda_device, tmp_path):
    from gs_tmi_b200 import synthetic
    from oracle.ref_cuda import REF

    if REF is None:
        pytest.skip("reference extension not built (oracle/build_ref.py)")
    shape = (128, 128, 96)
    case = synthetic.mri_case(shape, n_coils=8, accel=6.0, calib=24, seed=0, mask_kind="poisson")
    files = RT.write_case(case, str(tmp_path / "data"))
    runs = {}
    for key, vox in (("reference_cuda", "reference_cuda"), ("this_build", "this_build"),
                     ("reference_cuda_rerun", "reference_cuda")):
        runs[key] = RT.run(vox, files, str(tmp_path / key), accel=6, iterations=ITERS, eval_every=EVAL_EVERY,
                           num_points=50_000, device=str(cuda_device))
    a, b, c = runs["this_build"], runs["reference_cuda"], runs["reference_cuda_rerun"]
    assert a["backend"] == "tile_cuda" and b["backend"] == "tile_cuda"
    loss_rel = [abs(x / y - 1) for x, y in zip(a["losses"], b["losses"])]
    nmse_rel = [abs(x["nmse"] / y["nmse"] - 1) for x, y in zip(a["evals"], b["evals"])]
    self_loss = [abs(x / y - 1) for x, y in zip(c["losses"], b["losses"])]
    self_nmse = [abs(x["nmse"] / y["nmse"] - 1) for x, y in zip(c["evals"], b["evals"])]
    report = {"iterations": ITERS, "eval_every": EVAL_EVERY, "max_loss_rel_diff": max(loss_rel),
              "max_nmse_rel_diff": max(nmse_rel), "reference_rerun_max_loss_rel_diff": max(self_loss),
              "reference_rerun_max_nmse_rel_diff": max(self_nmse), "runs": runs}
    out = os.environ.get("GSV_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "reference_trainer.json"), "w") as f:
            json.dump(report, f, indent=1, default=float)
    print(json.dumps({k: v for k, v in report.items() if k != "runs"}),
          {k: (v["seconds"], v["evals"][-1]) for k, v in runs.items()})
    assert len(a["losses"]) == len(b["losses"]) == ITERS
    assert len(a["evals"]) == len(b["evals"]) >= ITERS // EVAL_EVERY
    assert max(nmse_rel) < 1e-3
    assert max(loss_rel) < 5e-3
