"""CPU checks of the reference-trainer harness (tests/reference_trainer.py):
the SSIM stand-in equals this package's 3-D SSIM of the same definition,
and the reference's unchanged trainer runs a few iterations on a small
seeded acquisition written as its .mat inputs, with its own PyTorch
voxelizer, on the CPU."""
import numpy as np
import pytest
import torch

from gs_tmi_b200 import sense, synthetic
from tests import reference_trainer as RT


def test_ssim_stand_in_matches_the_published_definition():
    g = np.random.default_rng(0)
    x = g.random((20, 18, 16))
    y = np.abs(x + 0.1 * g.standard_normal(x.shape))  # magnitudes, as both are used
    dr = float(y.max() - y.min())
    a = RT.structural_similarity(x, y, data_range=dr, win_size=7)
    b = sense.ssim3d(torch.from_numpy(x), torch.from_numpy(y), data_range=dr)
    assert abs(a - b) < 1e-12
    assert RT.structural_similarity(y, y, data_range=dr) == pytest.approx(1.0)


@pytest.mark.skipif(not RT.available(), reason="reference package not staged (oracle/build_ref.py)")
def test_reference_trainer_runs_on_cpu(tmp_path):
    shape = (16, 16, 16)
    case = synthetic.mri_case(shape, n_coils=4, accel=4.0, calib=8, seed=3)
    files = RT.write_case(case, str(tmp_path / "data"))
    r = RT.run("reference_cpu", files, str(tmp_path / "out"), accel=4, iterations=4, eval_every=2, num_points=300,
               device="cpu")
    assert r["backend"] == "tile" and len(r["losses"]) == 4
    assert [e["iteration"] for e in r["evals"]] == [0, 2, 3]
    assert all(np.isfinite(r["losses"])) and 0 < r["evals"][-1]["nmse"] < 10
