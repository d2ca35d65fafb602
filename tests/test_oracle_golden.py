"""The CPU oracle against the reference's own outputs (tests/golden/, made by
running the reference PyTorch path; see tests/golden/make_golden.py).

This is what pins the oracle: binning must be bit-exact, forward and
gradients must agree to FP32-vs-FP64 noise away from the cutoff boundary."""
import hashlib

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import GRAD_KEYS, SMALL_CASES, load, params_of, rel

from gs_tmi_b200 import synthetic  # CPU-only module, no library load needed


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", SMALL_CASES)
def test_preprocess_and_binning_bit_exact(name):
    z = load(name)
    shape, ts = tuple(int(x) for x in z["shape"]), int(z["tile_size"])
    c, r, _ = O.preprocess_f32(z["positions"], z["scales"], z["rotations"], shape)
    assert np.array_equal(c.view(np.int32), z["center"].view(np.int32))
    assert np.array_equal(r.view(np.int32), z["radius"].view(np.int32))
    tr, pid = O.build_tile_pairs(c, r, shape, ts)
    assert np.array_equal(tr, z["tile_ranges"])
    assert np.array_equal(pid, z["pair_ids"])


@pytest.mark.parametrize("name", SMALL_CASES)
def test_forward_and_gradients_match_reference(name):
    z = load(name)
    shape, ts = tuple(int(x) for x in z["shape"]), int(z["tile_size"])
    p = params_of(z)
    tr, pid = z["tile_ranges"], z["pair_ids"]
    vol, stats = O.forward(p, shape, ts, tr, pid)
    boundary = O.boundary_voxels(*p[:3], shape, ts, tr, pid, tol=1e-4)
    keep = ~boundary
    # FP32 reference vs FP64 oracle away from cutoff-boundary pairs
    assert rel(vol[keep], z["vol"][keep]) < 2e-6
    # boundary voxels are rare; there the two FP32 op orders may disagree on
    # a pair, costing at most exp(-4.5)|rho| each
    assert boundary.mean() < 0.01
    assert rel(vol, z["vol"]) < 1e-3
    assert stats[0] == O.candidate_evals(tr, shape, ts)
    grads = O.backward(p, shape, ts, tr, pid, z["grad_vol"])
    for k, g in zip(GRAD_KEYS, grads):
        assert rel(g, z[k]) < 2e-5, k


def test_64cube_n20000_reference_pin():
    """64^3, N=20,000 workload: bit-exact binning by hash, volume and
    gradient subsets against the reference."""
    z = load("cfg_64cube_n20000")
    shape, ts, n = (64, 64, 64), 8, 20000
    gs = synthetic.random_gaussians(n, shape, seed=0)
    gv = synthetic.upstream_grad(shape, seed=1).numpy()
    assert sha(np.concatenate([t.numpy().reshape(-1) for t in gs.tensors()])) == str(z["inputs_sha"])
    p = tuple(t.numpy() for t in gs.tensors())
    c, r, _ = O.preprocess_f32(*p[:3], shape)
    assert sha(c) == str(z["center_sha"]) and sha(r) == str(z["radius_sha"])
    tr, pid = O.build_tile_pairs(c, r, shape, ts)
    assert sha(tr) == str(z["tile_ranges_sha"]) and sha(pid) == str(z["pair_ids_sha"])
    assert pid.size == int(z["n_pairs"]) == 292047
    vol, stats = O.forward(p, shape, ts, tr, pid)
    assert stats[0] == 149528064
    boundary = O.boundary_voxels(*p[:3], shape, ts, tr, pid, tol=1e-4).reshape(-1)
    vidx = z["vol_idx"]
    keep = ~boundary[vidx]
    assert rel(vol.reshape(-1)[vidx][keep], z["vol_sub"][keep]) < 2e-6
    assert abs(np.linalg.norm(vol) / float(z["vol_norm"]) - 1) < 1e-5
    grads = O.backward(p, shape, ts, tr, pid, gv)
    gidx = z["g_idx"]
    for k, g in zip(GRAD_KEYS, grads):
        assert rel(g[gidx], z[k + "_sub"]) < 1e-5, k
        assert abs(np.linalg.norm(g) / float(z[k + "_norm"]) - 1) < 1e-5, k
