"""Generate the golden fixtures in this folder by running the REFERENCE's own
PyTorch tile voxelizer (3DGS/3dgsVC/gaussian/tile_voxelizer.py, CPU path:
``TileVoxelizer(use_cuda=False)`` -> ``build_tile_pairs`` (:87-162) ->
``_tile_forward_pytorch`` (:210-244) -> torch autograd).

The reference has no tests, fixtures or known-answer vectors of its own, so
these fixtures are what pins the oracle to the reference.  They are produced
once, in a checkout that has the reference source next to it, and committed:

    python tests/golden/make_golden.py --reference /path/to/GS_TMI

The fixtures hold, per case: the inputs, the reference's center_vox and
radius_vox (captured at the build_tile_pairs call), its tile lists (each
tile's list put in ascending-gid order, the order a stable sort gives; the
reference's torch.argsort is not stable), the complex64 volume and the
gradients for positions, scales, rotations and density (real, imag) under a
seeded complex upstream gradient.  The 64^3 / N=20,000 case stores hashes,
norms and seeded subsets instead of full arrays.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gs_tmi_b200 import synthetic  # noqa: E402


def _canonical(tile_ranges, pair_ids):
    tr = tile_ranges.cpu().numpy().astype(np.int32)
    pid = pair_ids.cpu().numpy().astype(np.int32).copy()
    for s, e in tr:
        if e > s:
            pid[s:e] = np.sort(pid[s:e])
    return tr, pid


def run_reference(tv_mod, gs: synthetic.GaussianSet, shape, ts, gv):
    captured = {}
    original = tv_mod.build_tile_pairs

    def recorder(center_vox, radius_vox, volume_shape, tile_size):
        captured["center"] = center_vox.detach().clone()
        captured["radius"] = radius_vox.detach().clone()
        out = original(center_vox, radius_vox, volume_shape, tile_size)
        captured["bins"] = out
        return out

    tv_mod.build_tile_pairs = recorder
    try:
        vox = tv_mod.TileVoxelizer(tuple(shape), tile_size=ts, use_cuda=False, device="cpu")
        pos = gs.positions.clone().requires_grad_(True)
        scl = gs.scales.clone().requires_grad_(True)
        rot = gs.rotations.clone().requires_grad_(True)
        dr = gs.density_r.clone().requires_grad_(True)
        di = gs.density_i.clone().requires_grad_(True)
        vol = vox(pos, scl, rot, torch.complex(dr, di))
        loss = (vol.real * gv.real + vol.imag * gv.imag).sum()
        loss.backward()
    finally:
        tv_mod.build_tile_pairs = original
    tr, pid = _canonical(*captured["bins"])
    grads = {k: t.grad.detach().numpy().copy() for k, t in
             (("g_pos", pos), ("g_scl", scl), ("g_rot", rot), ("g_dr", dr), ("g_di", di))}
    return dict(center=captured["center"].numpy(), radius=captured["radius"].numpy(), tile_ranges=tr,
                pair_ids=pid, vol=vol.detach().numpy().astype(np.complex64), **grads)


def small_cases():
    cases = []
    shape = (20, 12, 16)
    gs = synthetic.concat(synthetic.random_gaussians(200, shape, seed=11),
                          synthetic.edge_case_gaussians(shape, seed=12))
    cases.append(("edge_20x12x16_ts8", shape, 8, gs, 13))
    shape = (16, 16, 16)
    cases.append(("cube_16_ts4", shape, 4, synthetic.random_gaussians(300, shape, seed=21), 22))
    shape = (24, 16, 12)
    gs = synthetic.random_gaussians(150, shape, seed=31, log_scale_mean_vox=float(np.log(2.5)),
                                    log_scale_std=0.6)
    cases.append(("aniso_24x16x12_ts8", shape, 8, gs, 32))
    shape = (13, 11, 9)
    cases.append(("odd_13x11x9_ts5", shape, 5, synthetic.random_gaussians(80, shape, seed=41), 42))
    shape = (32, 32, 32)
    cases.append(("cube_32_ts8", shape, 8, synthetic.random_gaussians(1000, shape, seed=51), 52))
    return cases


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout")
    ap.add_argument("--skip-large", action="store_true")
    args = ap.parse_args()
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(args.reference, "3DGS", "3dgsVC"))
    import gaussian.tile_voxelizer as tv_mod  # the reference module

    torch.set_num_threads(min(8, os.cpu_count() or 1))
    for name, shape, ts, gs, gseed in small_cases():
        gv = synthetic.upstream_grad(shape, seed=gseed)
        ref = run_reference(tv_mod, gs, shape, ts, gv)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"), shape=np.array(shape, np.int32), tile_size=np.int32(ts),
            positions=gs.positions.numpy(), scales=gs.scales.numpy(), rotations=gs.rotations.numpy(),
            density_r=gs.density_r.numpy(), density_i=gs.density_i.numpy(),
            grad_vol=gv.numpy().astype(np.complex64), **ref)
        print(f"{name}: pairs={ref['pair_ids'].size}")

    if args.skip_large:
        return
    shape, ts, n = (64, 64, 64), 8, 20000
    gs = synthetic.random_gaussians(n, shape, seed=0)
    gv = synthetic.upstream_grad(shape, seed=1)
    ref = run_reference(tv_mod, gs, shape, ts, gv)
    rng = np.random.default_rng(1234)
    vidx = rng.choice(int(np.prod(shape)), 4096, replace=False).astype(np.int64)
    gidx = rng.choice(n, 1024, replace=False).astype(np.int64)
    out = dict(
        shape=np.array(shape, np.int32), tile_size=np.int32(ts), n=np.int64(n),
        inputs_sha=np.array(sha(np.concatenate([t.numpy().reshape(-1) for t in gs.tensors()]))),
        grad_vol_sha=np.array(sha(gv.numpy().astype(np.complex64))),
        center_sha=np.array(sha(ref["center"])), radius_sha=np.array(sha(ref["radius"])),
        tile_ranges_sha=np.array(sha(ref["tile_ranges"])), pair_ids_sha=np.array(sha(ref["pair_ids"])),
        n_pairs=np.int64(ref["pair_ids"].size), tile_ranges=ref["tile_ranges"],
        vol_norm=np.float64(np.linalg.norm(ref["vol"].astype(np.complex128))),
        vol_idx=vidx, vol_sub=ref["vol"].reshape(-1)[vidx], g_idx=gidx,
    )
    for k in ("g_pos", "g_scl", "g_rot", "g_dr", "g_di"):
        out[k + "_norm"] = np.float64(np.linalg.norm(ref[k].astype(np.float64)))
        out[k + "_sub"] = ref[k][gidx]
    np.savez_compressed(os.path.join(HERE, "cfg_64cube_n20000.npz"), **out)
    print(f"64^3 N=20000: pairs={ref['pair_ids'].size}")


if __name__ == "__main__":
    main()
