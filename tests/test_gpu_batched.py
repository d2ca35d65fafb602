"""Batched persistent launches: several volumes of uneven size voxelized by
one forward launch and one backward launch must give exactly what the
single-volume path gives, and the fixed-size batch must replay from a CUDA
graph."""
import numpy as np
import pytest
import torch

import gs_tmi_b200
from gs_tmi_b200 import batched, synthetic
from oracle import oracle as O
from tests.helpers import FWD_TOL, GRAD_TOL, rel

pytestmark = pytest.mark.gpu

SHAPES = [(40, 40, 40), (24, 32, 16), (48, 40, 56), (16, 16, 16), (33, 21, 27)]


def _sets(dev):
    out = []
    for i, s in enumerate(SHAPES):
        gs = synthetic.random_gaussians(400 + 300 * i, s, seed=200 + i)
        out.append(gs)
    return out


def _grads(shapes, seed):
    return [synthetic.upstream_grad(s, seed=seed + i) for i, s in enumerate(shapes)]


@pytest.mark.parametrize("deterministic", [True, False])
def test_batched_matches_single_volume(deterministic, cuda_device):
    dev = cuda_device
    sets = _sets(dev)
    gvs = [g.to(dev) for g in _grads(SHAPES, 300)]
    bv = batched.BatchedVoxelizer(SHAPES, device=str(dev), deterministic=deterministic)
    leaves = [[t.to(dev).requires_grad_(True) for t in gs.tensors()] for gs in sets]
    vols = bv([(p[0], p[1], p[2], torch.complex(p[3], p[4])) for p in leaves])
    loss = sum((v.real * g.real + v.imag * g.imag).sum() for v, g in zip(vols, gvs))
    loss.backward()
    for i, (gs, s) in enumerate(zip(sets, SHAPES)):
        ref_leaves = [t.to(dev).requires_grad_(True) for t in gs.tensors()]
        ref = gs_tmi_b200.voxelize(*ref_leaves, s, 8, deterministic=deterministic)
        (ref.real * gvs[i].real + ref.imag * gvs[i].imag).sum().backward()
        assert torch.equal(vols[i].detach(), ref.detach())  # same per-tile code, same order
        for a, b in zip(leaves[i], ref_leaves):
            if deterministic:
                assert torch.equal(a.grad, b.grad)
            else:
                assert rel(a.grad.cpu().numpy(), b.grad.cpu().numpy()) < 1e-5
    # and against the FP64 oracle for one of the volumes
    p = tuple(t.numpy() for t in sets[2].tensors())
    c, r, _ = O.preprocess_f32(*p[:3], SHAPES[2])
    tr, pid = O.build_tile_pairs(c, r, SHAPES[2], 8)
    assert rel(vols[2].detach().cpu().numpy(), O.forward(p, SHAPES[2], 8, tr, pid)[0]) < FWD_TOL
    og = O.backward(p, SHAPES[2], 8, tr, pid, gvs[2].cpu().numpy())
    for a, b in zip(leaves[2], og):
        assert rel(a.grad.cpu().numpy(), b) < GRAD_TOL


def test_static_batch_graph_replay(cuda_device):
    dev = cuda_device
    sets = _sets(dev)
    caps = []
    for gs, s in zip(sets, SHAPES):
        p = tuple(t.numpy() for t in gs.tensors())
        c, r, _ = O.preprocess_f32(*p[:3], s)
        caps.append(int(O.build_tile_pairs(c, r, s, 8)[1].size * 1.2) + 64)
    sb = batched.StaticBatch(SHAPES, [gs.n for gs in sets], caps, device=str(dev), deterministic=True)
    for i, gs in enumerate(sets):
        for dst, src in zip(sb.params[i], gs.tensors()):
            dst.copy_(src.to(dev))
        sb.grad_volumes[i].copy_(synthetic.upstream_grad(SHAPES[i], seed=400 + i).to(dev))
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        sb.bin()
        sb.forward()
        sb.backward()
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize(dev)
    eager_vols = [v.clone() for v in sb.volumes]
    eager_grads = [[g.clone() for g in gg] for gg in sb.grads]
    assert not any(sb.overflowed())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        sb.bin()
        sb.forward()
        sb.backward()
    for v in sb.volumes:
        v.zero_()
    g.replay()
    torch.cuda.synchronize(dev)
    for v, e in zip(sb.volumes, eager_vols):
        assert torch.equal(v, e)
    for gg, ee in zip(sb.grads, eager_grads):
        for a, b in zip(gg, ee):
            assert torch.equal(a, b)


def _recon(dev, cases, inits, caps):
    return batched.BatchedRecon(cases, inits, caps, device=str(dev), deterministic=True)


def test_batched_recon_iteration(cuda_device):
    """A whole batched reconstruction iteration (three volumes with their own
    coils and masks): the per-volume loss equals the fused data term + TV
    of the same volume, and replaying the iteration from a CUDA graph gives
    bitwise the parameters of the eager iterations."""
    from gs_tmi_b200 import sense

    dev = cuda_device
    shapes, ncoils = [(24, 32, 16), (40, 40, 40), (33, 21, 27)], [2, 4, 3]
    cases = [synthetic.mri_case(s, n_coils=c, accel=4.0, calib=6, seed=50 + i, device=dev)
             for i, (s, c) in enumerate(zip(shapes, ncoils))]
    inits = [synthetic.from_image_init(c.zero_filled.cpu(), 600 + 200 * i, seed=60 + i) for i, c in enumerate(cases)]
    caps = []
    for gs, s in zip(inits, shapes):
        p = tuple(t.numpy() for t in gs.tensors())
        c, r, _ = O.preprocess_f32(*p[:3], s)
        caps.append(int(O.build_tile_pairs(c, r, s, 8)[1].size * 2) + 256)
    a, b = _recon(dev, cases, inits, caps), _recon(dev, cases, inits, caps)
    a.step()
    torch.cuda.synchronize(dev)
    for i, (case, vol) in enumerate(zip(cases, a.sb.volumes)):
        want = float(sense.sense_data_term(vol, a.S[i], a.mask[i], a.ku[i])) + 0.1 * float(
            sense.magnitude_tv_fused(vol))
        assert abs(a.losses()[i] - want) <= 1e-5 * abs(want)
    for _ in range(2):
        a.step()
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        b.step()  # eager first step: Adam creates its state
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        b.step()
    g.replay()
    g.replay()
    torch.cuda.synchronize(dev)
    assert not any(a.sb.overflowed()) and not any(b.sb.overflowed())
    for la, lb in zip(a.leaves, b.leaves):
        for x, y in zip(la, lb):
            assert torch.equal(x.detach(), y.detach())
