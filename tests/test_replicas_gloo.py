"""Replica harness of bench.py on CPU ranks (gloo, world size 2): the
job's time is the slowest rank's, the rate counts every rank's units, and
the reference arm runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        times = [10.0 + 5.0 * rank, 3.0 - rank]  # ms per rank: (step total, e2e)
        got = bench.max_over_ranks(times, dist, torch.device("cpu"))
        out[rank] = got + [bench.whole_job_rate(1000, 10, world, got[0])]
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn")
    for r in range(world):
        step, e2e, rate = out[r]
        assert step == 15.0 and e2e == 3.0
        assert rate == 1000 * 10 * world / 15e-3


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_maps_no_product_library():
    """The reference arm builds its seeded inputs without importing the
    product package, so libgsv_b200.so is never mapped in its process."""
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "gs, gv = bench.make_inputs('cube64_n20k', standalone=True); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPPED' if 'libgsv_b200' in maps else 'CLEAN', gs.n, tuple(gv.shape))") % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["CLEAN", "20000", "(64,", "64,", "64)"], r.stdout
