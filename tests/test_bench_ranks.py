"""The multi-GPU bench path (replicas, one process per GPU) on CPU: two gloo ranks exercise the
same cross-rank reduction bench.py uses (max of the device time, sum of the work), the replica
seeds, and the reference arm's rule that only rank 0 measures and prints."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r ran for 10 + r ms and traced 100 * (r + 1) rays and 7 paths
        t, (rays, paths) = bench.reduce_over_ranks(10.0 + rank, [100 * (rank + 1), 7], world, device="cpu")
        dist.barrier()
        out[rank] = (t, rays, paths, bench.replica_seed(rank))
    finally:
        dist.destroy_process_group()


def test_reduce_over_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert set(res) == {0, 1}
    for r in (0, 1):
        t, rays, paths, _ = res[r]
        assert t == 11.0            # the slowest rank's time
        assert rays == 300.0        # 100 + 200
        assert paths == 14.0
    assert res[0][3] != res[1][3]   # every replica draws its own samples


def test_single_rank_reduction_is_identity():
    import bench

    assert bench.reduce_over_ranks(5.5, [3, 4], 1) == (5.5, [3.0, 4.0])


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr[-500:]
    assert r.stdout.strip() == ""
