"""The bench's multi-GPU path on the CPU: replicas only, so the only exchange is the
timing aggregate (max of the device times, sum of the units over ranks), run here
as two gloo ranks; and the reference arm, which works on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        # Rank r took 10 + 5 r ms for 100 + r units.
        results[rank] = bench.aggregate(10.0 + 5 * rank, 100.0 + rank, world, "gloo")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_aggregate_takes_max_time_and_summed_units_over_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        results = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs)
        assert results[0] == (15.0, 201.0)
        assert results[1] == (15.0, 201.0)


def test_aggregate_is_identity_on_one_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.aggregate(12.5, 8.0, 1, None) == (12.5, 8.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
