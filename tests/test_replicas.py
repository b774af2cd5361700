"""Replicas of bench.py on CPU: two gloo ranks solve disjoint seeded cube sets (rank 0 the
configuration's own seed), and the timing is the max over ranks (the multi-GPU path, without
GPUs)."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    import sys

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "cuda-cube-solver_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    from cuda_cube_solver import workloads
    from cuda_cube_solver.device import state_words

    w, r, _ = bench.dist_setup()
    per_rank = 6
    cubes = workloads.uniform_cubes(per_rank, seed=bench.rank_seed(2, r))
    slowest = bench.max_over_ranks(1.0 + r, w, r)
    bench.barrier(w)
    out.put((r, state_words(cubes).tolist(), slowest))
    import torch.distributed as dist

    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    got.sort()
    a, b = got[0][1], got[1][1]
    assert len(a) == len(b) == 6
    assert not {tuple(x) for x in a} & {tuple(x) for x in b}
    import sys

    sys.path.insert(0, str(ROOT / "cuda-cube-solver_b200"))
    from cuda_cube_solver import workloads
    from cuda_cube_solver.device import state_words

    assert a == state_words(workloads.uniform_cubes(6, seed=2)).tolist()
    assert got[0][2] == got[1][2] == 2.0
