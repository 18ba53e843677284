"""Replica ensembles over ranks: two gloo processes on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from cvfes_b200.cases import TubeCase, build_mesh
from cvfes_b200.replicas import SEED_STRIDE, max_over_ranks, rank_case, sum_over_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = rank_case(TubeCase("rep", 8, 6, 1.0, n_samples=2), rank)
        mesh = build_mesh(case, cache=False)
        ms = 10.0 + rank          # rank 1 is the slow one
        work = 2 * (rank + 1)     # samples x steps done by this rank
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), elmE=mesh.elmE,
                 slowest=max_over_ranks(ms), total=sum_over_ranks(work),
                 seed=case.seed_E)
    finally:
        dist.destroy_process_group()


def test_two_ranks_draw_different_ensembles_and_reduce_on_the_host(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    r0, r1 = (np.load(tmp_path / f"r{r}.npz") for r in range(world))
    assert int(r1["seed"]) - int(r0["seed"]) == SEED_STRIDE
    assert not np.array_equal(r0["elmE"], r1["elmE"])       # independent material samples
    assert float(r0["slowest"]) == float(r1["slowest"]) == 11.0
    assert float(r0["total"]) == float(r1["total"]) == 6.0


def test_single_process_reductions_are_the_identity():
    assert max_over_ranks(3.5) == 3.5 and sum_over_ranks(2.0) == 2.0
