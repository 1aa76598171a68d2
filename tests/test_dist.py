"""The multi-rank bookkeeping of the batched workloads, on two gloo ranks on
the host: the whole-job rate is all ranks' units over the slowest rank's
time, every rank gets the same totals (so ranks take the same decisions),
and every rank's query shard is its own."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from devil_ray_b200 import dist as D
    from devil_ray_b200 import meshgen
    r, w, local = D.dist_info()
    assert (r, w, local) == (rank, world, rank)
    pg = D.init("gloo", timeout_s=60)
    assert pg is not None
    slowest = D.max_over_ranks(pg, 1.0 + 1.5 * rank)
    total = D.sum_over_ranks(pg, 3 + rank)
    rate = D.job_rate(pg, units=100 * (rank + 1), ms=10.0 * (rank + 1))
    q = meshgen.uniform_queries(1000, D.shard_seed(rank))
    np.save(os.path.join(out_dir, f"rank{rank}.npy"),
            np.array([slowest, total, rate, float(q[0, 0]), float(q[0, 1])]))
    pg.barrier()
    pg.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    a = np.load(tmp_path / "rank0.npy")
    b = np.load(tmp_path / "rank1.npy")
    for v in (a, b):
        assert v[0] == pytest.approx(2.5)          # slowest rank's time
        assert v[1] == 7                            # 3 + 4
        assert v[2] == pytest.approx(300 / 0.020)   # (100 + 200) units / 20 ms
    assert not np.array_equal(a[3:], b[3:])         # each rank its own queries


def test_single_process_needs_no_group():
    from devil_ray_b200 import dist as D
    assert D.max_over_ranks(None, 4.0) == 4.0
    assert D.sum_over_ranks(None, 9) == 9
    assert D.job_rate(None, 1000, 2.0) == pytest.approx(5e5)
