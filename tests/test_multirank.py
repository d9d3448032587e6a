"""The multi-GPU form of bench.py is replicas only (rays and views are
independent; no data-path collective): each rank renders the whole workload
on its GPU, the ranks' device times are combined by a max over ranks, and the
whole-job throughput counts every replica's rays.  This checks that host
logic with two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as td

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world,
                          timeout=datetime.timedelta(seconds=60))
    try:
        mine = [10.0 + rank, 5.0 - rank, 7.0 * (rank + 1)]
        out = bench.max_over_ranks(mine, td, "cpu")
        q.put((rank, out.tolist()))
    finally:
        td.destroy_process_group()


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [11.0, 5.0, 14.0]


def test_whole_job_value_counts_every_replica():
    import bench

    # 1e6 rays per replica step, 4 replicas, 5 steps over 100 ms -> 200 Mrays/s
    assert np.isclose(bench.whole_job_mrays(1_000_000, 4, 5, 100.0), 200.0)
    assert np.array_equal(bench.max_over_ranks([1.0, 2.0], None, "cpu"), [1.0, 2.0])
