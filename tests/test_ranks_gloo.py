"""The multi-rank timing of bench.py --gpus N on the CPU: two gloo ranks on 127.0.0.1 (the
GPU runs use NCCL with the same calls).  Every rank must get the slowest rank's time, and the
whole-job figure counts the replicas of all ranks."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from dcc import ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ranks.barrier()
        r, w = ranks.world()
        mx = ranks.max_over_ranks(10.0 + 5.0 * rank)
        out.put((r, w, mx, ranks.job_seconds_per_iteration(mx, 4, w)))
        ranks.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    for r, w, mx, sec in res:
        assert w == 2
        assert mx == 15.0
        assert sec == pytest.approx(15.0 / 4 / 1e3 / 2)


def test_single_process_fallbacks():
    from dcc import ranks
    assert ranks.world() == (0, 1)
    assert ranks.max_over_ranks(3.5) == 3.5
    with pytest.raises(ValueError):
        ranks.job_seconds_per_iteration(1.0, 0, 1)
