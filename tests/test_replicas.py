"""The bench's multi-GPU form (one replica per GPU, no data-path exchange) reduces its timings
as the maximum over ranks; this runs that reduction on two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    out[rank] = bench.max_over_ranks(1.5 + rank, "cpu")
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
        assert all(p.exitcode == 0 for p in procs)
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_one_rank_is_its_own_maximum():
    import bench
    assert bench.max_over_ranks(3.25) == 3.25
