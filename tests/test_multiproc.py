"""The multi-process plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1 take the
slowest rank's time (max over ranks), as the GPU runs do over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, world)
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 15.0, 1: 15.0}


def test_single_rank_is_identity():
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5


if __name__ == "__main__":
    pytest.main([__file__])
