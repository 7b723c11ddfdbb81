"""The multi-rank bookkeeping of bench.py on CPU: two gloo ranks combine their
replicas' figures into the slowest time and the total work."""
import os
import socket

import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    secs, units = bench.combine_over_ranks(1.5 + rank, 100 * (rank + 1), "cpu")
    out[rank] = (secs, units)
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()


def test_two_rank_reduction():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        assert out[0] == out[1] == (2.5, 300.0)


def test_single_rank_is_identity():
    import bench
    assert bench.combine_over_ranks(3.0, 7, "cpu") == (3.0, 7)
