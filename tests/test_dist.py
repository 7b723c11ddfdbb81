"""The multi-rank bookkeeping of bench.py on CPU: gloo ranks combine their
replicas' figures into the slowest time and the total work, and the
reference arm runs on rank 0 alone (the other ranks exit 0 without work or
output, as the launcher expects of them)."""
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


def _rank(rank, world, port, out, secs=None, units=None):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    s = secs[rank] if secs else 1.5 + rank
    u = units[rank] if units else 100 * (rank + 1)
    out[rank] = bench.combine_over_ranks(s, u, "cpu")
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


def test_four_ranks_uneven():
    """the slowest of four ranks' times and the sum of their units, whatever
    rank holds them"""
    ctx = mp.get_context("spawn")
    secs = [0.25, 3.0, 1.0, 2.5]
    units = [7, 11, 13, 17]
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 4, port, out, secs, units)) for r in range(4)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        assert all(out[r] == (3.0, 48.0) for r in range(4))


def test_reference_arm_runs_on_rank_zero_only():
    """`bench.py --impl reference` under a launcher: a rank other than 0
    returns at once, prints nothing and exits 0"""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
