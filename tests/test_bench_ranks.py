"""The replica bookkeeping of bench.py under several ranks, on the CPU: two gloo processes stand in for two
GPUs (the collectives are the same calls; only the backend and the tensors' device differ)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: step 1.0 + r ms, 1000·(r + 1) particles, SOR launch 0.002·(r + 1) ms, e2e rate 100 − r
        ms, particles, sor = bench.reduce_ranks(1.0 + rank, 1000.0 * (rank + 1), 0.002 * (rank + 1), 'cpu')
        e2e = bench.reduce_e2e(100.0 - rank, world, 'cpu')
        out[rank] = (ms, particles, sor, e2e)
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_time_and_all_work():
    world, port = 2, _free_port()
    mgr = mp.get_context('spawn').Manager()
    out = mgr.dict()
    ctx = mp.get_context('spawn')
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, 'a rank did not finish'
    assert all(p.exitcode == 0 for p in procs)
    for r in range(world):
        ms, particles, sor, e2e = out[r]
        assert ms == 2.0                      # max over ranks
        assert particles == 3000.0            # sum over ranks
        assert sor == pytest.approx(0.004)    # max over ranks
        assert e2e == 99.0 * world            # slowest rank × ranks


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun the CPU reference arm prints one line from rank 0; other ranks exit at once."""
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    args = argparse.Namespace(steps=1, warmup=0, gpus=2)
    assert bench.run_reference(args, 1) is None
    assert capsys.readouterr().out == ''
