"""The multi-process path of bench.py on the CPU: two ranks over gloo (one
process each, rendezvous on 127.0.0.1) run the weak-scaling reduction with
different per-rank device times; both must report the slowest rank's time and
the whole-job throughput world_size * classes * steps / that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench
        my_ms = [12.0, 20.0][rank]  # rank 1 is the slow one
        value, total = bench.weak_scaling_value(my_ms, 6545, 10, ws, "cpu")
        out[rank] = (value, total)
    finally:
        dist.destroy_process_group()


def test_weak_scaling_value_two_ranks():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for rank in (0, 1):
        value, total = res[rank]
        assert total == 20.0
        assert value == pytest.approx(2 * 6545 * 10 / 20e-3)


def test_weak_scaling_value_single_rank():
    import bench
    value, total = bench.weak_scaling_value(5.0, 100, 4, 1, "cpu")
    assert total == 5.0 and value == pytest.approx(100 * 4 / 5e-3)
