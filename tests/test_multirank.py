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


# --- class-range partition (gausslectronitegrate_b200.sharded) --------------------

def test_class_ranges_cover_the_list():
    from gausslectronitegrate_b200.sharded import class_ranges
    for m in (0, 1, 7, 6545):
        for ws in (1, 2, 3, 8):
            r = class_ranges(m, ws)
            assert len(r) == ws and r[0][0] == 0 and r[-1][1] == m
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [hi - lo for lo, hi in r]
            assert max(sizes) - min(sizes) <= 1


def _shard_rank(rank, ws, port, out):
    import numpy as np
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from _common import core, g10
        from gausslectronitegrate_b200.sharded import evaluate_sharded
        from oracle_binding import Oracle

        idx = core()["erida_idx_33"]  # the reference's 33^3 class list (6,545 classes)
        ora = Oracle()
        grid = [(-16, 33)] * 3
        seen = []

        def evaluate(t):  # the CPU checker stands in for the GPU evaluation of a range
            seen.append(t.numel())
            return torch.from_numpy(ora.values("erida", g10(), grid, t.numpy(), 1e-10))

        vals, rng = evaluate_sharded(torch.from_numpy(idx), evaluate, rank, ws)
        out[rank] = (vals.numpy().copy(), rng, seen[0])
    finally:
        dist.destroy_process_group()


def test_sharded_evaluation_two_ranks_reassembles_the_list():
    import numpy as np

    from _common import core, g10
    from oracle_binding import Oracle

    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_shard_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    idx = core()["erida_idx_33"]
    single = Oracle().values("erida", g10(), [(-16, 33)] * 3, idx, 1e-10)
    assert res[0][1] == (0, 3273) and res[1][1] == (3273, 6545)  # contiguous halves of the sorted list
    assert res[0][2] == 3273 and res[1][2] == 3272               # each rank evaluated only its range
    for rank in (0, 1):
        assert np.array_equal(res[rank][0], single)              # every rank holds the whole list, bit for bit


@pytest.mark.gpu
def test_library_ranges_agree_with_the_whole_list():
    # what each rank computes: a contiguous range of the sorted list, planned
    # on its own; the concatenation equals the single evaluation within the
    # parity bar (no collective here: one GPU, one process)
    import numpy as np
    import torch

    import gausslectronitegrate_b200 as gli
    from _common import assert_parity, g10
    from gausslectronitegrate_b200.sharded import class_ranges, library_evaluator

    if gli.lib().gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    for kind, L in (("erida", 33), ("eri", 5)):
        grid = [(-(L // 2), L)] * 3
        whole = getattr(gli, f"compute_sparse_{kind}_gausslet_integrals")(g10(), grid, 1e-10)
        ev = library_evaluator(kind, g10(), grid, 1e-10, "fp64")
        d_idx = torch.from_numpy(whole.indices).cuda()
        parts = [ev(d_idx[lo:hi].contiguous()).cpu().numpy() for lo, hi in class_ranges(whole.indices.size, 3)]
        assert_parity(np.concatenate(parts), whole.values, what=f"{kind} {L}^3 in three ranges")
