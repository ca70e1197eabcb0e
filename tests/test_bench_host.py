"""Host-side logic of bench.py's reference arm, on the CPU: the reference core
runs on every host core the process may use whatever OMP_NUM_THREADS the
launcher set (torchrun sets 1 per rank), and under torchrun only rank 0 runs
it."""
import os
import sys

from _common import HERE

sys.path.insert(0, os.path.dirname(HERE))
import bench  # noqa: E402


def test_reference_arm_overrides_launcher_thread_count(monkeypatch):
    monkeypatch.setenv("OMP_NUM_THREADS", "1")
    n = bench.use_all_host_threads()
    assert n == len(os.sched_getaffinity(0))
    assert os.environ["OMP_NUM_THREADS"] == str(n)


def test_reference_arm_other_ranks_exit_without_work(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")

    class Args:
        gpus, steps, warmup = 2, 1, 1

    assert bench.run_reference(Args()) == 0
