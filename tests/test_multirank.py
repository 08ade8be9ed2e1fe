"""N > 1 host logic of bench.py on CPU with 2 gloo ranks: replicas each time
their own steps, the job time is the maximum over ranks and the throughput
sums the ranks' work; the reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
        t, tflops = bench.replica_throughput(local_ms, 2.0 * 8192 ** 3, 10, world, "cpu")
        out[rank] = (t, tflops)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_take_max_time_and_sum_work():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    assert out[0] == out[1]
    t, tflops = out[0]
    assert t == 150.0
    assert tflops == pytest.approx(world * 2.0 * 8192 ** 3 * 10 / 0.150 / 1e12)


def test_single_rank_needs_no_process_group():
    import bench
    t, tflops = bench.replica_throughput(50.0, 1e12, 4)
    assert t == 50.0 and tflops == pytest.approx(80.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        n, steps, warmup, gpus = 8192, 1, 0, 2
    bench.run_reference(Args())  # returns at once on rank 1
    assert capsys.readouterr().out == ""
