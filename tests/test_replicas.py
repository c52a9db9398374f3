"""Multi-GPU semantics of bench.py on CPU: world_size 2 gloo ranks.

The workload does not shard without exchange steps, so N GPUs run N independent
replicas (weak scaling).  What must hold across ranks: each rank gets its own
seed, every rank takes the same collective steps, and the reported time is the
maximum over ranks.  No GPU is touched here.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    seed = bench.rank_seed(2024, rank)
    ms = bench.max_over_ranks(10.0 + 5.0 * rank)  # rank 1 is slower
    value = 1000 * 7 * world / (ms / 1e3)
    dist.barrier()
    out[rank] = (seed, ms, value, bench.WORKLOAD["name"])
    dist.destroy_process_group()


def test_replicas_max_over_ranks():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert out[0][0] != out[1][0]                     # distinct seeds
    assert out[0][1] == out[1][1] == 15.0             # everyone reports the max
    assert out[0][2] == pytest.approx(1000 * 7 * 2 / 0.015)
    assert out[0][3] == out[1][3]


def test_reference_arm_only_rank0_prints(capsys, monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        steps, warmup, gpus = 1, 0, 2
    bench.run_reference(A, dict(bench.WORKLOAD))
    assert capsys.readouterr().out == ""
