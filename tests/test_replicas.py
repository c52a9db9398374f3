"""Multi-GPU semantics of bench.py on CPU: world_size 2 gloo ranks.

The batched ensemble shards by member (independent simulations, no exchange):
N ranks run 64 N members, each on exactly one rank (weak scaling).  A single
simulation does not shard without exchange steps, so N GPUs run N independent
replicas of it.  What must hold across ranks: each member or replica on one
rank with its own seed, every rank takes the same collective steps, and the
reported time is the maximum over ranks.  No GPU is touched here.
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


def _partition_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    mine = bench.rank_members(bench.ENSEMBLE_PER_RANK, rank, world)
    everyone = [None] * world
    dist.all_gather_object(everyone, mine)
    ms = bench.max_over_ranks(20.0 - rank)
    out[rank] = (everyone, ms)
    dist.destroy_process_group()


def test_ensemble_members_partitioned_over_ranks():
    """The batched ensemble shards by member: with N ranks the list has 64 N members and
    every member runs on exactly one rank; rank 0's block is the one-GPU workload."""
    import bench
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_partition_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert out[0][0] == out[1][0]
    blocks = out[0][0]
    flat = [i for b in blocks for i in b]
    assert sorted(flat) == list(range(bench.ENSEMBLE_PER_RANK * world))  # each member exactly once
    assert blocks[0] == list(range(bench.ENSEMBLE_PER_RANK))
    assert out[0][1] == out[1][1] == 20.0
    # a longer member list extends the one-GPU list unchanged
    short, long = bench.ensemble_members(64), bench.ensemble_members(64 * world)
    assert all(a["size_x"] == b["size_x"] and a["ppc"] == b["ppc"] and a["beta"] == b["beta"]
               for a, b in zip(short, long[:64]))


def test_ensemble_cpu_sample_is_bounded():
    import bench
    members = bench.ensemble_members(64)
    idx = bench.cpu_sample(members)
    n = sum(bench.member_particles(members[i]) for i in idx)
    assert idx == list(range(len(idx))) and n >= bench.CPU_SAMPLE_PARTICLES
    assert n - bench.member_particles(members[idx[-1]]) < bench.CPU_SAMPLE_PARTICLES
    assert sum(bench.member_particles(m) for m in members) == 265_764_864


def test_device_index_follows_torch(monkeypatch):
    """Contexts are created on the caller's torch device (one process per GPU under torchrun
    selects it with torch.cuda.set_device(LOCAL_RANK)); without torch, device 0."""
    import sys
    import types
    from spectral_rs_b200.sim import device_index
    fake = types.SimpleNamespace(cuda=types.SimpleNamespace(is_available=lambda: True, current_device=lambda: 3))
    monkeypatch.setitem(sys.modules, "torch", fake)
    assert device_index() == 3
    fake.cuda.is_available = lambda: False
    assert device_index() == 0
    monkeypatch.delitem(sys.modules, "torch")
    assert device_index() == 0
