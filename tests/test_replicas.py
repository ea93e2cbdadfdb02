"""The replica path of bench.py (one process per GPU) on CPU: two gloo ranks
take the maximum of their timings and report the same whole-job throughput;
an ensemble's members shard over the ranks and their force histories come
back in member order from one all-gather."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from ibpm_b200.replicas import job_throughput, max_over_ranks, world as env_world
    ws, r, local = env_world()
    ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
    m = max_over_ranks(ms)
    out.put((rank, ws, r, local, m, job_throughput(ws, 20, 1, m), job_throughput(ws, 20, 64, m)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_and_throughput():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ws, r, local, m, v1, v64 in res:
        assert (ws, r, local) == (2, rank, rank)
        assert m == 150.0                        # the slowest rank's time
        assert v1 == pytest.approx(2 * 20 / 0.150)
        assert v64 == pytest.approx(64 * v1)


def test_single_process_needs_no_group():
    from ibpm_b200.replicas import job_throughput, max_over_ranks
    assert max_over_ranks(12.5) == 12.5
    assert job_throughput(1, 200, 1, 250.0) == pytest.approx(800.0)
    with pytest.raises(ValueError):
        job_throughput(1, 1, 1, 0.0)


def _ensemble_rank(rank, world, port, out):
    import numpy as np
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from ibpm_b200.replicas import gather_histories, shard
    units, K = 7, 5
    mine = shard(units, world, rank)
    # member m's "force history": K steps of (m, step)
    local = np.array([[[m, k] for k in range(K)] for m in mine], dtype=float)
    full = gather_histories(local, units)
    out.put((rank, mine, full.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_members_shard_and_gather_in_member_order():
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ensemble_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == [0, 2, 4, 6] and res[1][1] == [1, 3, 5]
    want = np.array([[[m, k] for k in range(5)] for m in range(7)], dtype=float)
    for _, _, full in res:
        assert np.array_equal(np.array(full), want)


def test_shard_covers_every_member_once():
    from ibpm_b200.replicas import shard
    for units in (1, 7, 64):
        for ws in (1, 2, 3, 8):
            parts = [shard(units, ws, r) for r in range(ws)]
            assert sorted(sum(parts, [])) == list(range(units))
    with pytest.raises(ValueError):
        shard(4, 2, 2)
