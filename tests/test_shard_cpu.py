"""Sharding over ranks (physxcoopa_b200/shard.py), tested as two gloo processes on the CPU.

Each rank computes the same greedy split without communicating, steps only its share (here with
the oracle, the CPU restatement of solve_cloth), and the frame-end all-gather returns every
cloth's bounds and speed in global order, equal to stepping the whole batch in one process.
"""
import os
import sys

import numpy as np
import pytest

from physxcoopa_b200 import shard

HERE = os.path.dirname(os.path.abspath(__file__))
RESULT = np.dtype([("bounds_min", "<f4", 3), ("bounds_max", "<f4", 3), ("max_speed", "<f4")])


def test_partition_is_balanced_disjoint_and_deterministic():
    rng = np.random.default_rng(0)
    costs = [shard.cloth_cost(int(s) ** 2) for s in rng.integers(16, 129, 4096)]
    for n in (1, 2, 3, 8):
        shares = shard.partition(costs, n)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        assert max(loads) - min(loads) <= max(costs)  # LPT bound
        assert shares == shard.partition(costs, n)
    with pytest.raises(ValueError):
        shard.partition(costs, 0)


def _scene():
    sys.path.insert(0, HERE)
    from physxcoopa_b200 import scenes
    return scenes.uneven_batch(n=10, lo=8, hi=24, seed=9)


def _step_and_summarise(sc, idx):
    import _checkers as K
    out = np.zeros(len(idx), RESULT)
    for j, i in enumerate(idx):
        c = sc.cloths[i].copy()
        K.oracle_step_cloth(c, sc.colliders[i], sources=sc.sources[i])
        out[j]["bounds_min"] = c.bounds[:3]
        out[j]["bounds_max"] = c.bounds[3:]
        out[j]["max_speed"] = K.oracle().orc_max_particle_speed(
            __import__("physxcoopa_b200._abi", fromlist=["A"]).ptr(c.particles), len(c.particles))
    return out


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, HERE)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sc = _scene()
        costs = [shard.cloth_cost(len(c.particles)) for c in sc.cloths]
        shares = shard.partition(costs, world)
        local = _step_and_summarise(sc, shares[rank])
        merged = shard.gather_results(local, shares, len(sc.cloths))
        q.put((rank, merged.tobytes()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_their_shares_and_gather_results():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sc = _scene()
    whole = _step_and_summarise(sc, list(range(len(sc.cloths))))
    assert got[0] == got[1] == whole.tobytes()
