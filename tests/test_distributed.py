"""Multi-process host logic of the multi-GPU path, on CPU with gloo
(world size 2): sample sharding reproduces the single-process render of the
oracle (same counter-RNG streams), the frame reduce, LPT scene ownership and
the photon all-gather."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def test_shard_samples_covers_each_sample_once():
    import distributed as D
    for total in (0, 1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                b, k = D.shard_samples(total, world, r, sample_base=5)
                seen += list(range(b, b + k))
            assert seen == list(range(5, 5 + total))
    with pytest.raises(ValueError):
        D.shard_samples(4, 2, 2)


def test_partition_scenes_balances_cost():
    import distributed as D
    rng = np.random.default_rng(0)
    costs = list(np.exp(rng.uniform(np.log(1e4), np.log(2e6), 64)))
    parts = D.partition_scenes(costs, 8)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / 8 + max(costs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    from pathlib import Path
    repo = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(repo / "42-minirt_b200"))
    sys.path.insert(0, str(repo / "oracle"))
    import torch
    import torch.distributed as dist
    import distributed as D
    import oracle
    import scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sc = scenes.make_c0(0, 24, 16, depth=6)
        ro = oracle.Restatement(sc)
        first, count = D.shard_samples(6, world, rank)
        acc, _ = ro.render_counter(77, count, sample_base=first)
        frame = torch.from_numpy(acc.copy())
        D.reduce_frame(frame, dist)
        pos = np.full((rank + 2, 3), float(rank))
        pw = np.full((rank + 2, 3), 10.0 + rank)
        gp, gw = D.allgather_photons(pos, pw, dist)
        q.put((rank, frame.numpy() if rank == 0 else None, gp, gw))
    finally:
        dist.destroy_process_group()


def test_two_rank_sample_sharding_reproduces_single_render():
    import multiprocessing as mp
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    import oracle
    import scenes
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, frame, gp, gw = q.get(timeout=120)
        res[r] = (frame, gp, gw)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sc = scenes.make_c0(0, 24, 16, depth=6)
    single, _ = oracle.Restatement(sc).render_counter(77, 6)
    np.testing.assert_allclose(res[0][0], single, rtol=1e-12, atol=1e-12)
    for r in (0, 1):
        gp, gw = res[r][1], res[r][2]
        assert len(gp) == 2 + 3
        np.testing.assert_array_equal(gp[:2], 0.0)
        np.testing.assert_array_equal(gw[2:], 11.0)


def test_c_abi_shard_samples_matches_host_helper(mrt):
    """mrt_shard_samples (the C host's sharding arithmetic) equals
    distributed.shard_samples; no device needed."""
    import distributed as D
    for total in (0, 1, 7, 64, 1000, 4096):
        for world in (1, 2, 3, 8):
            for r in range(world):
                assert mrt.shard_samples(total, world, r) == D.shard_samples(total, world, r)
    assert mrt.shard_samples(10, 2, 5) == (0, 0)
