"""Instance sharding across ranks (host logic; gloo process group on CPU).

The ensemble workload splits its instances over ranks with a deterministic
longest-processing-time rule; every rank computes the split on its own, so
the tests check that two real ranks agree, cover every instance once, and
that the max-over-ranks timing reduction works.
"""
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest

from pfem2_b200 import sharding


def _costs(n=64, seed=2):
    rng = np.random.default_rng(seed)
    return list(np.exp(rng.uniform(np.log(5000), np.log(60000), n)))


def test_lpt_split_covers_and_balances():
    c = _costs()
    for world in (1, 2, 3, 4, 8):
        parts = sharding.lpt_split(c, world)
        assert sorted(i for p in parts for i in p) == list(range(len(c)))
        assert all(p == sorted(p) for p in parts)
        assert sharding.imbalance(c, parts) < 1.1


def test_lpt_split_is_deterministic_with_ties():
    c = [1.0] * 7
    assert sharding.lpt_split(c, 3) == sharding.lpt_split(c, 3)
    assert sharding.lpt_split(c, 3) == [[0, 3, 6], [1, 4], [2, 5]]
    assert sharding.lpt_split([], 2) == [[], []]
    with pytest.raises(ValueError):
        sharding.lpt_split(c, 0)


def test_instance_cost_and_shard():
    specs = [SimpleNamespace(mesh=SimpleNamespace(n_cells=n), q=(5, 5)) for n in (100, 400, 200, 300)]
    assert sharding.instance_cost(specs[0]) == 100 * 26
    idx0, s0 = sharding.shard(specs, 0, 2)
    idx1, s1 = sharding.shard(specs, 1, 2)
    assert sorted(idx0 + idx1) == [0, 1, 2, 3]
    assert [s.mesh.n_cells for s in s0] == [specs[i].mesh.n_cells for i in idx0]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = _costs(n)
        idx = sharding.lpt_split(c, world)[rank]
        ok = sharding.check_split_agrees(idx, n)
        mx = sharding.max_over_ranks(10.0 + rank)
        out.put((rank, ok, mx, idx))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_split():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, 64, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert all(ok for _, ok, _, _ in res)
    assert all(mx == 11.0 for _, _, mx, _ in res)
    assert sorted(res[0][3] + res[1][3]) == list(range(64))
