"""Multi-rank island logic on CPU: world_size 2 (and 3) gloo process groups.

The distributed migration (in-rank oracle migration + the cross-rank hop)
must equal the single-process oracle migration over all islands of all
ranks; global_best, broadcast_row, max_over_ranks and shard are checked on
the same groups.  No GPU is involved: the in-rank step is the oracle's.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _oracle_local(pop, fit, NI, k):
    import oracle
    p2, f2, order = oracle.island_migrate(pop.numpy(), fit.numpy(), NI, k)
    pop.copy_(torch.from_numpy(p2))
    fit.copy_(torch.from_numpy(f2))
    return torch.from_numpy(order)


def _worker(rank, world, port, glob_pop, glob_fit, NIl, k, out_q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from sidon_b200 import islands
        P = glob_pop.shape[0] // world
        pop = torch.from_numpy(glob_pop[rank * P:(rank + 1) * P].copy())
        fit = torch.from_numpy(glob_fit[rank * P:(rank + 1) * P].copy())
        islands.migrate_across_ranks(pop, fit, NIl, k, local_migrate=_oracle_local)
        best = islands.global_best(fit)
        row = pop[best[2]].clone() if best[1] == rank else torch.zeros(pop.shape[1])
        islands.broadcast_row(row, best[1])
        slow = islands.max_over_ranks(10.0 + rank)
        out_q.put((rank, pop.numpy(), fit.numpy(), best, row.numpy(), slow))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,NIl,k", [(2, 2, 1), (2, 3, 2), (3, 2, 1)])
def test_distributed_migration_equals_global_oracle(orc, world, NIl, k):
    rng = np.random.default_rng(world * 10 + NIl)
    PI, n = 6, 5
    P = world * NIl * PI
    glob_pop = rng.uniform(0, 1, (P, n)).astype(np.float32)
    glob_fit = rng.uniform(1.4, 1.8, P)
    glob_fit[3] = np.nan
    glob_fit[7] = glob_fit[8]
    want_pop, want_fit, _ = orc.island_migrate(glob_pop, glob_fit, world * NIl, k)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, glob_pop, glob_fit, NIl, k, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got_pop = np.concatenate([r[1] for r in res])
    got_fit = np.concatenate([r[2] for r in res])
    np.testing.assert_array_equal(got_pop, want_pop)
    np.testing.assert_array_equal(got_fit, want_fit)
    f = np.where(np.isnan(got_fit), np.inf, got_fit)
    g = int(np.argmin(f))
    for r in res:
        F, brank, bidx = r[3]
        assert F == f[g] and brank * (P // world) + bidx == g
        np.testing.assert_array_equal(r[4], got_pop[g])
        assert r[5] == 10.0 + world - 1


def test_shard_covers_everything():
    from sidon_b200 import islands
    for P in (0, 1, 7, 1024):
        for W in (1, 2, 3, 8):
            spans = [islands.shard(P, r, W) for r in range(W)]
            assert spans[0][0] == 0 and spans[-1][1] == P
            assert all(spans[i][1] == spans[i + 1][0] for i in range(W - 1))
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1


def test_single_process_paths_need_no_group(orc):
    """Without a process group (one GPU) the helpers reduce to local work."""
    from sidon_b200 import islands
    rng = np.random.default_rng(1)
    pop = torch.from_numpy(rng.uniform(0, 1, (12, 4)).astype(np.float32))
    fit = torch.from_numpy(rng.uniform(1, 2, 12))
    want_pop, want_fit, _ = orc.island_migrate(pop.numpy(), fit.numpy(), 3, 1)
    islands.migrate_across_ranks(pop, fit, 3, 1, local_migrate=_oracle_local)
    np.testing.assert_array_equal(pop.numpy(), want_pop)
    F, r, i = islands.global_best(fit)
    assert r == 0 and F == float(np.min(fit.numpy())) and fit[i].item() == F
    assert islands.max_over_ranks(3.5) == 3.5
