"""Case sharding of the batched workload across ranks (agal_b200.shard),
on the CPU: LPT packing properties, and a world-size-2 gloo run in which each
rank takes its shard of the bench's 64-case list and the ranks' timing
figures are reduced the way bench.py reduces them (sum of cell updates, max
of device times)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from agal_b200.shard import aggregate, case_cost, lpt_shards, shard_loads


def test_lpt_covers_every_case_once_and_balances():
    costs = [float(c) for c in (96 ** 3 * 4, 32 ** 3, 64 ** 3 * 2, 48 ** 3, 96 ** 3, 32 ** 3 * 4, 64 ** 3, 48 ** 3 * 2)]
    for n in (1, 2, 3, 4, 8):
        sh = lpt_shards(costs, n)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(costs)))
        loads = shard_loads(costs, sh)
        # LPT bound: the slowest rank is within 4/3 of the optimum, which is
        # at least max(mean load, largest case)
        opt_lb = max(sum(costs) / n, max(costs))
        assert max(loads) <= 4.0 / 3.0 * opt_lb + 1e-9


def test_lpt_is_deterministic_and_uses_every_rank():
    costs = [1.0] * 10
    assert lpt_shards(costs, 4) == lpt_shards(costs, 4)
    assert [len(s) for s in lpt_shards(costs, 4)] == [3, 3, 2, 2]
    with pytest.raises(ValueError):
        lpt_shards(costs, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, ws: int, port: int, out):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        import bench
        specs = bench.batched_specs(64, 2024)
        costs = [case_cost(s) for s in specs]
        mine = lpt_shards(costs, ws)[rank]
        # every rank sees the same packing: gather the shards and compare
        got = [None] * ws
        dist.all_gather_object(got, mine)

        def allsum(x):
            t = torch.tensor([x], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            return float(t.item())

        def allmax(x):
            t = torch.tensor([x], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())

        # a rank's "device time" proportional to its load, its updates its cells
        load = sum(costs[i] for i in mine)
        agg = aggregate(updates=load, ms=load / 1e6, allsum=allsum, allmax=allmax)
        out.put((rank, got, agg, sum(costs)))
    finally:
        dist.destroy_process_group()


def test_sharded_batch_over_two_gloo_ranks():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shards0, shards1 = res[0][1], res[1][1]
    assert shards0 == shards1                          # identical packing on every rank
    flat = sorted(i for s in shards0 for i in s)
    assert flat == list(range(64))                     # every case on exactly one rank
    total = res[0][3]
    for _, _, agg, _ in res:
        assert agg["cell_updates"] == pytest.approx(total)
        assert agg["ms"] >= total / 2 / 1e6 - 1e-9     # the slowest rank carries at least half
    assert res[0][2] == res[1][2]                      # both ranks report the same figures
