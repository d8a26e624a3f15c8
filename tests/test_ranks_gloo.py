"""Multi-rank plumbing on the CPU: two gloo ranks agree on the slowest rank's time and on a
disjoint, complete split of the batched form's instances."""
import multiprocessing as mp
import socket

from mphyfem_b200 import ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import os

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = ranks.max_over_ranks(10.0 + rank)
        r, lr, w = ranks.world_info()
        costs = [5, 1, 9, 3, 7, 2, 8]
        mine = ranks.shard_by_cost(costs, w)[r]
        dist.barrier()
        q.put((rank, t, (r, lr, w), mine, list(ranks.shard(11, r, w))))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [11.0, 11.0]            # every rank sees the slowest time
    assert [o[2] for o in out] == [(0, 0, 2), (1, 1, 2)]
    inst = out[0][3] + out[1][3]
    assert sorted(inst) == list(range(7)) and not set(out[0][3]) & set(out[1][3])
    loads = [sum([5, 1, 9, 3, 7, 2, 8][i] for i in o[3]) for o in out]
    assert abs(loads[0] - loads[1]) <= 9                  # LPT balance: within the largest item
    assert out[0][4] + out[1][4] == list(range(11))


def test_single_process_defaults():
    assert ranks.max_over_ranks(3.5) == 3.5
    assert list(ranks.shard(5, 0, 1)) == [0, 1, 2, 3, 4]
    assert ranks.shard_by_cost([1, 2, 3], 1) == [[0, 1, 2]]
