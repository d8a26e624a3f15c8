"""The batched form's multi-rank data path on one GPU: two gloo ranks (processes) share cuda:0,
each solves its LPT share of a 24-instance batch with ranks.batched_share (the path bench.py
--workload batched runs under torchrun), and the union of their per-instance Newton solutions
equals one rank solving all 24 (to 1e-9). The ranks' kernels never wait on each other: every instance is
solved by its own rank's persistent launch, and the ranks exchange results on the host only."""
import multiprocessing as mp
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCHEDULE = (2, 256)  # fixed, so that every instance runs the same solver schedule in every batch
# The mixed-precision assembly adds FP32 element blocks with atomics, whose order (and so the last
# bits of the stored operator) changes from run to run: the same instance agrees to about 1e-12.
TOL = 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problems():
    from tests.test_gpu_batch import small_batch
    probs = small_batch(24, seed=13)
    for q in probs:
        q.newton_rtol = 1e-8
        q.max_steps = 2
        q.t_final = 2 * q.dt
    return probs


def _solve(ids_and_batch):
    ids, b = ids_and_batch
    out = b.newton_run(max_newton=12)
    sols = {int(i): out["disp"][b.instance_slice(k)].copy() for k, i in enumerate(ids)}
    st = {int(i): int(out["status"][k]) for k, i in enumerate(ids)}
    b.close()
    return sols, st


def _worker(rank, world, port, q):
    import datetime
    import os

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from mphyfem_b200 import _lib, api, ranks
        torch.cuda.set_device(0)
        ctx = api.Context(0)
        share = ranks.batched_share(_problems(), rank, world, ctx, schedule=SCHEDULE, precision=_lib.PREC_MIXED,
                                    rtol=1e-10, norm_type=1, tangent=_lib.TANGENT_CONSISTENT)
        sols, st = _solve(share)
        gathered = [None] * world
        dist.all_gather_object(gathered, (sols, st))
        if rank == 0:
            q.put(gathered)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_one_gpu_equal_one_rank():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build, ranks
    build.build()
    ctx = mp.get_context("spawn")
    qu = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, qu)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = qu.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    sols, st = {}, {}
    for s_r, st_r in gathered:
        assert not set(s_r) & set(sols)  # disjoint shares
        sols.update(s_r)
        st.update(st_r)
    assert sorted(sols) == list(range(24))
    # one rank, every instance
    ref_sols, ref_st = _solve(ranks.batched_share(_problems(), 0, 1, api.Context(0), schedule=SCHEDULE,
                                                  precision=_lib.PREC_MIXED, rtol=1e-10, norm_type=1,
                                                  tangent=_lib.TANGENT_CONSISTENT))
    assert st == ref_st and all(v == 0 for v in st.values())
    for i in range(24):
        scale = max(np.abs(ref_sols[i]).max(), 1e-300)
        assert np.abs(sols[i] - ref_sols[i]).max() <= TOL * scale, i
