"""Multi-rank batch host logic on CPU (gloo, world size 2): cases are sharded
by a greedy bin pack, each rank solves its own with the CPU oracle (the CUDA
path is the same per case), and a gather merges the per-case results; the
merged result equals the single-process one."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from axisim import batch

N_CASES = 6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _solve_cases(indices):
    import oracle
    cs = batch.random_cases(N_CASES, seed=11, scale=0.01, max_iter=4, tol=1e-30)
    out = {}
    for i in indices:
        c = cs[i]
        m = oracle.multiblock(c.blocks)
        o = oracle.Oracle(m, c.bc_fields(), c.settings, threads=1)
        o.run()
        out[i] = {"u": o.get("u"), "p": o.get("p")}
    return out


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [sum(b["axial"][1] * b["radial"][1] for b in c.blocks)
             for c in batch.random_cases(N_CASES, seed=11, scale=0.01)]
    parts = batch.shard(sizes, world)
    local = _solve_cases(parts[rank])
    merged = batch.gather_results(local, world, dist)
    if rank == 0:
        q.put({k: {f: v[f].tolist() for f in v} for k, v in merged.items()})
    dist.barrier()
    dist.destroy_process_group()


def test_shard_covers_every_case_once_and_balances():
    sizes = [5, 9, 1, 7, 3, 8, 2]
    for world in (1, 2, 3, 4):
        parts = batch.shard(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)


@pytest.mark.timeout(300)
def test_two_rank_batch_equals_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = _solve_cases(range(N_CASES))
    assert sorted(int(k) for k in merged) == list(range(N_CASES))
    for i in range(N_CASES):
        for f in ("u", "p"):
            np.testing.assert_array_equal(np.array(merged[i][f]), ref[i][f])


def _worker_one_rank_fails(rank, world, port, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)  # a rank that dies between steps, before the gather
    try:
        batch.gather_results(_solve_cases([0]), world, dist)
        q.put("no error")
    except Exception as e:  # the peer's loss surfaces as an error, not a hang
        q.put("raised: " + type(e).__name__)
    q.close()
    q.join_thread()  # the message is delivered before the process ends
    os._exit(0)


@pytest.mark.timeout(300)
def test_a_rank_that_dies_makes_the_gather_fail_instead_of_hanging():
    # the surviving rank either gets an exception from the gather or is ended
    # by the communication library on the lost connection; both end the rank
    # (what must not happen is a gather that waits for good)
    import queue
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_one_rank_fails, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode is not None for p in procs), "a rank is still waiting"
    assert procs[1].exitcode == 3
    try:
        msg = q.get(timeout=5)
    except queue.Empty:
        msg = None
    if procs[0].exitcode == 0:
        assert msg is not None and msg.startswith("raised"), msg
    else:
        assert msg is None or msg.startswith("raised"), msg
