"""The multi-GPU case sharding on CPU: two gloo ranks, a stand-in solver.

Each rank solves its slice of the case stack; the all-gather must hand every
rank every case's result exactly once, in case order. The stand-in records
which rank solved which case, so the test also checks the partition. Further
cases send engine result objects through the gather, make one rank's solve
raise, and check the device each rank's solver is given.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from anukulan_b200 import distributed as D
from anukulan_b200.lpgen import CaseStack
from anukulan_b200.model import Csr, StandardLp


def _stack(num_cases):
    a = Csr.from_triplets(2, 3, [0, 0, 1], [0, 2, 1], [1.0, 2.0, 3.0])
    base = StandardLp(a, np.ones(3), np.ones(2), np.zeros(3), np.full(3, 5.0), 1, 1.0, 0.0,
                      np.arange(2, dtype=np.int32), np.ones(2), "tiny")
    c = np.tile(base.c, (num_cases, 1)) + np.arange(num_cases)[:, None]
    return CaseStack(base, [f"case{k}" for k in range(num_cases)], c,
                     np.tile(base.q, (num_cases, 1)), np.tile(base.lower, (num_cases, 1)),
                     np.tile(base.upper, (num_cases, 1)))


def _worker(rank, world, port, num_cases, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        stack = _stack(num_cases)
        res = D.solve_stack_sharded(
            stack, solve=lambda s: [(rank, float(c[0])) for c in s.c])
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("num_cases", [60, 7, 1])
def test_sharded_stack_two_ranks(num_cases):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, num_cases, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        res = got[rank]
        assert [c for _, c in res] == [1.0 + k for k in range(num_cases)]
        owners = [r for r, _ in res]
        assert owners == sorted(owners)
        for r in (0, 1):
            assert owners.count(r) == len(D.case_shard(num_cases, r, 2))


def test_case_shard_partition():
    for n in (0, 1, 5, 60, 61):
        for w in (1, 2, 3, 8):
            covered = [k for r in range(w) for k in D.case_shard(n, r, w)]
            assert covered == list(range(n))
    with pytest.raises(ValueError):
        D.case_shard(4, 2, 2)


def _node_worker(rank, world, port, num_nodes, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        base = _stack(1).base
        lower = np.tile(base.lower, (num_nodes, 1))
        upper = np.tile(base.upper, (num_nodes, 1))
        upper[:, 0] = np.arange(num_nodes)          # node k: column 0 capped at k
        res = D.solve_nodes_sharded(
            base, lower, upper, solve=lambda lp, lo, up: [(rank, float(u[0])) for u in up])
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("num_nodes", [9, 1])
def test_sharded_nodes_two_ranks(num_nodes):
    """Node relaxations shard like a case stack: every rank ends with every
    node's result once, in node order, each rank having solved its slice."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_node_worker, args=(r, 2, port, num_nodes, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        res = got[rank]
        assert [u for _, u in res] == [float(k) for k in range(num_nodes)]
        owners = [r for r, _ in res]
        for r in (0, 1):
            assert owners.count(r) == len(D.case_shard(num_nodes, r, 2))


def _host_result(k, n, m):
    """A PdhgResult as the engine returns it, built on the host: case k's
    x and y carry k so the order can be checked after the gather."""
    from anukulan_b200.abi import OPTIMAL, PdhgResult, Residual
    res = Residual(relative_primal=1e-7 * k, dual_objective=-float(k))
    return PdhgResult(OPTIMAL, np.full(n, float(k)), np.arange(m, dtype=float) + k, 2.5 * k,
                      40 * (k + 1), k, 0, 0, False, 0.01, 4.0, 0.9, 1.0,
                      {"scaling": 0.0, "matrix_norm": 0.0, "setup": 0.0, "iterating": 0.0,
                       "checks": 0.0, "polishing": 0.0}, res, (1.0, 1.0, 1.0, 1.0), 0, 12, 0.0,
                      0, f"case {k}")


def _spawn(target, *args, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, 2, port, *args, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=timeout) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return got


def _result_worker(rank, world, port, num_cases, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        stack = _stack(num_cases)
        first = D.case_shard(num_cases, rank, world).start
        res = D.solve_stack_sharded(
            stack, solve=lambda s: [_host_result(first + i, 3, 2) for i in range(s.num_cases)])
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_sharded_stack_gathers_engine_results():
    """Engine result objects, x and y arrays included, survive the pickled
    all-gather intact and in case order on every rank."""
    got = _spawn(_result_worker, 5)
    for rank in (0, 1):
        res = got[rank]
        assert len(res) == 5
        for k, r in enumerate(res):
            want = _host_result(k, 3, 2)
            assert r.status == want.status and r.objective == want.objective
            assert r.iterations == want.iterations and r.message == want.message
            np.testing.assert_array_equal(r.x, want.x)
            np.testing.assert_array_equal(r.y, want.y)
            assert r.residual == want.residual


def _failing_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        def solve(s):
            if rank == 1:
                raise ValueError("bad node bound")
            return [0] * s.num_cases
        try:
            D.solve_stack_sharded(_stack(6), solve=solve)
            out.put((rank, "no error"))
        except RuntimeError as e:
            out.put((rank, str(e)))
    finally:
        dist.destroy_process_group()


def test_sharded_stack_failure_raises_on_every_rank():
    """A rank whose solve raises still reaches the all-gather; every rank then
    raises with that rank's message instead of waiting for the timeout."""
    got = _spawn(_failing_worker)
    for rank in (0, 1):
        assert "rank 1: ValueError: bad node bound" in got[rank], got[rank]


def _device_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["LOCAL_RANK"] = str(3 + rank)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from anukulan_b200 import pdhg as P
        seen = []
        P.solve_case_stack = lambda s, **kw: seen.append(("stack", kw)) or [0] * s.num_cases
        P.solve_node_relaxations = (lambda lp, lo, up, **kw:
                                    seen.append(("nodes", kw)) or [0] * lo.shape[0])
        stack = _stack(4)
        D.solve_stack_sharded(stack, tolerance=1e-4)
        D.solve_stack_sharded(stack, device=7)
        D.solve_nodes_sharded(stack.base, stack.lower, stack.upper)
        out.put((rank, seen))
    finally:
        dist.destroy_process_group()


def test_sharded_default_device_is_local_rank():
    """Without a device named, each rank's solver gets its LOCAL_RANK device;
    a device the caller names is kept."""
    got = _spawn(_device_worker)
    for rank in (0, 1):
        seen = got[rank]
        assert seen[0] == ("stack", {"tolerance": 1e-4, "device": 3 + rank})
        assert seen[1] == ("stack", {"device": 7})
        assert seen[2] == ("nodes", {"device": 3 + rank})
