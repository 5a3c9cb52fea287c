"""Case stacks across GPUs: one process per GPU, cases partitioned by rank.

The cases of a stack are independent LPs that share the matrix, so the work
shards with no exchange on the data path. Each rank solves a contiguous
slice of the cases on its own GPU with the case-stack engine; the per-case
results then meet once, through one all-gather of the results (NCCL or
gloo, whichever process group the caller set up). Every rank ends with all
results in case order.

Each rank drives the GPU of its LOCAL_RANK (as torchrun sets it; the rank
itself without one) unless the caller names a device. A rank whose solve
raises still joins the all-gather, carrying its error, so every rank raises
together instead of waiting in the collective until the group times out.
"""
from __future__ import annotations

import os
from typing import Callable, List, Optional

import numpy as np

from .lpgen import CaseStack


def case_shard(num_cases: int, rank: int, world: int) -> range:
    """The contiguous slice of `num_cases` cases that `rank` of `world` solves;
    slice sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(num_cases, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def rank_device(rank: int) -> int:
    """The CUDA device a rank drives by default: LOCAL_RANK when the launcher
    set it, else the rank."""
    return int(os.environ.get("LOCAL_RANK", rank))


def _default_device(kw: dict, rank: int) -> dict:
    """kw with `device` set to the rank's device, unless kw names a device or
    passes a whole options struct (whose `device` field then decides)."""
    if "device" in kw or kw.get("options") is not None:
        return kw
    return dict(kw, device=rank_device(rank))


def _gather_results(local_solve: Callable[[], List], expected: int, what: str, group) -> List:
    """Runs this rank's share and all-gathers (ok, results or message) from
    every rank; raises on every rank when any rank failed."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    try:
        local = list(local_solve()) if expected else []
        if len(local) != expected:
            raise RuntimeError(f"the solver returned a result count different from its {what}")
        payload = (True, local)
    except Exception as e:  # every rank must reach the collective
        payload = (False, f"rank {rank}: {type(e).__name__}: {e}")
    gathered: List = [None] * world
    dist.all_gather_object(gathered, payload, group=group)
    failed = [msg for ok, msg in gathered if not ok]
    if failed:
        raise RuntimeError("sharded solve failed: " + "; ".join(failed))
    out: List = []
    for _, part in gathered:
        out.extend(part)
    return out


def sub_stack(stack: CaseStack, cases: range) -> CaseStack:
    idx = list(cases)
    return CaseStack(stack.base, [stack.names[i] for i in idx], stack.c[idx], stack.q[idx],
                     stack.lower[idx], stack.upper[idx])


def solve_stack_sharded(stack: CaseStack, solve: Optional[Callable] = None, group=None,
                        **kw) -> List:
    """Solves `stack` across the ranks of `group` (the default process group)
    and returns every case's result, in case order, on every rank. `solve`
    maps a CaseStack to a list of results (default: the engine's
    solve_case_stack with `kw` as options)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if solve is None:
        from .pdhg import solve_case_stack
        opts = _default_device(kw, rank)

        def solve(s):
            return solve_case_stack(s, **opts)
    mine = case_shard(stack.num_cases, rank, world)
    return _gather_results(lambda: solve(sub_stack(stack, mine)), len(mine), "cases", group)


def solve_nodes_sharded(lp, lower, upper, solve: Optional[Callable] = None, group=None,
                        **kw) -> List:
    """Branch-and-bound node relaxations across the ranks of `group`: the
    nodes' bounds (nodes x columns) are sliced like a case stack, each rank
    solves its slice as one stack, and one all-gather gives every rank every
    node's result in node order. `solve` maps (lp, lower, upper) to a list of
    results (default: pdhg.solve_node_relaxations with `kw` as options)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if solve is None:
        from .pdhg import solve_node_relaxations
        opts = _default_device(kw, rank)

        def solve(base, lo, up):
            return solve_node_relaxations(base, lo, up, **opts)
    lower = np.atleast_2d(np.asarray(lower, np.float64))
    upper = np.atleast_2d(np.asarray(upper, np.float64))
    if lower.shape != upper.shape:
        raise ValueError("node bounds must have the same shape")
    idx = list(case_shard(lower.shape[0], rank, world))
    return _gather_results(lambda: solve(lp, lower[idx], upper[idx]), len(idx), "nodes", group)
