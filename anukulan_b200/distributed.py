"""Case stacks across GPUs: one process per GPU, cases partitioned by rank.

The cases of a stack are independent LPs that share the matrix, so the work
shards with no exchange on the data path. Each rank solves a contiguous
slice of the cases on its own GPU with the case-stack engine; the per-case
results then meet once, through one all-gather of the results (NCCL or
gloo, whichever process group the caller set up). Every rank ends with all
results in case order.
"""
from __future__ import annotations

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
    if solve is None:
        from .pdhg import solve_case_stack

        def solve(s):
            return solve_case_stack(s, **kw)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = case_shard(stack.num_cases, rank, world)
    local = solve(sub_stack(stack, mine)) if len(mine) else []
    if len(local) != len(mine):
        raise RuntimeError("the solver returned a result count different from its cases")
    gathered: List = [None] * world
    dist.all_gather_object(gathered, list(local), group=group)
    out: List = []
    for part in gathered:
        out.extend(part)
    return out


def solve_nodes_sharded(lp, lower, upper, solve: Optional[Callable] = None, group=None,
                        **kw) -> List:
    """Branch-and-bound node relaxations across the ranks of `group`: the
    nodes' bounds (nodes x columns) are sliced like a case stack, each rank
    solves its slice as one stack, and one all-gather gives every rank every
    node's result in node order. `solve` maps (lp, lower, upper) to a list of
    results (default: pdhg.solve_node_relaxations with `kw` as options)."""
    import torch.distributed as dist
    if solve is None:
        from .pdhg import solve_node_relaxations

        def solve(base, lo, up):
            return solve_node_relaxations(base, lo, up, **kw)
    lower = np.atleast_2d(np.asarray(lower, np.float64))
    upper = np.atleast_2d(np.asarray(upper, np.float64))
    if lower.shape != upper.shape:
        raise ValueError("node bounds must have the same shape")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = case_shard(lower.shape[0], rank, world)
    idx = list(mine)
    local = solve(lp, lower[idx], upper[idx]) if idx else []
    if len(local) != len(idx):
        raise RuntimeError("the solver returned a result count different from its nodes")
    gathered: List = [None] * world
    dist.all_gather_object(gathered, list(local), group=group)
    out: List = []
    for part in gathered:
        out.extend(part)
    return out
