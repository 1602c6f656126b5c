"""Time sharding of an integration across processes (one GPU each).

DiFX's FxManager hands successive subintegrations to Core processes in turn
(mpifxcorr/src/fxmanager.cpp:334-337, ``coreids[sendcount % numcores]``) and
adds every returned core result into the integration (Visibility::addData,
visibility.cpp:181).  Here each rank correlates the subints assigned to it on
its own GPU and the integration is summed with one reduction of the
core-result buffers (FP32, sum) over the process group -- NCCL over
NVLink/NVSwitch on GPUs, gloo on CPU.  There is no other exchange: the
subints are independent.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def subints_for_rank(subints: Sequence[Tuple[int, int]], rank: int, world: int) -> List[Tuple[int, int]]:
    """Round-robin assignment of subint start times (sec, ns) to ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return [t for k, t in enumerate(subints) if k % world == rank]


def integration_subints(job, start_sec: int, start_ns: int, duration_s: float) -> List[Tuple[int, int]]:
    """Start times of the subints of one integration."""
    n = int(round(duration_s * 1e9 / job.subint_ns))
    t0 = start_sec * 1_000_000_000 + start_ns
    return [((t0 + k * job.subint_ns) // 1_000_000_000, (t0 + k * job.subint_ns) % 1_000_000_000) for k in range(n)]


def reduce_core_result(buf, dst: int = 0, group=None, all_ranks: bool = False) -> None:
    """Sum the core-result tensor over the process group, in place (into
    rank ``dst``, or into every rank when ``all_ranks``)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return
    if all_ranks:
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    else:
        dist.reduce(buf, dst=dst, op=dist.ReduceOp.SUM, group=group)
