"""Sharding of configurations over ranks, and the one exchange an LM step
needs across them.

Configurations are independent, so the objective and its normal equations
are sums over configurations: rank r evaluates the configurations it owns
and the ranks add
    JᵀJ (D × D), Jᵀr (D) and ‖F‖²
with one sum all-reduce (NCCL on GPUs, gloo in the CPU tests).  The shard
assignment balances the work by atom count (greedy longest-first into the
least-loaded rank), deterministically, so every rank computes the same
assignment without communicating.
"""
from __future__ import annotations

import numpy as np


def shard_configs(natoms, world: int):
    """Per-rank sorted index arrays of the configurations: the largest
    configuration goes to the least-loaded rank (ties to the lower rank)."""
    natoms = np.asarray(natoms)
    order = sorted(range(natoms.size), key=lambda c: (-int(natoms[c]), c))
    load = [0] * world
    own = [[] for _ in range(world)]
    for c in order:
        r = min(range(world), key=lambda k: (load[k], k))
        own[r].append(c)
        load[r] += int(natoms[c])
    return [np.array(sorted(o), dtype=np.int64) for o in own]


def pack_normal_equations(JtJ, Jtr, obj):
    """One FP64 buffer [JᵀJ (row-major), Jᵀr, ‖F‖²] for a single all-reduce
    (the layout fs_gpu_copy_normal_equations writes on the device)."""
    return np.concatenate([np.asarray(JtJ, np.float64).ravel(), np.asarray(Jtr, np.float64).ravel(),
                           [float(obj)]])


def unpack_normal_equations(buf, D):
    buf = np.asarray(buf)
    return buf[:D * D].reshape(D, D), buf[D * D:D * D + D], float(buf[D * D + D])


def allreduce_normal_equations(JtJ, Jtr, obj, group=None):
    """Sum (JᵀJ, Jᵀr, ‖F‖²) over the ranks of `group` (torch.distributed)."""
    import torch
    import torch.distributed as dist
    D = np.asarray(Jtr).size
    t = torch.from_numpy(pack_normal_equations(JtJ, Jtr, obj))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return unpack_normal_equations(t.numpy(), D)
