"""Multi-GPU replicas: one process per GPU, frequency points or designs
sharded across ranks, no collective on the data path.

Every frequency point of a sweep (and every design of a family) is an
independent solve, so N GPUs run N independent replicas of the hot path; the
only communication is the final gather of the (tiny) results to rank 0 over
``torch.distributed`` (NCCL between GPUs, gloo for host-only tests).
"""
from __future__ import annotations

import numpy as np


def shard(n, rank, world, mode="strided"):
    """Indices of items 0..n-1 owned by ``rank``: ``strided`` (i % world ==
    rank, balances sweeps whose cost grows along the list) or ``block``
    (contiguous, keeps a rank's frequencies adjacent)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside world %d" % (rank, world))
    if mode == "strided":
        return np.arange(rank, n, world)
    if mode == "block":
        q, r = divmod(n, world)
        lo = rank * q + min(rank, r)
        return np.arange(lo, lo + q + (1 if rank < r else 0))
    raise ValueError(mode)


def gather(values, idx, n, group=None):
    """Assemble the per-rank results (``values[k]`` belongs to item ``idx[k]``)
    into one array of n items on every rank (all_gather of Python objects;
    results are a few bytes per frequency point)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, (np.asarray(idx), np.asarray(values)), group=group)
    out = None
    seen = np.zeros(n, dtype=bool)
    for ids, vals in parts:
        if out is None:
            out = np.zeros((n,) + vals.shape[1:], dtype=vals.dtype)
        out[ids] = vals
        seen[ids] = True
    if not seen.all():
        raise RuntimeError("items %s were not computed by any rank" % np.nonzero(~seen)[0][:8])
    return out


def sharded_sweep(run, freqs, rank, world, group=None, mode="strided"):
    """Zin and S11 of ``freqs`` with this rank sweeping its shard through
    ``run(local_freqs) -> (Zin, S11)`` (e.g. ``SweepPlan.run``), gathered on
    every rank.  A rank whose ``run`` raises reports the failure to the
    others through the gather (every rank raises), so no rank waits forever."""
    import torch.distributed as dist

    freqs = np.asarray(freqs, dtype=np.float64)
    idx = shard(freqs.size, rank, world, mode)
    err = None
    try:
        Zin, S11 = run(freqs[idx]) if idx.size else (np.zeros(0, complex), np.zeros(0, complex))
        vals = np.stack([Zin, S11], axis=1)
    except Exception as e:  # noqa: BLE001 -- forwarded to every rank below
        err = "rank %d: %s: %s" % (rank, type(e).__name__, e)
        vals = np.zeros((idx.size, 2), dtype=complex)
    flags = [None] * dist.get_world_size(group)
    dist.all_gather_object(flags, err, group=group)
    failed = [f for f in flags if f]
    if failed:
        raise RuntimeError("sharded sweep failed: " + "; ".join(failed))
    out = gather(vals, idx, freqs.size, group)
    return out[:, 0], out[:, 1]
