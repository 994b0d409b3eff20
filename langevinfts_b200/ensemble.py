"""Replica ensembles over several GPUs (one process per GPU).

Replicas are independent systems, so a Langevin step needs no communication:
each rank owns its own replicas with their own PCG64 streams.  The only
exchange is optional and happens at recording time: ensemble sums of the
structure functions, Hamiltonians and dH/dchiN over all replicas of all
ranks (one all-reduce per quantity, NCCL between GPUs, gloo on CPU).
"""
import numpy as np


def replica_seeds(rank, n_replicas, base=1000):
    """PCG64 seeds of the replicas of one rank: disjoint across ranks."""
    return [base + rank * n_replicas + r for r in range(n_replicas)]


def _device(group):
    import torch.distributed as dist
    return "cuda" if dist.get_backend(group) == "nccl" else "cpu"


def max_over_ranks(values, group=None):
    """Element-wise maximum of a list of floats over all ranks (the job time of
    a step is the slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(v) for v in t.cpu()]


def ensemble_sum(arrays, group=None):
    """Sum each array of a dict over its leading (replica) axis and then over
    all ranks.  Complex arrays are reduced as interleaved real pairs.  Returns
    (sums, number of replicas in the ensemble)."""
    import torch
    import torch.distributed as dist
    distributed = dist.is_available() and dist.is_initialized()
    out, count = {}, None
    for key in sorted(arrays):
        a = np.asarray(arrays[key])
        n = a.shape[0]
        count = n if count is None else count
        if n != count:
            raise ValueError("every array needs the same number of replicas")
        local = np.ascontiguousarray(a.sum(axis=0))
        if not distributed:
            out[key] = local
            continue
        flat = local.view(np.float64) if np.iscomplexobj(local) else local.astype(np.float64)
        t = torch.from_numpy(np.ascontiguousarray(flat)).to(_device(group))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        red = t.cpu().numpy()
        out[key] = red.view(np.complex128).reshape(local.shape) if np.iscomplexobj(local) else red.reshape(local.shape)
    total = count or 0
    if distributed:
        t = torch.tensor([float(total)], dtype=torch.float64, device=_device(group))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        total = int(round(float(t.cpu()[0])))
    return out, total
