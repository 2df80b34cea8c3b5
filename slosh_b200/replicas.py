"""Independent tank replicas across ranks (one process per GPU).

A single tank does not shard: every smoother sweep and every CG dot product would need an exchange.
Multi-GPU runs therefore advance one independent tank per rank with no data-path collective; the only
cross-rank step is the end-of-run aggregation of the measurement (timed region = max over ranks, work
= sum over ranks)."""
import torch
import torch.distributed as dist


def reduce_run(substeps, device_ms, wall_ms, device=None):
    """Returns (total substeps over ranks, max device ms, max wall ms). Works on NCCL (device tensors)
    and gloo (CPU tensors); a single process returns its own numbers."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(substeps), float(device_ms), float(wall_ms)
    dev = device if device is not None else ("cuda" if dist.get_backend() == "nccl" else "cpu")
    t = torch.tensor([float(device_ms), float(wall_ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    s = torch.tensor([float(substeps)], dtype=torch.float64, device=dev)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    return float(s[0]), float(t[0]), float(t[1])
