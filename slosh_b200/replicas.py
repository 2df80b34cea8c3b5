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


def lpt_partition(costs, parts):
    """Longest-processing-time partition of independent tanks over `parts` ranks: tanks in decreasing cost
    (ties by index) each go to the rank with the least total so far (ties by rank). Returns one sorted
    index list per rank; deterministic, so every rank computes the same plan without communication."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * parts
    plan = [[] for _ in range(parts)]
    for i in order:
        r = min(range(parts), key=lambda k: (load[k], k))
        plan[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in plan]


def gather_tank_stats(stats, device=None, width=4):
    """All-gather of per-tank result rows (tank index, substeps, last solve iterations, fluid cells, and
    any further per-tank figures up to `width` columns) from every rank, as one list sorted by tank
    index; a single process returns its own rows."""
    rows = [tuple(float(v) for v in r) for r in stats]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return sorted(rows)
    world = dist.get_world_size()
    dev = device if device is not None else ("cuda" if dist.get_backend() == "nccl" else "cpu")
    n = torch.tensor([len(rows)], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    cap = int(max(int(c.item()) for c in counts))
    mine = torch.zeros((max(cap, 1), width), dtype=torch.float64, device=dev)
    if rows:
        mine[:len(rows)] = torch.tensor(rows, dtype=torch.float64, device=dev)
    parts = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine)
    out = []
    for c, p in zip(counts, parts):
        out.extend(tuple(float(v) for v in row) for row in p[:int(c.item())].cpu().tolist())
    return sorted(out)
