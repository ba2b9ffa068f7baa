"""Work-list sharding of independent problems over ranks (one process per GPU).

A batch of independent 2D solves (the batched-solve form) partitions naturally:
every problem is solved whole on one GPU, so the only cross-rank traffic is
the final gather of per-problem statistics.  Problems are assigned by longest
processing time first on the estimated cost n^2 (the unknowns of the fine
grid; a V-cycle costs about 4/3 of a fine-grid sweep), each to the rank with
the smallest load so far, ties to the lowest rank: a deterministic split that
every rank computes identically, with no exchange.
"""
import numpy as np


def partition(sizes, world):
    """Problem ids per rank for edge sizes `sizes` (one entry per problem)."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]) ** 2, i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(sizes[i]) ** 2
    return [sorted(p) for p in parts]


def loads(sizes, parts):
    """Estimated cost (sum of n^2) per rank."""
    sizes = np.asarray(sizes, dtype=np.int64)
    return [int((sizes[p] ** 2).sum()) if len(p) else 0 for p in parts]


def gather_stats(ids, values, dist=None):
    """All ranks' per-problem values in problem order: ids and values (rows) of
    this rank's problems in, the full table (n_problems x columns) out on every
    rank.  One all-gather of a padded tensor (gloo or NCCL); without a process
    group the local table is returned."""
    import torch
    ids = np.asarray(ids, dtype=np.int64)
    values = np.asarray(values, dtype=np.float64).reshape(len(ids), -1)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        out = np.full((ids.max() + 1 if len(ids) else 0, values.shape[1]), np.nan)
        out[ids] = values
        return out
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    world = dist.get_world_size()
    n_local = torch.tensor([len(ids)], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(counts, n_local)
    m = int(max(int(c.item()) for c in counts))
    cols = values.shape[1]
    buf = torch.full((m, cols + 1), float("nan"), dtype=torch.float64, device=dev)
    if len(ids):
        buf[:len(ids), 0] = torch.from_numpy(ids.astype(np.float64)).to(dev)
        buf[:len(ids), 1:] = torch.from_numpy(values).to(dev)
    bufs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf)
    rows = torch.cat([b[:int(c.item())] for b, c in zip(bufs, counts)]).cpu().numpy()
    n = int(rows[:, 0].max()) + 1 if len(rows) else 0
    out = np.full((n, cols), np.nan)
    out[rows[:, 0].astype(np.int64)] = rows[:, 1:]
    return out
