"""Multi-GPU replicas of the forward model: one process per GPU, draws sharded
across ranks, no exchange inside a solve (a solve never spans GPUs).

* `shard_ids` gives each rank its own draw ids (weak scaling: a fixed number of
  draws per rank, ids rank*per_rank ... so every rank's draws are distinct).
* `partition_lpt` splits one fixed ensemble across ranks by the
  longest-processing-time greedy rule on a per-draw cost (cells x expected
  iterations), for strong scaling of a calibration stage.
* `reduce_step` combines the per-rank step outcome: the step time is the max
  over ranks, converged solves are summed, and (optionally) the per-draw
  log-likelihoods are gathered to every rank for the importance weights.
* `sharded_posterior_weights` normalises the importance weights of an ensemble
  sharded across ranks without gathering it: each rank's log-sum-exp of its own
  draws on its GPU, one all-reduce (MAX) and one all-reduce (SUM) of FP64 scalars,
  then every rank rescales its own weights.

Collectives use whatever process group is initialised: NCCL on GPUs, gloo in the
CPU tests.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard_ids(rank: int, world: int, per_rank: int) -> np.ndarray:
    if not (0 <= rank < world) or per_rank < 0:
        raise ValueError("need 0 <= rank < world and per_rank >= 0")
    return np.arange(rank * per_rank, (rank + 1) * per_rank)


def partition_lpt(cost, world: int) -> list:
    """Indices of the draws each rank solves: draws in decreasing cost, each to the
    rank with the least total cost so far (ties to the lower rank)."""
    cost = np.asarray(cost, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be positive")
    order = sorted(range(len(cost)), key=lambda i: (-cost[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + cost[i], r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def reduce_max(value: float, device=None) -> float:
    """Max of one FP64 scalar over ranks (the value itself on one process)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else torch.device("cpu"))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_count(count: int, device=None) -> int:
    """Sum of one integer over ranks (the value itself on one process)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return int(count)
    t = torch.tensor([int(count)], dtype=torch.int64,
                     device=device if device is not None else torch.device("cpu"))
    dist.all_reduce(t)
    return int(t.item())


def reduce_step(ms: float, converged: int, loglik=None, device=None):
    """(max step ms over ranks, total converged, gathered logliks or None)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return ms, converged, (None if loglik is None else np.asarray(loglik, dtype=np.float64))
    dev = device if device is not None else torch.device("cpu")
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([converged], dtype=torch.int64, device=dev)
    dist.all_reduce(c)
    gathered = None
    if loglik is not None:
        x = torch.as_tensor(np.asarray(loglik, dtype=np.float64), device=dev)
        n = torch.tensor([x.numel()], dtype=torch.int64, device=dev)
        sizes = [torch.zeros_like(n) for _ in range(dist.get_world_size())]
        dist.all_gather(sizes, n)
        cap = int(max(int(s.item()) for s in sizes))
        pad = torch.full((cap,), float("nan"), dtype=torch.float64, device=dev)
        pad[: x.numel()] = x
        parts = [torch.empty_like(pad) for _ in sizes]
        dist.all_gather(parts, pad)
        gathered = np.concatenate([p[: int(s.item())].cpu().numpy() for p, s in zip(parts, sizes)])
    return float(t.item()), int(c.item()), gathered


def _device_local_weights(loglik, log_q):
    from . import statistics

    return statistics.posterior_weight_parts(loglik, log_q)


def sharded_posterior_weights(loglik, log_q=None, device=None, local=None):
    """Normalised weights of this rank's draws in the whole sharded ensemble
    (cfdr.statistics.posterior_weights, rans-uq/python/cfdr/statistics.py:217-232,
    over the union of all ranks' draws) and the global log evidence.

    Each rank r computes its own weights w_r, m_r = max(l - log q) and
    s_r = sum exp(l - log q - m_r) on its GPU (`local`, by default
    rq_posterior_weights_parts). One all-reduce (MAX) gives M = max_r m_r and one
    all-reduce (SUM) gives S = sum_r s_r exp(m_r - M); this rank's weights are
    w_r * s_r exp(m_r - M) / S and the log evidence M + log S. The parts stay apart
    so that no large log value is rounded before the exponential. A rank with no
    draws contributes nothing."""
    import torch
    import torch.distributed as dist

    ll = np.ascontiguousarray(np.asarray(loglik, dtype=np.float64).ravel())
    lq = None if log_q is None else np.ascontiguousarray(np.asarray(log_q, np.float64).ravel())
    local = local or _device_local_weights
    if ll.size:
        w, m, s = local(ll, lq)
    else:
        w, m, s = np.empty(0), -np.inf, 0.0
    if not dist.is_initialized() or dist.get_world_size() == 1:
        if not ll.size:
            raise ValueError("at least one evaluation is required")
        return np.asarray(w, dtype=np.float64), m + float(np.log(s))
    dev = device if device is not None else torch.device("cpu")
    mt = torch.tensor([m], dtype=torch.float64, device=dev)
    dist.all_reduce(mt, op=dist.ReduceOp.MAX)
    big = float(mt.item())
    if not np.isfinite(big):
        raise ValueError("at least one evaluation is required")
    part = s * float(np.exp(m - big)) if ll.size else 0.0
    st = torch.tensor([part], dtype=torch.float64, device=dev)
    dist.all_reduce(st)
    total = float(st.item())
    return np.asarray(w, dtype=np.float64) * (part / total), big + float(np.log(total))
