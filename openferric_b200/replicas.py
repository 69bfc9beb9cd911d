"""Several GPUs as independent replicas over torch.distributed.

One process per GPU prices its own paths: replica r draws with seed + r, so
the replicas' samples are independent, and no collective touches the path
data.  Two small collectives remain:

- `max_over_ranks`: a job's device time is the slowest rank's, so a
  throughput over N GPUs is (units of all ranks) / max(time);
- `combine_sums`: an FP64 all-reduce of the five running sums of
  MonteCarloEngine::run (src/mc/simulation.rs:305-347) and the sample
  counts, after which every rank holds the estimator over all replicas'
  samples (`finish` is the same statistics as the device's).

Works with any backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import math
from typing import Optional, Sequence, Tuple

import torch
import torch.distributed as dist

from . import _abi as A


def _active() -> bool:
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def replica_seed(seed: int, rank: int) -> int:
    """The seed of replica `rank` (wrapping u64)."""
    return (int(seed) + int(rank)) & 0xFFFFFFFFFFFFFFFF


def max_over_ranks(value: float, device: Optional[torch.device] = None) -> float:
    """The largest `value` over all ranks (itself without a process group)."""
    if not _active():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def finish(sums: Sequence[float], count: int, cv_kind: int = A.OF_CV_NONE, cv_expected: float = 0.0,
           discount: float = 1.0) -> Tuple[float, float]:
    """Price and stderr from the five sums (simulation.rs:305-347), with the
    control-variate adjustment when cv_kind is set."""
    sx, sx2, sy, sxy, sy2 = (float(v) for v in sums)
    n = float(count)
    if cv_kind != A.OF_CV_NONE:
        denom = max(n - 1.0, 1.0)
        cov_xy = (sxy - sx * sy / n) / denom
        var_y = (sy2 - sy * sy / n) / denom
        beta = cov_xy / var_y if var_y > 1e-16 else 0.0
        e = cv_expected
        s_adj = sx + beta * (n * e - sy)
        s_adj2 = sx2 + 2.0 * beta * e * sx - 2.0 * beta * sxy + beta * beta * (n * e * e - 2.0 * e * sy + sy2)
        mean = s_adj / n
        var = (s_adj2 - s_adj * s_adj / n) / (n - 1.0) if n > 1.0 else 0.0
    else:
        mean = sx / n
        var = (sx2 - sx * sx / n) / (n - 1.0) if n > 1.0 else 0.0
    return discount * mean, discount * math.sqrt(max(var, 0.0) / n)


def combine_sums(result: A.OfMcResult, cv_kind: int = A.OF_CV_NONE, cv_expected: float = 0.0,
                 discount: float = 1.0, device: Optional[torch.device] = None) -> Tuple[float, float, int]:
    """All-reduces a replica's five sums and sample count and returns
    (price, stderr, samples) of the estimator over every replica's samples."""
    v = [result.sum_x, result.sum_x2, result.sum_y, result.sum_xy, result.sum_y2, float(result.samples)]
    if _active():
        t = torch.tensor(v, dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        v = t.tolist()
    count = int(round(v[5]))
    price, stderr = finish(v[:5], count, cv_kind, cv_expected, discount)
    return price, stderr, count
