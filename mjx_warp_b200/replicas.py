"""Multi-GPU replicas: worlds are independent, so N GPUs run N disjoint world slices.

The batched step has no exchange between worlds (every reference kernel is world-parallel,
mujoco_warp/_src/*.py launch over (nworld, ...)), so scaling over GPUs is sharding the world axis:
rank r owns worlds [start, start + count) with its own Model copy and Data.  There is no
collective on the data path; torch.distributed is used only to align the timing region
(barrier) and to take the maximum elapsed time over ranks.
"""

from __future__ import annotations

import os
from typing import Tuple

import numpy as np
import torch


def shard_worlds(nworld_total: int, rank: int, world_size: int) -> Tuple[int, int]:
  """Contiguous, balanced slice (start, count) of the world axis owned by `rank`."""
  if world_size <= 0 or not 0 <= rank < world_size:
    raise ValueError(f"bad rank {rank} / world_size {world_size}")
  base, extra = divmod(nworld_total, world_size)
  start = rank * base + min(rank, extra)
  return start, base + (1 if rank < extra else 0)


def world_seeds(seed: int, start: int, count: int) -> np.ndarray:
  """Per-world seeds that do not depend on how the world axis is sharded."""
  ss = np.random.SeedSequence(seed)
  children = ss.spawn(start + count)[start:]
  return np.array([c.generate_state(1)[0] for c in children], dtype=np.uint64)


def dist_env() -> Tuple[int, int, int]:
  """(rank, world_size, local_rank) from the torchrun environment (1 process when absent)."""
  return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
          int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(value: float, device=None) -> float:
  """Maximum of a per-rank scalar (e.g. elapsed seconds) over the process group."""
  if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
    return float(value)
  t = torch.tensor([float(value)], dtype=torch.float64, device=device)
  torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
  return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
  if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
    return float(value)
  t = torch.tensor([float(value)], dtype=torch.float64, device=device)
  torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
  return float(t.item())
