"""World sharding over ranks (replicas) and the max-over-ranks timing reduction, gloo on CPU."""

import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from mjx_warp_b200 import replicas


def test_shard_worlds_partition():
  for total in (1, 7, 8192, 8193):
    for ws in (1, 2, 3, 8):
      slices = [replicas.shard_worlds(total, r, ws) for r in range(ws)]
      assert sum(c for _, c in slices) == total
      assert slices[0][0] == 0
      for (s0, c0), (s1, _) in zip(slices, slices[1:]):
        assert s0 + c0 == s1
      assert max(c for _, c in slices) - min(c for _, c in slices) <= 1


def test_world_seeds_independent_of_sharding():
  full = replicas.world_seeds(3, 0, 10)
  parts = np.concatenate([replicas.world_seeds(3, *replicas.shard_worlds(10, r, 3)) for r in range(3)])
  np.testing.assert_array_equal(full, parts)


def _free_port():
  s = socket.socket()
  s.bind(("127.0.0.1", 0))
  port = s.getsockname()[1]
  s.close()
  return port


def _worker(rank, world_size, port, out):
  os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
  torch.distributed.init_process_group("gloo", rank=rank, world_size=world_size)
  try:
    start, count = replicas.shard_worlds(10, rank, world_size)
    elapsed = 1.0 + rank  # rank 1 is the slow one
    out[rank] = (start, count, replicas.max_over_ranks(elapsed), replicas.sum_over_ranks(count))
  finally:
    torch.distributed.destroy_process_group()


def test_gloo_two_ranks():
  manager = mp.Manager()
  out = manager.dict()
  mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
  assert out[0][:2] == (0, 5) and out[1][:2] == (5, 5)
  assert out[0][2] == out[1][2] == 2.0
  assert out[0][3] == out[1][3] == 10.0
