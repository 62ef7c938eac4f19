"""Replica bookkeeping across ranks with the gloo backend on the CPU
(world size 2): max-over-ranks time, summed atoms, and detection of a rank
that dies (a short process-group timeout turns the missing rank into an
error on the survivor instead of a hang)."""

import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp

from prolix_b200 import replicas


def _free_port():
  s = socket.socket()
  s.bind(("127.0.0.1", 0))
  p = s.getsockname()[1]
  s.close()
  return p


def _worker(rank, world, port, mode, q):
  import torch.distributed as dist
  os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                    RANK=str(rank), LOCAL_RANK=str(rank))
  dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=6))
  try:
    if mode == "ok":
      out = replicas.aggregate(local_ms=10.0 + 5.0 * rank, local_atoms=1000 * (rank + 1), steps=4)
      q.put((rank, out))
    else:  # rank 1 leaves between steps without joining the next collective
      replicas.barrier()
      if rank == 1:
        q.put((rank, "left"))
        return
      try:
        replicas.reduce_max(1.0)
        q.put((rank, "no error"))
      except Exception as e:  # noqa: BLE001 - the timeout surfaces as a runtime error
        q.put((rank, f"detected: {type(e).__name__}"))
  finally:
    try:
      dist.destroy_process_group()
    except Exception:
      pass


def _run(mode):
  ctx = mp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
  for p in procs:
    p.start()
  for p in procs:
    p.join(timeout=60)
  for p in procs:
    if p.is_alive():
      p.kill()
  return dict(q.get(timeout=5) for _ in range(2))


def test_aggregate_takes_slowest_rank_and_total_atoms():
  res = _run("ok")
  for r in (0, 1):
    assert res[r]["ms"] == 15.0
    assert res[r]["atoms"] == 3000
    assert res[r]["atom_steps_per_s"] == pytest.approx(3000 * 4 / 15e-3)


def test_dead_rank_is_detected_by_timeout():
  res = _run("fail")
  assert res[1] == "left"
  assert res[0].startswith("detected")


def test_rank_seeds_differ():
  assert replicas.rank_seed(2024, 0) != replicas.rank_seed(2024, 1)
