"""Multi-GPU runs of one workload on N GPUs of a node, one process per GPU.

A single scene does not shard at one-GPU scale (the reference runs one scene per process,
run_simulation.py:649-708, and one B200 holds the largest scene with room to spare), so
each rank steps its own copy of it (replicas).  An ensemble of independent strips is
sharded instead: each rank steps its share (sigmasph_b200.ensemble.shard) and the strips'
final states are gathered once, in float64 (gather_rows).  Neither data path has a
per-step collective.  The timing's collectives are taken by every rank in the same order:
a barrier on each side of the timed region and the maximum of the ranks' times.  The
whole-job throughput is the units all ranks processed over that maximum.

Launched as `torchrun --nproc-per-node N` (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR and
MASTER_PORT from the environment); with WORLD_SIZE 1 nothing is initialised.  The backend
is NCCL on GPUs; the tests run the same code on gloo.
"""
from __future__ import annotations

import datetime
import os


def env_ranks():
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """The process group of a replica run, or a stand-in for one process."""

    def __init__(self, backend="nccl", timeout_s=300.0):
        self.world, self.rank, self.local = env_ranks()
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            # a short group timeout ends a wait on a rank that left with an error
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def reporter(self):
        """Rank 0 prints the result line."""
        return self.rank == 0

    def _device(self):
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, x):
        """The maximum of x over the ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def gather(self, x):
        """x from every rank, in rank order (a check that the replicas agree)."""
        if self.dist is None:
            return [float(x)]
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        out = [torch.zeros_like(t) for _ in range(self.world)]
        self.dist.all_gather(out, t)
        return [float(o.item()) for o in out]

    def sum_over_ranks(self, x):
        """The sum of x over the ranks, in float64 (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def gather_rows(self, rows, index, total):
        """Rows (k, m) float64 of the units this rank owns, at global positions `index`:
        the (total, m) table of all ranks, on every rank.  One float64 sum-reduction of a
        table that is zero outside each rank's own rows, so every entry is exact; a last
        column counts the owners, and a unit owned by no rank or by two is an error."""
        import numpy as np
        rows = np.asarray(rows, dtype=np.float64).reshape(len(index), -1)
        m = rows.shape[1]
        table = np.zeros((int(total), m + 1), dtype=np.float64)
        table[np.asarray(index, dtype=np.int64), :m] = rows
        table[np.asarray(index, dtype=np.int64), m] = 1.0
        if self.dist is not None:
            import torch
            t = torch.from_numpy(table).to(self._device())
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
            table = t.cpu().numpy()
        if not np.all(table[:, m] == 1.0):
            raise RuntimeError("gather_rows: every unit must be owned by exactly one rank")
        return table[:, :m]

    def throughput(self, units_per_rank, seconds):
        """Whole-job units per second: every rank processed units_per_rank in at most
        `seconds` (the max over ranks)."""
        return self.world * float(units_per_rank) / float(seconds)

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
