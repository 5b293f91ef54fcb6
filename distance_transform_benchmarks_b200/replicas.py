"""Multi-GPU execution of the transform: replicas only.

Images are independent and a single image does not shard naturally (its fixpoint would need a halo exchange
after every re-activation), so N GPUs run N replicas, one process per GPU: each rank transforms its own images
and its results stay on its GPU.  There is no data-path collective; the only collectives are host-side
reductions of timings and counters (the step time of a job is the max over ranks, its pixel count the sum).

Launch one process per GPU (``torchrun --nproc-per-node N``, rendezvous on 127.0.0.1); RANK / WORLD_SIZE /
LOCAL_RANK come from the environment.  With WORLD_SIZE 1 no process group is created.
"""
import datetime
import os

import torch


class ReplicaGroup:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, backend="nccl", timeout_s=180.0):
        """Joins the process group (nccl on GPUs, gloo for host-only ranks).  A short timeout makes ranks that
        wait for a missing peer fail with an error instead of waiting for good."""
        if self.world > 1:
            import torch.distributed as td
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = True
        return self

    def barrier(self):
        if self.pg:
            import torch.distributed as td
            td.barrier()

    def _reduce(self, x, device, op):
        if not self.pg:
            return float(x)
        import torch.distributed as td
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        td.all_reduce(t, op=getattr(td.ReduceOp, op))
        return float(t.item())

    def max(self, x, device="cpu"):
        """Max of x over ranks (the job's step time)."""
        return self._reduce(x, device, "MAX")

    def sum(self, x, device="cpu"):
        """Sum of x over ranks (the job's pixels)."""
        return self._reduce(x, device, "SUM")

    def seed(self, base):
        """Seed of this rank's own workload (weak scaling: every rank generates different images)."""
        return int(base) + 1000 * self.rank

    def shard(self, items):
        """This rank's share of a fixed list (strong scaling): items rank, rank + N, rank + 2N, ..."""
        return list(items)[self.rank::self.world]

    def close(self):
        if self.pg:
            import torch.distributed as td
            td.destroy_process_group()
            self.pg = False
