"""Replicas across GPUs: one process per GPU, each sweeping its own instances.

The sweep of one mesh partition does not shard across GPUs here (the
reference's spatial decomposition, GraphTraverser.cc:659-731, is out of
scope), so N GPUs run N independent replicas with no collective on the data
path.  The group below is the plumbing around them: a barrier to bracket the
timed region, max-over-ranks of a device time, sum-over-ranks of the units
processed, and a round-robin split of independent instances (solve requests)
across ranks.  It is torch.distributed underneath: NCCL between GPUs, gloo
on the host.
"""
import datetime
import os

import torch
import torch.distributed as dist


class ReplicaGroup:
    """World of replica ranks read from the torchrun environment.

    world_size 1 needs no process group; larger worlds initialise one with
    `backend` ("nccl" for GPUs, "gloo" on the host) and a short timeout, so a
    rank that never arrives ends the others' next collective with an error.
    """

    def __init__(self, backend=None, timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        self._owns = False
        if self.world > 1:
            if self.backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            if not dist.is_initialized():
                dist.init_process_group(self.backend,
                                        timeout=datetime.timedelta(seconds=timeout_s))
                self._owns = True

    @property
    def device(self):
        """CUDA ordinal this rank sweeps on."""
        return self.local_rank if self.world > 1 else 0

    def _tensor(self, x):
        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self.backend == "nccl" and torch.cuda.is_available():
            torch.cuda.synchronize()
        if self.world > 1:
            dist.barrier()

    def max(self, x):
        """Largest value over ranks (device times: the job ends with the slowest)."""
        if self.world == 1:
            return float(x)
        t = self._tensor(x)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        """Sum over ranks (units processed by the whole job)."""
        if self.world == 1:
            return float(x)
        t = self._tensor(x)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def shard(self, n):
        """Indices of n independent instances owned by this rank (round robin)."""
        return list(range(self.rank, n, self.world))

    def throughput(self, units, seconds):
        """Whole-job rate: the units of all ranks over the slowest rank's time."""
        return self.sum(units) / self.max(seconds)

    def close(self):
        if self._owns and dist.is_initialized():
            dist.destroy_process_group()
            self._owns = False
