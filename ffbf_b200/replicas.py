"""Replicas: one process per GPU, each scanning its own workload with no data-path collective.

The scan shards naturally (texts are independent; a pattern set's filter is read-only during a scan), and
the feed-forward filter of sharded runs would need an OR reduction that NCCL does not offer, so several
GPUs run independent replicas: rank r scans the workload drawn from seed + r on GPU LOCAL_RANK. The only
collectives are host-side plumbing: a barrier around the timed region and a MAX of the per-rank device
time, so the whole-job throughput is (units processed by all ranks) / (slowest rank's time).

Ranks come from the torchrun environment (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT). The backend is
NCCL on GPUs and gloo on CPU (the tests run two gloo ranks).
"""
import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass
class Replicas:
    world: int
    rank: int
    local: int
    backend: str = "nccl"
    _pg: bool = False

    @classmethod
    def from_env(cls, backend="nccl", timeout_s=300, device=None):
        world = int(os.environ.get("WORLD_SIZE", "1"))
        r = cls(world, int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), backend)
        if world > 1:
            import torch.distributed as dist

            kw = {"device_id": device} if device is not None and backend == "nccl" else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            r._pg = True
        return r

    def seed(self, base):
        """The seed of this rank's workload: replicas scan different data of the same shape."""
        return base + self.rank

    def barrier(self):
        if self._pg:
            import torch.distributed as dist

            dist.barrier()

    def _reduce(self, x, op):
        if not self._pg:
            return float(x)
        import torch
        import torch.distributed as dist

        dev = torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        import torch.distributed as dist

        return self._reduce(x, dist.ReduceOp.MAX if self._pg else None)

    def sum(self, x):
        import torch.distributed as dist

        return self._reduce(x, dist.ReduceOp.SUM if self._pg else None)

    def throughput(self, units_this_rank, seconds_this_rank):
        """Whole-job units per second: every rank's units over the slowest rank's time."""
        return self.sum(units_this_rank) / self.max(seconds_this_rank)

    def close(self):
        if self._pg:
            import torch.distributed as dist

            dist.destroy_process_group()
            self._pg = False
