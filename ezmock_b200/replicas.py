"""Replica bookkeeping for runs over several GPUs of one node.

A mock does not shard (its 3D FFT would need a global transpose and fits one
B200), so N GPUs run N independent mock streams, one process per GPU, with
different seeds and no collective on the data path.  The only exchanges are
host-side: a barrier around the timed region and the maximum of the ranks'
device times, which defines the job time.
"""
import datetime
import os

SEED_STRIDE = 100000


def rank_env():
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(rank, base=1):
    """First seed of a rank's mock stream; ranks never share a seed as long as
    each makes fewer than SEED_STRIDE mocks."""
    return base + rank * SEED_STRIDE


class Replicas:
    """Process group of the replicas (None when running alone)."""

    def __init__(self, world, backend="nccl", timeout_s=300):
        self.dist = None
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def reduce_max(self, x, device="cpu"):
        """Maximum of a float over ranks (every rank receives it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def job_seconds_per_mock(t_max, n_ranks, steps):
    """Whole-job seconds per mock: every rank made `steps` mocks in at most
    `t_max` seconds of device time."""
    return t_max / (n_ranks * steps)
