"""Process-group plumbing for running independent instances on several GPUs
(one process per GPU, "replicas only": no data crosses ranks; the ranks
only agree on the timed region and on the slowest rank's time).

Launched by torchrun; reads RANK, LOCAL_RANK, WORLD_SIZE and MASTER_*.
NCCL on GPUs, gloo without them (the CPU tests use gloo)."""
import datetime
import os


class Replicas:
    def __init__(self, backend=None, timeout_s=120):
        import torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.cuda = torch.cuda.is_available() and backend != "gloo"
        self.dist = None
        if self.cuda:
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend or ("nccl" if self.cuda else "gloo"),
                                    timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is None:
            return
        if self.cuda:
            self.dist.barrier(device_ids=[self.local])
        else:
            self.dist.barrier()

    def _reduce(self, x, op):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.cuda else "cpu")
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        """Largest value over the ranks (the slowest rank's time)."""
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.MAX)

    def sum(self, x):
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.SUM)

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def aggregate_rate(units_per_rank, seconds_per_rank, replicas):
    """Whole-job throughput: units summed over ranks / slowest rank's time."""
    total = replicas.sum(units_per_rank)
    slowest = replicas.max(seconds_per_rank)
    return total / slowest
