"""One process per GPU: rank discovery, the timing reduction, and how independent work is split.

The SPH step of one simulation does not shard (one instance is one GPU).  What does split is a set
of independent units -- batch instances or served requests -- and those need no exchange on the
data path: each rank runs its share, and only the timing and the counters are combined (max of
the device times, sum of the work), outside the timed region.
"""
import os


class Ranks:
    def __init__(self, world=1, rank=0, local=0):
        self.world = world
        self.rank = rank
        self.local = local

    @classmethod
    def from_env(cls):
        return cls(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                   int(os.environ.get("LOCAL_RANK", "0")))

    def init(self, backend="nccl", timeout_s=300):
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, init_method="env://", timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def finish(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()

    def reduce_timing(self, ms, counts=(), device="cpu"):
        """(max over ranks of `ms`, [sum over ranks of each count])."""
        if self.world == 1:
            return float(ms), [float(c) for c in counts]
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
        c = torch.tensor([float(x) for x in counts] or [0.0], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
        return float(t[0]), [float(x) for x in c[: len(counts)]]

    def gather(self, obj):
        """Every rank's `obj`, in rank order (host objects; outside the timed region)."""
        if self.world == 1:
            return [obj]
        import torch.distributed as dist
        out = [None] * self.world
        dist.all_gather_object(out, obj)
        return out


def partition(weights, world):
    """Split item indices over `world` ranks, balancing the summed weight: heaviest first onto the
    least-loaded rank (ties to the lower rank), each share in its original order.  Deterministic,
    so every rank computes the same split without communicating."""
    loads = [0.0] * world
    shares = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda k: (-weights[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        shares[r].append(i)
        loads[r] += weights[i]
    return [sorted(s) for s in shares]
