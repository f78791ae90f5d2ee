"""Replica plumbing for one process per GPU.

The evaluator's units of work (ciphertexts, products) are independent and its
keys are replicated, so several GPUs run as replicas: every rank processes its
own batch, there is no collective on the data path, and the only collectives
are the host-side barrier around a timed region and the max-over-ranks
reduction of its device time.  The same functions run over NCCL (GPUs) and
gloo (CPU tests)."""
import os
from datetime import timedelta


def ranks():
    """(world_size, rank, local_rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=120, device=None):
    """Join the process group when WORLD_SIZE > 1 (rendezvous from MASTER_ADDR /
    MASTER_PORT); returns torch.distributed or None for a single process."""
    world, _, _ = ranks()
    if world <= 1:
        return None
    import torch.distributed as dist
    kw = {"timeout": timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def barrier(pg):
    if pg:
        pg.barrier()


def max_over_ranks(value, pg, device="cpu"):
    """The largest `value` over all ranks (the job's time for a timed region)."""
    if not pg:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, max_ms):
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return world * units_per_rank / (max_ms / 1000.0)


def replica_seed(base, rank):
    """Each replica draws its own synthetic inputs."""
    return base + rank


def finish(pg):
    if pg:
        pg.barrier()
        pg.destroy_process_group()
