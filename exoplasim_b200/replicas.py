"""Runs of one process per GPU over independent replicas.

Transform instances, ensemble members and radiation columns are independent
units, so ranks exchange no data.  The reference's own decomposition splits
one model over latitude blocks with MPI reductions (mpimod.f90:243-291);
here every rank owns whole units, and the only cross-rank steps are the
barrier around a timed region and the maximum over ranks of its duration.
The functions work under any torch.distributed backend (NCCL on GPUs, gloo
on CPU) and reduce to no-ops in a single process.
"""
import torch
import torch.distributed as dist


def rank_world():
    """(rank, world size) of the current process group, (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(n, rank, world):
    """Contiguous block of n units owned by `rank`: sizes differ by at most one,
    lower ranks take the remainder, and the blocks tile range(n)."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request n={n} rank={rank} world={world}")
    q, r = divmod(n, world)
    start = rank * q + min(rank, r)
    return range(start, start + q + (1 if rank < r else 0))


def unit_seed(base, rank, unit=0, stride=1000003):
    """Seed of one unit's synthetic input: distinct across ranks and units."""
    return int(base) + int(rank) * int(stride) + int(unit)


def barrier():
    if rank_world()[1] > 1:
        dist.barrier()


def _reduce_device():
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x):
    """The largest value of x over all ranks (a timed duration in ms, say)."""
    if rank_world()[1] == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x):
    """The sum of x over all ranks (units processed, say)."""
    if rank_world()[1] == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_per_rank, ms_max):
    """Whole-job throughput: units summed over ranks / the slowest rank's time."""
    return sum_over_ranks(units_per_rank) / (ms_max / 1000.0)
