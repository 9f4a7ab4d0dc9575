"""Multi-GPU plumbing of the FMM-FFT: one process per GPU, each an independent replica.

The reference spreads ONE transform over P MPI ranks (src/fmmfft.c:384-978: halo exchange per
level, a complex MPI_Reduce/Bcast of the section sums at :452-453, an MPI_Alltoall at :970).  On
a B200 a whole N = 2^24..2^26 transform fits one GPU's HBM, so several GPUs serve several
transforms: every rank owns its plan, its inputs and its stream, no data-path collective runs,
and the only cross-rank traffic is the timing reduction here (max over ranks) and barriers.

Everything takes the process group as an argument so the same code runs under NCCL on GPUs and
under gloo on CPU processes (tests/test_replicas.py).
"""
import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class RankInfo:
    world: int
    rank: int
    local: int


def rank_info(env=None):
    """WORLD_SIZE / RANK / LOCAL_RANK as torchrun sets them (defaults: one rank)."""
    env = os.environ if env is None else env
    world = int(env.get("WORLD_SIZE", "1"))
    rank = int(env.get("RANK", "0"))
    local = int(env.get("LOCAL_RANK", str(rank)))
    if world < 1 or not 0 <= rank < world or local < 0:
        raise ValueError(f"bad rank layout: WORLD_SIZE={world} RANK={rank} LOCAL_RANK={local}")
    return RankInfo(world, rank, local)


def init_group(info, backend, timeout_s=120.0, device=None):
    """torch.distributed process group for `info` (None for one rank).  A short timeout makes a
    rank that never arrives end the others' next collective with an error instead of a hang."""
    if info.world == 1:
        return None
    import torch.distributed as dist
    kw = {}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s),
                            world_size=info.world, rank=info.rank, **kw)
    return dist


def replica_seed(base, rank):
    """Input seed of a replica: ranks transform different data (seed base + rank)."""
    return base + rank


def max_over_ranks(value, dist, device="cpu"):
    """max of a float over all ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank_per_step, steps, world, total_ms):
    """Whole-job throughput in units/s when every rank processed `units_per_rank_per_step` per
    step for `steps` steps and the slowest rank took `total_ms`."""
    if total_ms <= 0:
        raise ValueError("total_ms must be positive")
    return units_per_rank_per_step * steps * world / (total_ms / 1e3)


def barrier(dist):
    if dist is not None:
        dist.barrier()


def finish(dist):
    """Last barrier and teardown (every rank calls it, on the error path too)."""
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
