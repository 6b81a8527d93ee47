"""Replica plumbing for running the advection step on several GPUs of one node.

The units of work (ensemble members, served requests, whole domains) are
independent, so N GPUs run N independent replicas, one process per GPU,
with no exchange on the data path.  The only collectives are the barrier
around a timed region and the maximum of the per-rank device times, from
which the whole-job rate is formed: units of all ranks / slowest rank's
time.  torchrun (or any launcher setting RANK / WORLD_SIZE / LOCAL_RANK /
MASTER_ADDR / MASTER_PORT) starts the processes; backend "nccl" on GPUs,
"gloo" for the CPU tests of this module.
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Ranks:
    rank: int
    world: int
    local: int

    @property
    def is_root(self) -> bool:
        return self.rank == 0


def from_env() -> Ranks:
    return Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def init(r: Ranks, backend: str = "nccl", timeout_s: float = 300.0) -> None:
    """Join the process group when there is more than one rank.  A short
    timeout makes a rank that never arrives end the others' next collective
    with an error instead of a hang."""
    if r.world <= 1:
        return
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", r.local)
    dist.init_process_group(backend, rank=r.rank, world_size=r.world, timeout=timedelta(seconds=timeout_s), **kw)


def barrier(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(r: Ranks, value: float) -> float:
    """Maximum of a per-rank scalar (a device time in ms) over all ranks."""
    if r.world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Units processed by all ranks per second of the slowest rank."""
    return units_per_rank * world / max_seconds


def replica_seed(base: int, r: Ranks) -> int:
    """Each replica advances its own independently seeded inputs."""
    return base + r.rank


def finalize(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
