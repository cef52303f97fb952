"""Multi-GPU plumbing of the band-parallel path: one process per GPU, bands
split into contiguous slices (block H*psi and the Chebyshev filter act on
each band independently, ApplyHam_block.cpp:23-165, so no collective runs
inside the path), and the device timings reduced as the maximum over ranks.
Works over any torch.distributed backend (NCCL on GPUs, gloo on CPU)."""
from __future__ import annotations


def band_slices(nb, world):
    """Contiguous (start, count) per rank covering nb bands, the first
    nb % world ranks one band larger."""
    base, extra = divmod(int(nb), int(world))
    out, start = [], 0
    for r in range(int(world)):
        cnt = base + (1 if r < extra else 0)
        out.append((start, cnt))
        start += cnt
    return out


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def world_size():
    d = _dist()
    return d.get_world_size() if d else 1


def max_over_ranks(value, device=None):
    """The maximum of a per-rank float over all ranks (every rank gets it)."""
    d = _dist()
    if d is None or d.get_world_size() == 1:
        return float(value)
    import torch
    if device is None:
        device = "cuda" if d.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def barrier():
    d = _dist()
    if d is not None and d.get_world_size() > 1:
        d.barrier()


def weak_throughput(units_per_rank, world, seconds_max):
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return float(units_per_rank) * int(world) / float(seconds_max)
