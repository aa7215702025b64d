"""Energy sharding across ranks (one process per GPU) -- the host logic of the
multi-GPU path.

The RGF solve has no data dependence between energy points, so ranks share
no data while solving.  Like the reference's MPI energy decomposition
(src/main3d.f90:142-153: contiguous chunks, first_local_energy), each rank
takes a contiguous slice of the energy grid; unlike it, the grid need not be
a multiple of the number of ranks (the first nen % world ranks take one
extra point).  After the solve the only exchange is the reduction of the
per-energy spectra into the terminal current, the reference's
``MPI_Reduce(SUM)`` of tr / current (src/green_rgf.f90:1352-1356), here an
all-reduce over the process group.
"""
from __future__ import annotations

import numpy as np

E0 = 1.6022e-19      # green_rgf.f90:22
HBAR = 1.0546e-34    # green_rgf.f90:18
TPI = 3.14159265359 * 2.0


def shard_range(nen: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of this rank's contiguous slice of nen energies."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(nen, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def terminal_current_distributed(tr_local: np.ndarray, dE: float, spindeg: float = 1.0, nk: int = 1,
                                 group=None) -> float:
    """sum(tr)*dE*e0/tpi/hbar*e0*spindeg/nk (green_rgf.f90:2938) over all ranks'
    shards: one all-reduce of the local sums (FP64)."""
    import torch
    import torch.distributed as dist
    local = float(np.sum(tr_local))
    if dist.is_available() and dist.is_initialized():
        t = torch.tensor([local], dtype=torch.float64)
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        local = float(t.item())
    return local * dE * E0 / TPI / HBAR * E0 * spindeg / nk


def gather_spectrum(x_local: np.ndarray, nen: int, group=None) -> np.ndarray:
    """All ranks' per-energy values (tr, tre, T) in grid order."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return np.asarray(x_local, np.float64)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nloc = max(shard_range(nen, r, world)[1] - shard_range(nen, r, world)[0] for r in range(world))
    buf = torch.zeros(nloc, dtype=torch.float64)
    s, e = shard_range(nen, rank, world)
    buf[: e - s] = torch.from_numpy(np.asarray(x_local, np.float64))
    if dist.get_backend(group) == "nccl":
        buf = buf.cuda()
    out = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    full = np.empty(nen)
    for r in range(world):
        a, b = shard_range(nen, r, world)
        full[a:b] = out[r].cpu().numpy()[: b - a]
    return full
