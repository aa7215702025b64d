"""Energy <-> (i,j) redistribution of the GW loop across ranks (one rank per
GPU): the reference's energies_to_ijs_2 / ijs_to_energies_2
(src/green_rgf.f90:243-329).  Each is a local transpose, an all-to-all of
equal blocks (MPI_Alltoall there; torch.distributed.all_to_all_single here,
NCCL on GPUs), and a second local transpose.  The transposes run on the GPU
(rgf_permute_c16); `permute` can be replaced by another implementation of
the same Fortran RESHAPE(..., ORDER=) (the CPU tests pass the oracle's).

Layouts (column-major, cs = number of ranks):
  energies_to_ijs_2:  buf (local_nij, cs, nx, local_ne, nk)  = g(nm*nm, nx, local_ne, nk)
                   -> buf (local_ne, cs, nk, nx, local_nij)  = g(all ne, nk, nx, local_nij)
  ijs_to_energies_2:  the inverse.
"""
from __future__ import annotations


def _gpu_permute(ctx):
    def permute(src, dst, src_shape, order):
        ctx.permute(src, dst, src_shape, order, stream=None)
    return permute


def _exchange(tmp0, tmp1, group):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_to_all_single(tmp1, tmp0, group=group)
    else:
        tmp1.copy_(tmp0)


def energies_to_ijs_2(buf, tmp0, tmp1, nx, nk, local_nij, local_ne, comm_size, group=None,
                      permute=None, ctx=None):
    """buf, tmp0, tmp1: flat complex128 tensors of local_nij*cs*nx*local_ne*nk
    elements (buf is overwritten with the result, as in the reference)."""
    permute = permute or _gpu_permute(ctx)
    permute(buf, tmp0, (local_nij, comm_size, nx, local_ne, nk), (1, 5, 2, 3, 4))   # :259-261
    _exchange(tmp0, tmp1, group)                                                      # :267-268
    permute(tmp1, buf, (local_nij, nx, local_ne, nk, comm_size), (5, 4, 1, 3, 2))    # :271-273


def ijs_to_energies_2(buf, tmp0, tmp1, nx, nk, local_nij, local_ne, comm_size, group=None,
                      permute=None, ctx=None):
    """Inverse of energies_to_ijs_2 (green_rgf.f90:306-329)."""
    permute = permute or _gpu_permute(ctx)
    permute(buf, tmp0, (local_ne, comm_size, nk, nx, local_nij), (3, 5, 4, 2, 1))    # :316-318
    _exchange(tmp0, tmp1, group)                                                      # :321-322
    permute(tmp1, buf, (local_nij, nx, local_ne, nk, comm_size), (1, 3, 4, 5, 2))    # :325-327
