"""CPU tests of the energy <-> (i,j) redistribution (energies_to_ijs_2 /
ijs_to_energies_2, green_rgf.f90:243-329): the RESHAPE-with-ORDER oracle
against the intrinsic's element-by-element definition, and two gloo ranks
exchanging through torch.distributed.all_to_all_single with the oracle's
transposes, checked against the global array they must hold."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle.redistribute import fortran_reshape_order, fortran_reshape_order_loops


@pytest.mark.parametrize("shape,order", [((2, 3, 4, 2, 3), (1, 5, 2, 3, 4)), ((3, 2, 2, 4, 2), (5, 4, 1, 3, 2)),
                                         ((2, 2, 3, 3, 2), (3, 5, 4, 2, 1)), ((2, 3, 2, 2, 4), (1, 3, 4, 5, 2))])
def test_reshape_order_oracle_matches_definition(shape, order):
    x = np.arange(int(np.prod(shape))) + 0.5j
    assert np.array_equal(fortran_reshape_order(x, shape, order), fortran_reshape_order_loops(x, shape, order))


def _np_permute(src, dst, shape, order):
    import torch
    dst.copy_(torch.from_numpy(fortran_reshape_order(src.numpy(), shape, order)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


NM, NX, NE, NK = 4, 3, 6, 2     # nm*nm = 16 (i,j) pairs, 6 energies


def _global():
    rng = np.random.default_rng(0)
    g = rng.normal(size=(NM * NM, NX, NE, NK)) + 1j * rng.normal(size=(NM * NM, NX, NE, NK))
    return g                      # g(ij, ix, ie, ik), index order as the Fortran array


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from liteqt_b200 import redistribute as R
        g = _global()
        lne, lij = NE // world, NM * NM // world
        mine = g[:, :, rank * lne:(rank + 1) * lne, :]           # energy slice of this rank
        buf = torch.from_numpy(mine.reshape(-1, order="F").copy())
        tmp0, tmp1 = torch.empty_like(buf), torch.empty_like(buf)
        R.energies_to_ijs_2(buf, tmp0, tmp1, NX, NK, lij, lne, world, permute=_np_permute)
        ijs = buf.numpy().copy()
        R.ijs_to_energies_2(buf, tmp0, tmp1, NX, NK, lij, lne, world, permute=_np_permute)
        q.put((rank, ijs, buf.numpy().copy()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_redistribute_and_back():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = _global()
    lne, lij = NE // world, NM * NM // world
    for rank, ijs, back in res:
        # after energies_to_ijs_2: (local_ne, cs, nk, nx, local_nij) = g(all E, nk, nx, my ij slice)
        got = ijs.reshape((lne, world, NK, NX, lij), order="F").reshape((NE, NK, NX, lij), order="F")
        want = np.transpose(g[rank * lij:(rank + 1) * lij], (2, 3, 1, 0))   # (ie, ik, ix, ij)
        assert np.array_equal(got, want)
        assert np.array_equal(back, g[:, :, rank * lne:(rank + 1) * lne, :].reshape(-1, order="F"))
