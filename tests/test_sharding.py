"""The multi-rank path on CPU: world_size-2 gloo process groups shard the
energy grid, each rank solves its shard (the CPU oracle stands in for the
per-rank GPU solve, which has no cross-rank data), and the spectra and the
terminal current are reduced -- the result must equal the single-process
one."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from liteqt_b200 import sharding


def test_shard_ranges_cover_the_grid():
    for nen in (1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            spans = [sharding.shard_range(nen, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nen
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    # the reference's case nen % world == 0 gives its contiguous chunks
    assert sharding.shard_range(12, 2, 4) == (6, 9)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from liteqt_b200 import synthetic as S
        d = S.make_device(8, 4, seed=5)
        E = S.energy_grid(11, -0.4, 0.4)
        a, b = sharding.shard_range(len(E), rank, world)
        temp = (S.temperature_for_kT(0.025),) * 2
        r = O.rgf_batch(d.Hii, d.H1i, E[a:b], (0.1, -0.1), temp, O.Opts(), outputs=(), threads=1)
        I = sharding.terminal_current_distributed(r["tr"], E[1] - E[0], spindeg=2.0)
        T = sharding.gather_spectrum(r["T"], len(E))
        q.put((rank, I, T))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_single_process():
    from oracle import oracle as O
    from liteqt_b200 import synthetic as S
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    d = S.make_device(8, 4, seed=5)
    E = S.energy_grid(11, -0.4, 0.4)
    temp = (S.temperature_for_kT(0.025),) * 2
    full = O.rgf_batch(d.Hii, d.H1i, E, (0.1, -0.1), temp, O.Opts(), outputs=(), threads=1)
    I_ref = O.terminal_current(full["tr"], E[1] - E[0], 2.0, 1)
    for _, I, T in res:
        assert abs(I - I_ref) <= 1e-12 * abs(I_ref)
        assert np.array_equal(T, full["T"])
