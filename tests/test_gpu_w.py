"""GPU tests of the screened-interaction solve (green_rgf_calc_w / RGF_W,
NBC = 0) through the C ABI: parity with the CPU oracle (Coulomb V, physical
polarizations and general complex inputs), the dense known answer
W^R = (I - V P^R)^-1 V, mixed block sizes in one launch, and the drop-in.
Tolerance 1e-10 relative to the largest magnitude of each output (the W
problem is well conditioned: the FP64 oracle is within 2e-15 of its 80-bit
evaluation on these inputs)."""
import numpy as np
import pytest

from conftest import rel_err
from liteqt_b200 import synthetic as S

pytestmark = pytest.mark.gpu
TOL = 1e-10
KEYS = ("WL", "WG", "WR")


@pytest.fixture(scope="module")
def rgf():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf as R
    build.build()
    R.load()
    return R


def _gpu_w(R, Vii, V1i, PL, PG, PR):
    shape = PL.shape
    out = {k: np.zeros(shape, complex) for k in KEYS + ("WRi1",)}
    info = np.zeros(shape[0], R.INFO_DTYPE)
    with R.Context(R.Options()) as ctx:
        ctx.w_solve_energies(Vii, V1i, PL, PG, PR, WL=out["WL"], WG=out["WG"], WR=out["WR"],
                             WRi1=out["WRi1"], info=info)
    assert np.all(info["status"] == 0)
    return out, info


def _check(g, r):
    for k in KEYS:
        assert rel_err(g[k], r[k]) < TOL, k
    assert rel_err(g["WRi1"][:, :-1], r["WRi1"][:, :-1]) < TOL
    assert np.all(g["WRi1"][:, -1] == 0)   # block nx untouched


# (64, 40): the block size and chain length of the GW workload's W solves
@pytest.mark.parametrize("nm,nx", [(8, 2), (16, 7), (32, 6), (48, 5), (64, 4), (128, 3), (64, 40)])
def test_w_matches_oracle_coulomb(rgf, nm, nx):
    from oracle import oracle as O
    Vii, V1i = S.make_coulomb(nm, nx, seed=nm)
    PL, PG, PR = S.make_polarization(nm, nx, 4, seed=nx)
    g, info = _gpu_w(rgf, Vii, V1i, PL, PG, PR)
    r = O.rgf_w_batch(Vii, V1i, PL, PG, PR)
    _check(g, r)
    assert np.all(info["n_inv"] == nx)


def test_w_matches_oracle_general_inputs(rgf):
    """Non-symmetric complex V and P: the routine's transposes and the
    zeroed real part are reproduced, not only the physical case."""
    from oracle import oracle as O
    rng = np.random.default_rng(4)
    nm, nx, nE = 16, 5, 3

    def blocks(scale, shape):
        return (rng.normal(0, scale, shape) + 1j * rng.normal(0, scale, shape)).astype(complex)
    Vb = blocks(0.1, (nx, nm, nm))
    Vii = O.from_blocks(np.array([np.eye(nm) + b + b.conj().T for b in Vb]))
    V1i = O.from_blocks(blocks(0.2, (nx, nm, nm)))
    PL, PG, PR = (np.array([O.from_blocks(blocks(0.2, (nx, nm, nm))) for _ in range(nE)]) for _ in range(3))
    g, _ = _gpu_w(rgf, Vii, V1i, PL, PG, PR)
    r = O.rgf_w_batch(Vii, V1i, PL, PG, PR)
    _check(g, r)


def test_w_dense_known_answer(rgf):
    from oracle import oracle as O
    nm, nx = 24, 4
    Vii, V1i = S.make_coulomb(nm, nx, seed=1)
    PL, PG, PR = S.make_polarization(nm, nx, 2, seed=2)
    g, _ = _gpu_w(rgf, Vii, V1i, PL, PG, PR)
    for e in range(2):
        W = O.dense_w(O.to_blocks(Vii), O.to_blocks(V1i), O.to_blocks(PR[e]))
        WR, Wo = O.to_blocks(g["WR"][e]), O.to_blocks(g["WRi1"][e])
        for l in range(nx):
            s = slice(l * nm, (l + 1) * nm)
            assert np.max(np.abs(WR[l] - W[s, s])) < 1e-11 * np.max(np.abs(W))
            if l < nx - 1:
                s1 = slice((l + 1) * nm, (l + 2) * nm)
                assert np.max(np.abs(Wo[l] - W[s, s1])) < 1e-11 * np.max(np.abs(W))


def test_w_mixed_sizes_one_launch(rgf):
    """q-points with different nm / nx in one rgf_w_solve_batch launch give
    the same bits as solving each alone."""
    devs, tasks, meta = [], [], []
    for di, (nm, nx, nE) in enumerate([(32, 5, 3), (64, 3, 2), (16, 8, 4)]):
        Vii, V1i = S.make_coulomb(nm, nx, seed=di)
        PL, PG, PR = S.make_polarization(nm, nx, nE, seed=10 + di)
        cd = rgf.c_w_device()
        cd.nm, cd.nx = nm, nx
        cd.Vii, cd.V1i = Vii.ctypes.data, V1i.ctypes.data
        devs.append(cd)
        out = {k: np.zeros(PL.shape, complex) for k in KEYS}
        for e in range(nE):
            t = rgf.c_w_task()
            t.device = di
            t.PL, t.PG, t.PR = PL[e].ctypes.data, PG[e].ctypes.data, PR[e].ctypes.data
            t.WL, t.WG, t.WR = (out[k][e].ctypes.data for k in KEYS)
            tasks.append(t)
        meta.append((Vii, V1i, PL, PG, PR, out))
    DA = (rgf.c_w_device * len(devs))(*devs)
    TA = (rgf.c_w_task * len(tasks))(*tasks)
    with rgf.Context(rgf.Options()) as ctx:
        n0 = ctx.stats()["launches"]
        rc = rgf.load().rgf_w_solve_batch(ctx.h, DA, len(devs), TA, len(tasks), None, None)
        assert rc == 0 and ctx.stats()["launches"] - n0 == 1
    for Vii, V1i, PL, PG, PR, out in meta:
        alone, _ = _gpu_w(rgf, Vii, V1i, PL, PG, PR)
        for k in KEYS:
            assert np.array_equal(out[k], alone[k]), k


def test_green_rgf_calc_w_drop_in(rgf):
    from oracle import oracle as O
    nm, nx = 16, 4
    Vii, V1i = S.make_coulomb(nm, nx, seed=6)
    PL, PG, PR = S.make_polarization(nm, nx, 1, seed=6)
    WL, WG, WR, WRi1 = (np.zeros((nx, nm, nm), complex) for _ in range(4))
    rgf.green_rgf_calc_w(0, nm, nx, Vii, V1i, PL[0], PG[0], PR[0], WL, WG, WR, WRi1=WRi1)
    r = O.rgf_w_batch(Vii, V1i, PL, PG, PR)
    for k, v in (("WL", WL), ("WG", WG), ("WR", WR)):
        assert rel_err(v, r[k][0]) < TOL, k
    assert rel_err(WRi1[:-1], r["WRi1"][0, :-1]) < TOL
    with pytest.raises(rgf.RgfError, match="NBC"):
        rgf.green_rgf_calc_w(1, nm, nx, Vii, V1i, PL[0], PG[0], PR[0], WL, WG, WR)
