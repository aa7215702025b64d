"""GPU tests of green_RGF_CMS (non-orthogonal basis, overlap blocks Sii;
src/green_rgf.f90:4167-4383) through the C ABI: parity with the CMS oracle,
the S = I reduction to green_RGF_RS, the Fortran-order drop-in, and the
adjoint's refusal of an overlap."""
import numpy as np
import pytest

from conftest import compare, perturbed_inputs, random_sigma, rel_err
from liteqt_b200 import synthetic as S

pytestmark = pytest.mark.gpu

MU = (0.1, -0.1)


def _temp():
    return (S.temperature_for_kT(0.025),) * 2


@pytest.fixture(scope="module")
def rgf():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf as R
    build.build()
    R.load()
    return R


OUTS = ("ldos", "ndens", "pdens", "GRi1", "GLi1", "GGi1", "cur")


def _gpu(R, d, Sii, E, opts, sl=None, sr=None):
    """All outputs (incl. GLi1 / GGi1) through rgf_solve_batch, host arrays."""
    nen, nx, nm = len(E), d.nx, d.nm
    shape = (nen, nx, nm, nm)
    o = {k: np.zeros(shape, complex) for k in OUTS if k != "cur"}
    o["cur"] = np.zeros(shape)
    for k in ("tr", "tre", "T"):
        o[k] = np.zeros(nen)
    cd = R.c_device()
    cd.nm, cd.nx = nm, nx
    cd.Hii, cd.H1i = d.Hii.ctypes.data, d.H1i.ctypes.data
    cd.Sii = None if Sii is None else Sii.ctypes.data
    cd.mu[0], cd.mu[1] = MU
    cd.temp[0], cd.temp[1] = _temp()
    tasks = []
    for e in range(nen):
        t = R.c_task()
        t.E = float(E[e])
        if sl is not None:
            t.sigma_lesser, t.sigma_r = sl[e].ctypes.data, sr[e].ctypes.data
        for k in OUTS:
            setattr(t, k, o[k][e].ctypes.data)
        for k in ("tr", "tre", "T"):
            setattr(t, k, o[k][e:].ctypes.data)
        tasks.append(t)
    info = np.zeros(nen, R.INFO_DTYPE)
    with R.Context(opts) as ctx:
        ctx.solve_batch([cd], tasks, info=info)
    assert np.all(info["status"] == 0)
    return o


def _oracle(d, Sii, E, oopts, sl=None, sr=None, extended=False, H=None):
    from oracle import oracle as O
    Hii, H1i = (d.Hii, d.H1i) if H is None else H
    return O.rgf_batch(Hii, H1i, E, MU, _temp(), oopts, sig_lesser=sl, sig_r=sr, Sii=Sii,
                       outputs=OUTS, extended=extended)


@pytest.mark.parametrize("nm,nx,consistent,scatter", [(8, 5, False, True), (32, 6, True, True),
                                                      (64, 4, False, False), (128, 3, False, True),
                                                      (48, 4, True, False)])
def test_cms_matches_oracle(rgf, nm, nx, consistent, scatter):
    from oracle import oracle as O
    d = S.make_device(nm, nx, seed=700 + nm + nx)
    Sii = S.make_overlap(nm, nx, seed=nm)
    E = S.energy_grid(5, -2.5, 2.5)
    sl = sr = None
    if scatter:
        sl, sr = random_sigma(nm, nx, len(E), seed=nx)
    opts = rgf.Options(consistent=consistent)
    oopts = O.Opts(consistent=consistent)
    g = _gpu(rgf, d, Sii, E, opts, sl, sr)
    r = _oracle(d, Sii, E, oopts, sl, sr)
    try:
        compare(g, r, nm, d.H1i)
    except AssertionError:
        x = _oracle(d, Sii, E, oopts, sl, sr, extended=True)
        floor = [_oracle(d, Sii, E, oopts, sl, sr, H=perturbed_inputs(d.Hii, d.H1i, s)) for s in range(2)]
        compare(g, r, nm, d.H1i, truth=x, floor=floor)
    assert rel_err(g["GLi1"][:, :-1], r["GLi1"][:, :-1]) < 1e-9
    assert rel_err(g["GGi1"][:, :-1], r["GGi1"][:, :-1]) < 1e-9


def test_cms_with_unit_overlap_equals_rs_on_gpu(rgf):
    """S = I: every output but G^>_ll (l < nx) and GGi1 equals the
    green_RGF_RS solve (the overlap products by I are exact)."""
    nm, nx = 32, 6
    d = S.make_device(nm, nx, seed=3)
    Sii = S._to_fortran_blocks(np.broadcast_to(np.eye(nm, dtype=complex), (nx, nm, nm)).copy())
    E = S.energy_grid(4, -1.5, 1.5)
    sl, sr = random_sigma(nm, nx, len(E), seed=1)
    opts = rgf.Options()
    rs = _gpu(rgf, d, None, E, opts, sl, sr)
    cms = _gpu(rgf, d, Sii, E, opts, sl, sr)
    for k in ("ldos", "ndens", "GRi1", "GLi1", "cur", "tr", "tre", "T"):
        assert np.array_equal(rs[k], cms[k]), k
    assert np.array_equal(rs["pdens"][:, -1], cms["pdens"][:, -1])
    assert not np.allclose(rs["pdens"][:, :-1], cms["pdens"][:, :-1])


def test_green_rgf_cms_drop_in(rgf):
    from oracle import oracle as O
    nm, nx = 16, 4
    d = S.make_device(nm, nx, seed=9)
    Sii = S.make_overlap(nm, nx, seed=2)
    sl, sr = random_sigma(nm, nx, 1, seed=5)
    E = 0.37
    shape = (nx, nm, nm)
    ndens, pdens, ldos = (np.zeros(shape, complex) for _ in range(3))
    cur = np.zeros(shape)
    GRi1 = np.zeros(shape, complex)
    tr, tre = np.zeros(1), np.zeros(1)
    rgf.green_RGF_CMS(np.array(_temp()), nm, nx, E, MU, Sii, d.Hii, d.H1i, sl[0], sl[0], sr[0],
                      ndens, pdens, ldos, tr, tre, cur, GRi1=GRi1)
    r = O.rgf_batch(d.Hii, d.H1i, np.array([E]), MU, _temp(), O.Opts(), sig_lesser=sl, sig_r=sr, Sii=Sii)
    assert rel_err(ldos, r["ldos"][0]) < 1e-10
    assert rel_err(ndens, r["ndens"][0]) < 1e-10
    assert rel_err(pdens, r["pdens"][0], scale=np.max(np.abs(r["ldos"]))) < 1e-10
    assert rel_err(GRi1[:-1], r["GRi1"][0, :-1]) < 1e-10
    trs = max(abs(r["tr"][0]), abs(r["tre"][0]), 1e-300)
    assert abs(tr[0] - r["tr"][0]) < 1e-10 * trs and abs(tre[0] - r["tre"][0]) < 1e-10 * trs


def test_adjoint_refuses_an_overlap(rgf):
    d = S.make_device(8, 3, seed=1)
    Sii = S.make_overlap(8, 3)
    cd = rgf.c_device()
    cd.nm, cd.nx = 8, 3
    cd.Hii, cd.H1i, cd.Sii = d.Hii.ctypes.data, d.H1i.ctypes.data, Sii.ctypes.data
    cd.temp[0] = cd.temp[1] = 300.0
    E = np.array([0.1, 0.2])
    T = np.zeros(2)
    with rgf.Context(rgf.Options()) as ctx:
        rc = rgf.load().rgf_adjoint_energies(ctx.h, rgf.ctypes.byref(cd), 2, E.ctypes.data, T.ctypes.data,
                                             None, None, 1.0, None, None, None, None)
    assert rc == rgf.RGF_E_UNSUPPORTED


def test_cms_longer_chain_matches_oracle(rgf):
    """green_RGF_CMS on a 20-block chain (nb = 64, overlap and scattering in
    every block) against the FP64 oracle within the spread of one input
    rounding, GLi1 / GGi1 included."""
    from conftest import compare_spread
    from oracle import oracle as O
    nm, nx = 64, 20
    d = S.make_device(nm, nx, seed=910)
    Sii = S.make_overlap(nm, nx, seed=911)
    E = np.array([-1.83, 0.37, 1.41])
    sl, sr = random_sigma(nm, nx, len(E), seed=912)
    g = _gpu(rgf, d, Sii, E, rgf.Options(), sl, sr)
    r = _oracle(d, Sii, E, O.Opts(), sl, sr)
    floors = [_oracle(d, Sii, E, O.Opts(), sl, sr, H=perturbed_inputs(d.Hii, d.H1i, s)) for s in range(2)]
    compare_spread(g, r, floors, nm, d.H1i)   # _gpu has checked every task status
    for k in ("GLi1", "GGi1"):
        spread = max(rel_err(f[k][:, :-1], r[k][:, :-1]) for f in floors)
        assert rel_err(g[k][:, :-1], r[k][:, :-1]) <= max(1e-9, 8.0 * spread), k
