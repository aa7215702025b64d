"""GPU parity at the sizes the benchmarks run.

The other parity files compare short chains against the FP64 oracle and the
80-bit evaluation.  Here the chains and block sizes are those of the
benchmark workloads, where the 80-bit evaluation takes minutes per energy,
so the rule is conftest.compare_spread: every output within 1e-10 of the FP64
oracle (the C++ restatement of green_RGF_RS, src/green_rgf.f90:3950-4164), or
within 8x the FP64 spread of the problem -- the distance between the oracle
on the exact input and on inputs perturbed elementwise by one rounding.
Sancho-Rubio iteration counts must equal the oracle's exactly.  The spread
is the problem's conditioning, and it varies by orders of magnitude: in the
uneven launch, the 200-block nb = 64 chain at E = -1.61 eV moves its G^R by
1.2e-4 (relative) under one rounding of the input, the same chain at
0.83 eV by 3e-9.

Workloads:
  * nb = 128, Nx = 100, eta = 1e-5 in device and leads (the throughput
    benchmark), 8 energies of its 296-point grid including the two nearest a
    subband edge of either lead, with the benchmark's output set
    (G^R_ll, G^<_ll, T, tr, tre: the ballistic shortcuts of the kernel);
  * nb = 256, Nx = 64, eta = 1e-6 (the band-edge configuration in plain
    FP64) with the reference's full output set, one energy within 1e-3 eV of
    a subband edge;
  * the adjoint at nb = 64, Nx = 200 (per-block potential U[-0.2, 0.2] eV);
  * one uneven launch of devices with nb in {32, 64, 128} and Nx up to 200;
  * GLi1 / GGi1 of the green_RGF_RS path against the oracle;
  * sigma^R without sigma^< (the lowest-rank Cholesky path with an
    energy-dependent broadening) at nb = 32 and the largest block size.
"""
import numpy as np
import pytest

from conftest import compare, compare_spread, perturbed_inputs, random_sigma
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


def _gpu(R, d, E, opts, keys, sl=None, sr=None):
    nen = len(E)
    shape = (nen, d.nx, d.nm, d.nm)
    out = {k: None for k in ("ldos", "ndens", "pdens", "GRi1", "cur")}
    for k in keys:
        out[k] = np.zeros(shape, float if k == "cur" else complex)
    for k in ("tr", "tre", "T"):
        out[k] = np.zeros(nen)
    info = np.zeros(nen, R.INFO_DTYPE)
    with R.Context(opts) as ctx:
        rc = ctx.solve_energies(d.Hii, d.H1i, np.ascontiguousarray(E, float), MU, _temp(),
                                sigma_lesser=sl, sigma_r=sr, info=info, **out)
    out["rc"] = rc
    out["info"] = info
    return out


def _oracle(Hii, H1i, E, oo, sl=None, sr=None, outputs=("ldos", "ndens", "pdens", "cur", "GRi1")):
    from oracle import oracle as O
    return O.rgf_batch(Hii, H1i, np.asarray(E, float), MU, _temp(), oo, sig_lesser=sl, sig_r=sr,
                       outputs=outputs)


def _nearest_edges(d, E, count):
    edges = np.concatenate([S.lead_band_edges(d.Hii, d.H1i, 0, 256),
                            S.lead_band_edges(d.Hii, d.H1i, d.nx - 1, 256)])
    dist = np.min(np.abs(E[:, None] - edges[None, :]), axis=1)
    return list(np.argsort(dist)[:count]), edges


def _check_iters(g, r):
    assert np.array_equal(g["info"]["sancho_iters_left"], r["stats"]["sancho_iters_left"])
    assert np.array_equal(g["info"]["sancho_iters_right"], r["stats"]["sancho_iters_right"])


def test_benchmark_workload_nb128_nx100(rgf):
    from oracle import oracle as O
    nm, nx = 128, 100
    d = S.make_device(nm, nx, seed=1)          # the benchmark's device
    grid = S.energy_grid(296, -3.0, 3.0)       # the benchmark's grid
    edge_idx, _ = _nearest_edges(d, grid, 2)
    idx = sorted(set(edge_idx) | {5, 60, 120, 175, 230, 290})
    E = grid[idx]
    opts = rgf.Options(eta_dev=1e-5, eta_lead=1e-5)
    oo = O.Opts(eta_dev=1e-5, eta_lead=1e-5)
    g = _gpu(rgf, d, E, opts, ("ldos", "ndens"))
    assert g["rc"] == 0 and np.all(g["info"]["status"] == 0)
    r = _oracle(d.Hii, d.H1i, E, oo, outputs=("ldos", "ndens"))
    floors = [_oracle(*perturbed_inputs(d.Hii, d.H1i, s), E, oo, outputs=("ldos", "ndens")) for s in range(2)]
    compare_spread(g, r, floors, nm, d.H1i)
    _check_iters(g, r)


@pytest.mark.parametrize("nm,nx", [(128, 100), (256, 24)])
def test_consistent_coupling_at_size(rgf, nm, nx):
    """The consistent backward coupling H1i(:,:,l+1) on the benchmark's
    device (nb = 128, Nx = 100) and at nb = 256, eta = 1e-5: there the G^<
    recursion is stable (|G^<| ~ 1 along the chain), unlike the reference's
    coupling, whose recursion grows by ~1e110 over the 100 blocks."""
    from oracle import oracle as O
    d = S.make_device(nm, nx, seed=1)
    E = np.array([-1.7635, 0.5676, 2.3716])
    opts = rgf.Options(eta_dev=1e-5, eta_lead=1e-5, consistent=True)
    oo = O.Opts(eta_dev=1e-5, eta_lead=1e-5, consistent=1)
    g = _gpu(rgf, d, E, opts, ("ldos", "ndens"))
    assert g["rc"] == 0 and np.all(g["info"]["status"] == 0)
    r = _oracle(d.Hii, d.H1i, E, oo, outputs=("ldos", "ndens"))
    floors = [_oracle(*perturbed_inputs(d.Hii, d.H1i, s), E, oo, outputs=("ldos", "ndens")) for s in range(2)]
    compare_spread(g, r, floors, nm, d.H1i)
    _check_iters(g, r)


def test_band_edge_workload_nb256_nx64_plain(rgf):
    from oracle import oracle as O
    nm, nx = 256, 64
    d = S.make_device(nm, nx, seed=3)
    edges = S.lead_band_edges(d.Hii, d.H1i, 0, 128)
    inside = edges[np.abs(edges) < 2.5]
    E = np.array([inside[len(inside) // 2] + 4e-4, -0.77])
    opts = rgf.Options(eta_dev=1e-6, eta_lead=1e-6)
    oo = O.Opts(eta_dev=1e-6, eta_lead=1e-6)
    keys = ("ldos", "ndens", "pdens", "GRi1", "cur")
    g = _gpu(rgf, d, E, opts, keys)
    assert g["rc"] == 0 and np.all(g["info"]["status"] == 0)
    r = _oracle(d.Hii, d.H1i, E, oo)
    floors = [_oracle(*perturbed_inputs(d.Hii, d.H1i, s), E, oo) for s in range(2)]
    compare_spread(g, r, floors, nm, d.H1i)
    _check_iters(g, r)


def test_adjoint_workload_nb64_nx200(rgf):
    """The adjoint at the adjoint benchmark's sizes against the analytic
    adjoint of the oracle (NumPy) and central differences of the FP64
    oracle at five interior blocks and the coupling scale."""
    from oracle import oracle as O
    nm, nx = 64, 200
    pot = np.random.default_rng(2).uniform(-0.2, 0.2, nx)
    d = S.make_device(nm, nx, seed=1, potential=pot)
    E = np.array([-1.234, 0.517])
    oo = O.Opts(eta_dev=1e-5, eta_lead=1e-5)
    T = np.zeros(len(E))
    dTdV = np.zeros((len(E), nx))
    dTds = np.zeros(len(E))
    info = np.zeros(len(E), rgf.INFO_DTYPE)
    with rgf.Context(rgf.Options(eta_dev=1e-5, eta_lead=1e-5)) as ctx:
        ctx.adjoint_energies(d.Hii, d.H1i, E, MU, _temp(), T=T, dTdV=dTdV, dTds=dTds, spindeg=2.0,
                             info=info)
    assert np.all(info["status"] == 0)
    Hb, H1b = O.to_blocks(d.Hii), O.to_blocks(d.H1i)
    h = 1e-6
    o = O.Opts(**{**oo.__dict__, "want_T": True})
    for ie, e in enumerate(E):
        Tr, dVr, dsr = O.adjoint_numpy(Hb, H1b, e, oo)
        scale = np.max(np.abs(dVr))
        assert abs(T[ie] - Tr) < 1e-8 * max(1.0, abs(Tr))
        assert np.max(np.abs(dTdV[ie] - dVr)) < 1e-7 * scale
        assert abs(dTds[ie] - dsr) < 1e-7 * max(abs(dsr), 1.0)
        eye = np.eye(nm, dtype=complex)
        for l in (1, 57, 100, 151, 198):
            Hp, Hm = d.Hii.copy(), d.Hii.copy()
            Hp[l] += h * eye
            Hm[l] -= h * eye
            fd = (O.rgf_batch(Hp, d.H1i, np.array([e]), MU, _temp(), o, outputs=())["T"][0]
                  - O.rgf_batch(Hm, d.H1i, np.array([e]), MU, _temp(), o, outputs=())["T"][0]) / (2 * h)
            assert abs(dTdV[ie, l] - fd) < 1e-5 * scale, (l, dTdV[ie, l], fd)
        Sp, Sm = d.H1i.copy(), d.H1i.copy()
        Sp[1:nx - 1] *= (1 + h)
        Sm[1:nx - 1] *= (1 - h)
        fds = (O.rgf_batch(d.Hii, Sp, np.array([e]), MU, _temp(), o, outputs=())["T"][0]
               - O.rgf_batch(d.Hii, Sm, np.array([e]), MU, _temp(), o, outputs=())["T"][0]) / (2 * h)
        assert abs(dTds[ie] - fds) < 1e-5 * max(abs(fds), 1.0)


def test_uneven_launch_up_to_nx200(rgf):
    """Devices of the batched configuration's sizes (nb in {32, 64, 128},
    Nx up to 200) in one persistent launch, two energies each."""
    from oracle import oracle as O
    shapes = [(64, 200), (32, 200), (128, 50), (64, 20), (64, 137), (32, 64)]
    devs = [S.make_device(nb, nx, seed=900 + i) for i, (nb, nx) in enumerate(shapes)]
    E = np.array([-1.61, 0.83])
    opts = rgf.Options(eta_dev=1e-5, eta_lead=1e-5)
    oo = O.Opts(eta_dev=1e-5, eta_lead=1e-5)
    cdevs, ctasks, outs = [], [], []
    for i, d in enumerate(devs):
        cd = rgf.c_device()
        cd.nm, cd.nx = d.nm, d.nx
        cd.Hii, cd.H1i = d.Hii.ctypes.data, d.H1i.ctypes.data
        cd.mu[0], cd.mu[1] = MU
        cd.temp[0], cd.temp[1] = _temp()
        cdevs.append(cd)
        o = {k: np.zeros((len(E), d.nx, d.nm, d.nm), complex) for k in ("ldos", "ndens")}
        for k in ("tr", "tre", "T"):
            o[k] = np.zeros(len(E))
        outs.append(o)
        for ie, e in enumerate(E):
            t = rgf.c_task()
            t.device, t.E = i, float(e)
            t.ldos, t.ndens = o["ldos"][ie].ctypes.data, o["ndens"][ie].ctypes.data
            t.tr, t.tre, t.T = o["tr"][ie:].ctypes.data, o["tre"][ie:].ctypes.data, o["T"][ie:].ctypes.data
            ctasks.append(t)
    info = np.zeros(len(ctasks), rgf.INFO_DTYPE)
    with rgf.Context(opts) as ctx:
        rc = ctx.solve_batch(cdevs, ctasks, info=info)
    assert rc == 0 and np.all(info["status"] == 0)
    for i, d in enumerate(devs):
        r = _oracle(d.Hii, d.H1i, E, oo, outputs=("ldos", "ndens"))
        floors = [_oracle(*perturbed_inputs(d.Hii, d.H1i, s), E, oo, outputs=("ldos", "ndens"))
                  for s in range(2)]
        g = dict(outs[i])
        g["info"] = info[2 * i:2 * i + 2]
        compare_spread(g, r, floors, d.nm, d.H1i)
        _check_iters(g, r)


@pytest.mark.parametrize("scatter", [False, True])
def test_gli1_ggi1_rs_path(rgf, scatter):
    """G^<_{l,l+1} and the reference's GGi1 (green_rgf.f90:4094-4103) of the
    green_RGF_RS drop-in against the oracle, with and without scattering."""
    from oracle import oracle as O
    nm, nx = 32, 9
    d = S.make_device(nm, nx, seed=71)
    E = 0.41
    sl, sr = random_sigma(nm, nx, 1, seed=5) if scatter else (None, None)
    nd, pd, ld, gr, gl, gg = (np.zeros((nx, nm, nm), complex) for _ in range(6))
    cur = np.zeros((nx, nm, nm))
    tr, tre = np.zeros(1), np.zeros(1)
    rgf.green_RGF_RS(_temp(), nm, nx, E, MU, d.Hii, d.H1i, None if sl is None else sl[0], None,
                     None if sr is None else sr[0], nd, pd, ld, tr, tre, cur, GRi1=gr, GLi1=gl, GGi1=gg)
    outputs = ("ldos", "ndens", "pdens", "cur", "GRi1", "GLi1", "GGi1")
    r = _oracle(d.Hii, d.H1i, [E], O.Opts(), sl, sr, outputs=outputs)
    x = O.rgf_batch(d.Hii, d.H1i, np.array([E]), MU, _temp(), O.Opts(), sig_lesser=sl, sig_r=sr,
                    outputs=outputs, extended=True)
    g = dict(ldos=ld[None], ndens=nd[None], pdens=pd[None], GRi1=gr[None], GLi1=gl[None],
             GGi1=gg[None], cur=cur[None], tr=tr, tre=tre, T=r["T"])
    compare(g, r, nm, d.H1i, truth=x)


@pytest.mark.parametrize("nm,nx", [(32, 7), (256, 3)])
def test_sigma_r_without_sigma_lesser(rgf, nm, nx):
    """sigma^R present, sigma^< absent: the ballistic running-column path
    (pivoted Cholesky of Gamma_L) with a scattering broadening in every
    block; nb = 256 is the largest block the Cholesky handles."""
    from oracle import oracle as O
    d = S.make_device(nm, nx, seed=33 + nm)
    E = np.array([-0.93, 0.12])
    _, sr = random_sigma(nm, nx, len(E), seed=nm + 1)
    keys = ("ldos", "ndens", "pdens", "GRi1", "cur")
    g = _gpu(rgf, d, E, rgf.Options(), keys, sl=None, sr=sr)
    assert g["rc"] == 0 and np.all(g["info"]["status"] == 0)
    r = _oracle(d.Hii, d.H1i, E, O.Opts(), None, sr)
    if nm <= 64:
        x = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(), sig_r=sr, extended=True)
        compare(g, r, nm, d.H1i, truth=x)
    else:
        floors = [_oracle(*perturbed_inputs(d.Hii, d.H1i, s), E, O.Opts(), None, sr) for s in range(2)]
        compare_spread(g, r, floors, nm, d.H1i)


def test_indefinite_lead_broadening_takes_general_form(rgf):
    """sigma^R of the first block with the wrong sign of its broadening (an
    advanced self-energy) makes Gamma_L indefinite; the pivoted Cholesky
    factor of the ballistic path does not exist then, and the kernel must
    fall back to the general recursion g^< = g sigma^< g^H (four products),
    matching the oracle, which always uses it."""
    from oracle import oracle as O
    nm, nx = 16, 5
    d = S.make_device(nm, nx, seed=808)
    E = np.array([-0.41, 0.66])
    _, sr = random_sigma(nm, nx, len(E), seed=17, scale=0.2)
    sr[:, 0] = np.conj(np.swapaxes(sr[:, 0], -1, -2))   # sigma^R(1)^H: broadening of the wrong sign
    keys = ("ldos", "ndens", "pdens", "GRi1", "cur")
    g = _gpu(rgf, d, E, rgf.Options(), keys, sl=None, sr=sr)
    assert np.all(g["info"]["status"] == 0)
    r = _oracle(d.Hii, d.H1i, E, O.Opts(), None, sr)
    x = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(), sig_r=sr, extended=True)
    compare(g, r, nm, d.H1i, truth=x)


def test_concurrent_drop_in_calls_are_coalesced(rgf):
    """green_RGF_RS called per energy from 12 host threads at once, as the
    reference's `!$omp do` loop does (green_rgf.f90:2916-2925), without a
    context: the calls are queued and solved in shared batches.  Each
    thread's outputs must equal the oracle's for its own energy, and the
    solver must have run fewer launches than calls."""
    import threading
    from oracle import oracle as O
    nm, nx, nthr = 16, 6, 12
    d = S.make_device(nm, nx, seed=61)
    E = np.linspace(-2.2, 2.1, nthr)
    outs = []
    for _ in range(nthr):
        outs.append(dict(nd=np.zeros((nx, nm, nm), complex), pd=np.zeros((nx, nm, nm), complex),
                         ld=np.zeros((nx, nm, nm), complex), gr=np.zeros((nx, nm, nm), complex),
                         cur=np.zeros((nx, nm, nm)), tr=np.zeros(1), tre=np.zeros(1)))
    errors = []
    start = threading.Barrier(nthr)

    def work(k):
        try:
            o = outs[k]
            start.wait()
            rgf.green_RGF_RS(_temp(), nm, nx, E[k], MU, d.Hii, d.H1i, None, None, None, o["nd"], o["pd"],
                             o["ld"], o["tr"], o["tre"], o["cur"], GRi1=o["gr"])
        except Exception as exc:  # noqa: BLE001 - reported below
            errors.append(exc)
    threads = [threading.Thread(target=work, args=(k,)) for k in range(nthr)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    r = _oracle(d.Hii, d.H1i, E, O.Opts())
    g = dict(ldos=np.stack([o["ld"] for o in outs]), ndens=np.stack([o["nd"] for o in outs]),
             pdens=np.stack([o["pd"] for o in outs]), GRi1=np.stack([o["gr"] for o in outs]),
             cur=np.stack([o["cur"] for o in outs]), tr=np.array([o["tr"][0] for o in outs]),
             tre=np.array([o["tre"][0] for o in outs]), T=r["T"])
    compare(g, r, nm, d.H1i)
