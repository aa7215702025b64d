"""GPU tests of the mixed-precision form (RGF_PREC_MIXED, nb = 128).

Block level, through rgf_block_product / rgf_block_inverse:
  * the split-integer product (int8 digit products on the tensor cores,
    6 slices of 8 bits, 46-bit scaled integers) against the FP64 product:
    every element within 2^-43 n max_k |op(A)_ik| max_k |op(B)_kj| (the
    scaling is per row of op(A) and per column of op(B)), for all four op
    combinations, rows and columns of very different magnitudes, zero rows;
    the FP64 form of the same entry point to 1e-14 of sum_k |op(A)_ik|
    |op(B)_kj|;
  * the refined inverse (FP32 Gauss-Jordan + Newton-Schulz steps against the
    FP64 residual) against the FP64 inverse: max |I - X Y| within 1e-10 (the
    residual products' own accuracy, ~2^-44 n |X| |Y|) and
    the FP64 fallback for a singular and an ill-conditioned block;
  * the FP64 inverse's pivot rule on a near tie (two candidates within
    2^-20): the inverse stays accurate to rounding.

Solver level: the chain of green_RGF_RS (src/green_rgf.f90:3950-4164) in
the mixed form against the FP64 oracle at nb = 128.  Tolerance stated by
the form: T(E) (relative to max(1, T)) and the terminal current (the
energy sum of tr) within 1e-8; the contact current spectra tr / tre per
energy within 2e-8 of the batch's largest |tr|, |tre|, T; the G^R and G^<
diagonal blocks and the density within 1e-7 of their batch maximum.  At the
benchmark size (nb = 128, Nx = 100, eta = 1e-5) the measured errors are
T 1.9e-9, current 1.1e-9, tre 1.5e-8, G^R 2.3e-8, G^< 2.2e-8.
"""
import numpy as np
import pytest

from liteqt_b200 import synthetic as S

pytestmark = pytest.mark.gpu

MU = (0.1, -0.1)
TOL_T = 1e-8
TOL_TR = 2e-8
TOL_G = 1e-7


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


def _blocks(rng, count, nb=128, row_scale=False):
    """(count, nb, nb) complex blocks in the Fortran block layout (the last
    two axes are (column, row)); row_scale: rows and columns spread over
    2^-40 .. 2^40."""
    A = rng.normal(size=(count, nb, nb)) + 1j * rng.normal(size=(count, nb, nb))
    if row_scale:
        A *= 2.0 ** rng.integers(-40, 41, size=(count, 1, nb))   # rows (last axis)
        A *= 2.0 ** rng.integers(-40, 41, size=(count, nb, 1))   # columns
    return A


def _math(X):
    """Mathematical blocks of the Fortran block layout."""
    return np.swapaxes(X, -1, -2)


@pytest.mark.parametrize("conj_a,conj_b", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("row_scale", [False, True])
def test_block_product_error_bound(rgf, conj_a, conj_b, row_scale):
    import torch
    rng = np.random.default_rng(11 + 2 * conj_a + conj_b + 4 * row_scale)
    count = 6
    A = _blocks(rng, count, row_scale=row_scale)
    B = _blocks(rng, count, row_scale=row_scale)
    A[0, :, 5] = 0.0      # a zero row of A
    B[1, 7, :] = 0.0      # a zero column of B
    dev = torch.device("cuda:0")
    Ad, Bd = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
    Cm = torch.empty_like(Ad)
    Cf = torch.empty_like(Ad)
    with rgf.Context() as ctx:
        ctx.block_product(Ad, Bd, Cm, conj_a, conj_b, precision=rgf.RGF_PREC_MIXED)
        ctx.block_product(Ad, Bd, Cf, conj_a, conj_b, precision=rgf.RGF_PREC_FP64)
    torch.cuda.synchronize()
    opA = _math(A).conj().swapaxes(-1, -2) if conj_a else _math(A)
    opB = _math(B).conj().swapaxes(-1, -2) if conj_b else _math(B)
    ref = opA @ opB
    bound_f = np.abs(opA) @ np.abs(opB)
    rmax = np.max(np.maximum(np.abs(opA.real), np.abs(opA.imag)), axis=-1)
    cmax = np.max(np.maximum(np.abs(opB.real), np.abs(opB.imag)), axis=-2)
    bound_m = 128.0 * rmax[:, :, None] * cmax[:, None, :]
    gm = _math(Cm.cpu().numpy())
    gf = _math(Cf.cpu().numpy())
    with np.errstate(invalid="ignore", divide="ignore"):
        em = np.where(bound_m > 0, np.abs(gm - ref) / bound_m, np.abs(gm - ref))
        ef = np.where(bound_f > 0, np.abs(gf - ref) / bound_f, np.abs(gf - ref))
    assert np.max(em) < 2.0 ** -43, np.max(em)
    assert np.max(ef) < 1e-14, np.max(ef)
    assert np.all(gm[ref == 0.0] == 0.0)     # the zero row of A and column of B stay exact zeros


def _device_like_blocks(rng, count, nb=128, shift=0.0):
    """E - H - Sigma-like blocks: Hermitian H with the synthetic devices'
    statistics, a complex self-energy part with a negative imaginary part."""
    out = np.empty((count, nb, nb), complex)
    for b in range(count):
        X = rng.normal(0.0, 0.1, (nb, nb)) + 1j * rng.normal(0.0, 0.1, (nb, nb))
        H = np.triu(X, 1)
        H = H + H.conj().T + np.diag(rng.uniform(-0.5, 0.5, nb))
        W = rng.normal(size=(nb, nb)) + 1j * rng.normal(size=(nb, nb))
        Sig = 0.3 * (W + W.T) / np.sqrt(nb) - 0.05j * np.eye(nb)
        E = rng.uniform(-1.0, 1.0) + shift
        out[b] = (E * np.eye(nb) - H - Sig).T
    return out


def test_refined_inverse(rgf):
    import torch
    rng = np.random.default_rng(5)
    count = 8
    X = _device_like_blocks(rng, count)
    dev = torch.device("cuda:0")
    Xd = torch.from_numpy(X).to(dev)
    Ym = torch.empty_like(Xd)
    Yf = torch.empty_like(Xd)
    st = np.zeros(count, np.int32)
    with rgf.Context() as ctx:
        rc = ctx.block_inverse(Xd, Ym, status=st, precision=rgf.RGF_PREC_MIXED)
        ctx.block_inverse(Xd, Yf, precision=rgf.RGF_PREC_FP64)
    torch.cuda.synchronize()
    assert rc == 0 and np.all(st == 0), st
    Xm = _math(X)
    I = np.eye(128)
    for b in range(count):
        ym, yf = _math(Ym.cpu().numpy()[b]), _math(Yf.cpu().numpy()[b])
        res_m = np.max(np.abs(I - Xm[b] @ ym))
        res_f = np.max(np.abs(I - Xm[b] @ yf))
        assert res_m < 1e-10, (b, res_m, res_f)
        assert np.max(np.abs(ym - yf)) < 1e-10 * np.max(np.abs(yf)), b


def test_refined_inverse_falls_back_to_fp64(rgf):
    """A singular block (zero) and one whose FP32 factorization is too poor
    for the refinement (condition number ~1e9) take the FP64 inverse: the
    zero block with RGF_ST_SINGULAR, and an accurate inverse with
    RGF_ST_REFINE_NC."""
    import torch
    rng = np.random.default_rng(9)
    Q, _ = np.linalg.qr(rng.normal(size=(128, 128)) + 1j * rng.normal(size=(128, 128)))
    s = np.logspace(0, -9, 128)
    M = (Q * s) @ Q.conj().T
    X = np.stack([np.zeros((128, 128), complex), M.T])
    dev = torch.device("cuda:0")
    Xd = torch.from_numpy(X).to(dev)
    Y = torch.empty_like(Xd)
    st = np.zeros(2, np.int32)
    with rgf.Context() as ctx:
        rc = ctx.block_inverse(Xd, Y, status=st, precision=rgf.RGF_PREC_MIXED)
    torch.cuda.synchronize()
    assert rc == rgf.RGF_E_STATUS
    assert st[0] & 1 and np.all(Y.cpu().numpy()[0] == 0)
    assert st[1] & 8 and not st[1] & 1
    y = _math(Y.cpu().numpy()[1])
    ref = np.linalg.inv(M)
    assert np.max(np.abs(y - ref)) < 1e-4 * np.max(np.abs(ref))


@pytest.mark.parametrize("nb", [32, 64, 128])
def test_fp64_inverse_near_tie_pivot(rgf, nb):
    """The pivot search of the FP64 inverses compares the high 32 bits of
    |re| + |im|: candidates within 2^-20 tie and the first row wins, where
    LAPACK's zgetrf takes the larger.  Column 0 here has its two largest
    entries in rows 0 and 1, row 1 larger by 2^-22 (relative): the GPU
    pivots on row 0, LAPACK on row 1, and both inverses agree to rounding."""
    import torch
    rng = np.random.default_rng(nb)
    M = 0.1 * (rng.normal(size=(nb, nb)) + 1j * rng.normal(size=(nb, nb))) + np.eye(nb) * 0.5
    M[0, 0] = 3.0 + 1.0j
    M[1, 0] = (3.0 + 1.0j) * (1.0 + 2.0 ** -22)
    X = M.T[None].copy()
    dev = torch.device("cuda:0")
    Xd = torch.from_numpy(X).to(dev)
    Y = torch.empty_like(Xd)
    with rgf.Context() as ctx:
        rc = ctx.block_inverse(Xd, Y, precision=rgf.RGF_PREC_FP64)
    torch.cuda.synchronize()
    assert rc == 0
    y = _math(Y.cpu().numpy()[0])
    ref = np.linalg.inv(M)
    cond = np.linalg.cond(M)
    assert np.max(np.abs(np.eye(nb) - M @ y)) < 1e-13 * cond
    assert np.max(np.abs(y - ref)) < 1e-14 * cond * np.max(np.abs(ref))


def _solve(R, d, E, opts):
    nen = len(E)
    shape = (nen, d.nx, d.nm, d.nm)
    out = dict(ldos=np.zeros(shape, complex), ndens=np.zeros(shape, complex), tr=np.zeros(nen),
               tre=np.zeros(nen), T=np.zeros(nen))
    info = np.zeros(nen, R.INFO_DTYPE)
    with R.Context(opts) as ctx:
        rc = ctx.solve_energies(d.Hii, d.H1i, np.ascontiguousarray(E, float), MU, _temp(), info=info, **out)
        st = ctx.stats()
    out["rc"], out["info"], out["stats"] = rc, info, st
    return out


def _mixed_errors(g, r):
    trs = max(np.max(np.abs(r["tr"])), np.max(np.abs(r["tre"])), np.max(np.abs(r["T"])))
    dens_g = np.imag(np.diagonal(g["ndens"], axis1=-2, axis2=-1)).sum(-1)
    dens_r = np.imag(np.diagonal(r["ndens"], axis1=-2, axis2=-1)).sum(-1)
    return dict(
        ldos=float(np.max(np.abs(g["ldos"] - r["ldos"])) / np.max(np.abs(r["ldos"]))),
        ndens=float(np.max(np.abs(g["ndens"] - r["ndens"])) / np.max(np.abs(r["ndens"]))),
        density=float(np.max(np.abs(dens_g - dens_r)) / np.max(np.abs(dens_r))),
        T=float(np.max(np.abs(g["T"] - r["T"]) / np.maximum(1.0, np.abs(r["T"])))),
        tr=float(np.max(np.abs(g["tr"] - r["tr"])) / trs),
        tre=float(np.max(np.abs(g["tre"] - r["tre"])) / trs),
        current=float(abs(np.sum(g["tr"]) - np.sum(r["tr"])) / max(abs(np.sum(r["tr"])), 1e-300)),
    )


@pytest.mark.parametrize("nx,eta", [(6, 1e-3), (12, 1e-5)])
def test_mixed_chain_matches_oracle(rgf, nx, eta):
    from oracle import oracle as O
    d = S.make_device(128, nx, seed=700 + nx)
    E = S.energy_grid(8, -2.8, 2.8)
    g = _solve(rgf, d, E, rgf.Options(eta_dev=eta, eta_lead=eta, precision=rgf.RGF_PREC_MIXED))
    assert g["rc"] == 0 and np.all(g["info"]["status"] & ~8 == 0), g["info"]["status"]
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(eta_dev=eta, eta_lead=eta), outputs=("ldos", "ndens"))
    e = _mixed_errors(g, r)
    print("mixed vs FP64 oracle nb=128 nx=%d eta=%g: %s" % (nx, eta, {k: f"{v:.2e}" for k, v in e.items()}))
    assert e["T"] < TOL_T and e["current"] < TOL_T and e["tr"] < TOL_TR and e["tre"] < TOL_TR, e
    assert e["ldos"] < TOL_G and e["ndens"] < TOL_G and e["density"] < TOL_G, e
    assert np.array_equal(g["info"]["sancho_iters_left"], r["stats"]["sancho_iters_left"])
    assert np.all(g["info"]["mixed_pairs"] > 0)
    assert g["stats"]["last_int8_ops"] > 0


def test_mixed_benchmark_workload(rgf):
    """The throughput workload (nb = 128, Nx = 100, eta = 1e-5) in the mixed
    form, on the 8 energies of the FP64 parity test, against the FP64 oracle."""
    from oracle import oracle as O
    d = S.make_device(128, 100, seed=1)
    grid = S.energy_grid(296, -3.0, 3.0)
    edges = np.concatenate([S.lead_band_edges(d.Hii, d.H1i, 0, 256),
                            S.lead_band_edges(d.Hii, d.H1i, d.nx - 1, 256)])
    dist = np.min(np.abs(grid[:, None] - edges[None, :]), axis=1)
    idx = sorted(set(np.argsort(dist)[:2]) | {5, 60, 120, 175, 230, 290})
    E = grid[idx]
    g = _solve(rgf, d, E, rgf.Options(eta_dev=1e-5, eta_lead=1e-5, precision=rgf.RGF_PREC_MIXED))
    assert g["rc"] == 0, g["info"]["status"]
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(eta_dev=1e-5, eta_lead=1e-5), outputs=("ldos", "ndens"))
    e = _mixed_errors(g, r)
    print("mixed vs FP64 oracle, benchmark workload: %s" % {k: f"{v:.2e}" for k, v in e.items()})
    assert e["T"] < TOL_T and e["current"] < TOL_T and e["tr"] < TOL_TR and e["tre"] < TOL_TR, e
    assert e["ldos"] < TOL_G and e["ndens"] < TOL_G and e["density"] < TOL_G, e
