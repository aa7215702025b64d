"""GPU tests of the GW-loop convolutions (green_rgf.f90:2944-3092):
rgf_gw_polarization and rgf_gw_self_energy against the CPU oracle
(restatements of the reference's direct banded sums and post-processing),
host and device arrays, several k-grids and band widths.  Tolerance 1e-12
relative to the largest magnitude of each output (the sums are the same in
order; only fused multiply-adds differ)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rgf():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf as R
    build.build()
    R.load()
    return R


def _arrays(rng, nk, nen, nx, nm, n):
    return [np.ascontiguousarray(rng.normal(size=(nk, nen, nx, nm, nm)) + 1j * rng.normal(size=(nk, nen, nx, nm, nm)))
            for _ in range(n)]


# the last case is too long in energy for the shared-memory staged kernels
# (the direct kernels run)
@pytest.mark.parametrize("nky,nkz,ndiag,nm,nx,nen,imag", [(1, 1, 0, 6, 3, 40, True), (2, 2, 2, 8, 4, 48, True),
                                                       (1, 3, 1, 5, 3, 64, False), (3, 1, 8, 8, 5, 33, True),
                                                       (1, 1, 0, 2, 3, 2200, True)])
def test_gw_polarization_matches_oracle(rgf, nky, nkz, ndiag, nm, nx, nen, imag):
    from oracle import oracle as O
    rng = np.random.default_rng(nm * nen)
    nk = nky * nkz
    G = _arrays(rng, nk, nen, nx, nm, 3)
    P = [np.zeros_like(G[0]) for _ in range(3)]
    with rgf.Context(rgf.Options()) as ctx:
        ctx.gw_polarization(*G, PL=P[0], PG=P[1], PR=P[2], nky=nky, nkz=nkz, ndiag=ndiag, dE=0.01,
                            spindeg=2.0, imag_only=imag)
    R = O.gw_polarization(*G, nky, nkz, ndiag, 0.01, 2.0, imag_only=imag)
    for g, r in zip(P, R):
        assert rel_err(g, r) < 1e-12
        assert np.array_equal(g == 0, r == 0)   # band and window structure


@pytest.mark.parametrize("nky,nkz,ndiag,nm,nx,nen", [(1, 2, 1, 6, 6, 40), (2, 1, 3, 5, 4, 36), (1, 1, 0, 4, 3, 30),
                                                  (1, 1, 0, 2, 3, 2200)])
def test_gw_self_energy_matches_oracle(rgf, nky, nkz, ndiag, nm, nx, nen):
    from oracle import oracle as O
    rng = np.random.default_rng(nx * 100 + nen)
    nk = nky * nkz
    G = _arrays(rng, nk, nen, nx, nm, 3)
    W = _arrays(rng, nk, nen, nx, nm, 3)
    S0 = _arrays(rng, nk, nen, nx, nm, 3)
    S = [s.copy() for s in S0]
    with rgf.Context(rgf.Options()) as ctx:
        ctx.gw_self_energy(*G, *W, SL=S[0], SG=S[1], SR=S[2], nky=nky, nkz=nkz, ndiag=ndiag, dE=0.02,
                           alpha_mix=0.3)
    R = [s.copy() for s in S0]
    O.gw_self_energy(*G, *W, *R, nky, nkz, ndiag, 0.02, 0.3)
    for g, r in zip(S, R):
        assert rel_err(g, r) < 1e-12


def test_gw_device_arrays_match_host(rgf):
    import torch
    rng = np.random.default_rng(5)
    nky, nkz, nm, nx, nen = 2, 1, 6, 4, 40
    G = _arrays(rng, 2, nen, nx, nm, 3)
    P_h = [np.zeros_like(G[0]) for _ in range(3)]
    dev = torch.device("cuda", 0)
    Gd = [torch.from_numpy(g).to(dev) for g in G]
    P_d = [torch.zeros_like(Gd[0]) for _ in range(3)]
    with rgf.Context(rgf.Options()) as ctx:
        ctx.gw_polarization(*G, PL=P_h[0], PG=P_h[1], PR=P_h[2], nky=nky, nkz=nkz, ndiag=2, dE=0.01, spindeg=1.0)
        ctx.gw_polarization(*Gd, PL=P_d[0], PG=P_d[1], PR=P_d[2], nky=nky, nkz=nkz, ndiag=2, dE=0.01, spindeg=1.0)
    torch.cuda.synchronize()
    for h, d in zip(P_h, P_d):
        assert np.array_equal(h, d.cpu().numpy())
