"""GPU tests of the FFT form of the GW convolutions (rgf_gw_polarization_fft,
rgf_gw_self_energy_fft) against the oracle's restatement of the reference's
'fft' paths (oracle/gw_fft.py: corr1d2 / conv1d2 by length-(2n-1) FFTs,
src/fft_mod.f90:56-89, :175-212, summed per (k, q) pair as
src/green_rgf.f90:1397-1473 and :1598-1678 do).  Both sides are FFT
evaluations of the same sums, so they agree to FFT rounding: the bound is
1e-12 relative to each output's largest magnitude."""
import numpy as np
import pytest

from oracle import gw_fft as F

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def rgf():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf as R
    build.build()
    R.load()
    return R


def _inputs(nij, nx, nk, n, k, seed):
    rng = np.random.default_rng(seed)
    return [rng.normal(size=(nij, nx, nk, n)) + 1j * rng.normal(size=(nij, nx, nk, n)) for _ in range(k)]


def _check(got, want):
    for g, w in zip(got, want):
        scale = np.max(np.abs(w))
        assert scale > 0
        assert np.max(np.abs(g - w)) <= TOL * scale, np.max(np.abs(g - w)) / scale


@pytest.mark.parametrize("nky,nkz,nen,nm,ndiag,nij,first_ij,chunk", [
    (1, 1, 16, 4, 1, 16, 1, None),      # one k-point, the whole 4 x 4 block
    (2, 2, 12, 3, 1, 6, 2, None),       # 2 x 2 k-grid, a rank's slice starting mid-column
    (1, 4, 10, 5, 2, 10, 6, "3"),       # nky = 1, chunks of 3 lines with a ragged tail
    (3, 2, 8, 4, 0, 8, 5, "1"),         # odd nky, diagonal only, one line per chunk
    (4, 4, 64, 6, 2, 12, 13, None),     # the GW workload's 4 x 4 k-grid
])
def test_fft_convolutions_match_oracle(rgf, monkeypatch, nky, nkz, nen, nm, ndiag, nij, first_ij, chunk):
    import torch
    if chunk:
        monkeypatch.setenv("RGF_GW_FFT_CHUNK", chunk)
    nx, nk = 2, nky * nkz
    dEn, spindeg = 0.013, 2.0
    GL, GG, GR, GLt, GGt, WL, WG, WR = _inputs(nij, nx, nk, nen, 8, nen + nij)
    dev = lambda a: torch.from_numpy(a).cuda()
    out = [torch.full((nij, nx, nk, nen), complex(7.0, 7.0), dtype=torch.complex128, device="cuda")
           for _ in range(6)]
    with rgf.Context(rgf.Options()) as ctx:
        ctx.gw_polarization_fft(dev(GL), dev(GG), dev(GR), dev(GLt), dev(GGt), PL=out[0], PG=out[1], PR=out[2],
                                nky=nky, nkz=nkz, nm=nm, ndiag=ndiag, first_ij=first_ij, dEn=dEn,
                                spindeg=spindeg)
        ctx.gw_self_energy_fft(dev(GL), dev(GG), dev(GR), dev(WL), dev(WG), dev(WR), SL=out[3], SG=out[4],
                               SR=out[5], nky=nky, nkz=nkz, nm=nm, ndiag=ndiag, first_ij=first_ij, dEn=dEn)
    torch.cuda.synchronize()
    got = [o.cpu().numpy() for o in out]
    want_p = F.gw_polarization_fft(GL, GG, GR, GLt, GGt, nky, nkz, nm, ndiag, first_ij, dEn, spindeg)
    want_s = F.gw_self_energy_fft(GL, GG, GR, WL, WG, WR, nky, nkz, nm, ndiag, first_ij, dEn)
    _check(got[:3], want_p)
    _check(got[3:], want_s)
    # elements outside the band are written as zeros
    for i in range(nij):
        if not F.in_band(i, first_ij, nm, ndiag):
            for g in got:
                assert not np.any(g[i])


def test_fft_form_rejects_odd_energy_counts(rgf):
    import torch
    a = torch.zeros((1, 1, 1, 7), dtype=torch.complex128, device="cuda")
    with rgf.Context(rgf.Options()) as ctx:
        with pytest.raises(rgf.RgfError):
            ctx.gw_polarization_fft(a, a, a, a, a, PL=a, PG=a, PR=a, nky=1, nkz=1, nm=1, ndiag=0, first_ij=1,
                                    dEn=0.01, spindeg=2.0)
