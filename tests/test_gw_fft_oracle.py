"""CPU tests of the FFT-form GW convolution oracle (oracle/gw_fft.py) and of
the algorithm the GPU kernels use for it.

  * corr1d2 / conv1d2 'fft' (src/fft_mod.f90:56-89, :175-212) restated with
    numpy's FFT equal the explicit sums the module docstring states;
  * the k - q index matches the reference's 1-based loop arithmetic
    (src/green_rgf.f90:1413-1426);
  * the GPU's formulation -- one 3-D FFT over (ky, kz, energy) per (i,j,
    block) with the energy axis zero-padded to any length >= 2n - 1, the
    k - q sums done as products in frequency space (the y side at negated
    frequencies for the correlation), the nk/2 - 1 shift as a phase, and
    the output window read back -- reproduces the per-pair loops of the
    oracle (here in NumPy; tests/test_gpu_gw_fft.py runs the kernels)."""
import numpy as np
import pytest

from oracle import gw_fft as F


@pytest.mark.parametrize("n", [2, 4, 8, 16, 30])
def test_fft_paths_equal_their_explicit_sums(n):
    rng = np.random.default_rng(n)
    X = rng.normal(size=n) + 1j * rng.normal(size=n)
    Y = rng.normal(size=n) + 1j * rng.normal(size=n)
    assert np.allclose(F.corr1d2_fft(X, Y), F.corr1d2_sum(X, Y), rtol=0, atol=1e-12)
    assert np.allclose(F.conv1d2_fft(X, Y), F.conv1d2_sum(X, Y), rtol=0, atol=1e-12)


@pytest.mark.parametrize("nky,nkz", [(1, 1), (1, 4), (4, 4), (3, 2), (2, 5)])
def test_kd_index_matches_reference_loop(nky, nkz):
    for iky in range(1, nky + 1):
        for ikz in range(1, nkz + 1):
            for iqy in range(1, nky + 1):
                for iqz in range(1, nkz + 1):
                    ikzd = ikz - iqz + nkz // 2
                    ikyd = iky - iqy + nky // 2
                    if ikzd < 1:
                        ikzd += nkz
                    if ikzd > nkz:
                        ikzd -= nkz
                    if ikyd < 1:
                        ikyd += nky
                    if ikyd > nky:
                        ikyd -= nky
                    if nky == 1:
                        ikyd = 1
                    if nkz == 1:
                        ikzd = 1
                    ik = ikz + (iky - 1) * nkz
                    iq = iqz + (iqy - 1) * nkz
                    ikd = ikzd + (ikyd - 1) * nkz
                    assert F.kd_index(ik - 1, iq - 1, nky, nkz) == ikd - 1


def _nice(m):
    n = m
    while True:
        r = n
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return n
        n += 1


def _phase(nky, nkz, N, sign):
    """exp(sign * 2 pi i p.s / nk) over (ky, kz) frequencies, s = nk/2 - 1."""
    py = np.arange(nky)[:, None, None]
    pz = np.arange(nkz)[None, :, None]
    sy = (nky // 2 - 1) % nky if nky > 1 else 0
    sz = (nkz // 2 - 1) % nkz if nkz > 1 else 0
    return np.exp(sign * 2j * np.pi * (py * sy / nky + pz * sz / nkz)) * np.ones((1, 1, N))


def _neg(A):
    """A at negated frequencies over the last three axes."""
    return np.roll(np.flip(A, axis=(-3, -2, -1)), 1, axis=(-3, -2, -1))


def polarization_3d(GL, GG, GR, GLt, GGt, nky, nkz, nm, ndiag, first_ij, dEn, spindeg):
    nij, nx, nk, n = GL.shape
    N = _nice(2 * n - 1) + 3   # any length >= 2n - 1 works
    out = [np.zeros_like(GL) for _ in range(3)]

    def fwd(A):
        P = np.zeros((nky, nkz, N), complex)
        P[:, :, :n] = A.reshape(nky, nkz, n)
        return np.fft.fftn(P)
    for i in range(nij):
        if not F.in_band(i, first_ij, nm, ndiag):
            continue
        for ix in range(nx):
            xl, xg, xr = fwd(GL[i, ix]), fwd(GG[i, ix]), fwd(GR[i, ix])
            ygt, ylt, ycr = _neg(fwd(GGt[i, ix])), _neg(fwd(GLt[i, ix])), _neg(fwd(np.conj(GR[i, ix])))
            ph = _phase(nky, nkz, N, -1)
            for o, c in enumerate((xl * ygt, xg * ylt, xl * ycr + xr * ylt)):
                z = np.fft.ifftn(c * ph)
                b = np.arange(n) - n // 2
                out[o][i, ix] = z[:, :, b % N].reshape(nk, n)
    f = complex(0.0, -dEn / 2.0 / F.PI) * spindeg / nk
    return tuple(o * f for o in out)


def self_energy_3d(GL, GG, GR, WL, WG, WR, nky, nkz, nm, ndiag, first_ij, dEn):
    nij, nx, nk, n = GL.shape
    N = _nice(2 * n - 1) + 1
    h = n // 2
    out = [np.zeros_like(GL) for _ in range(3)]

    def fwd_g(A):
        P = np.zeros((nky, nkz, N), complex)
        P[:, :, :n] = A.reshape(nky, nkz, n)
        return np.fft.fftn(P)

    def fwd_w(A):
        A = A.reshape(nky, nkz, n)
        P = np.zeros((nky, nkz, N), complex)
        P[:, :, :h] = A[:, :, h - 1:n - 1]          # nop = 0 .. n/2 - 1
        if h > 1:
            P[:, :, N - (h - 1):] = A[:, :, :h - 1]   # nop = -(n/2 - 1) .. -1
        return np.fft.fftn(P)
    for i in range(nij):
        if not F.in_band(i, first_ij, nm, ndiag):
            continue
        for ix in range(nx):
            gl, gg, gr = fwd_g(GL[i, ix]), fwd_g(GG[i, ix]), fwd_g(GR[i, ix])
            wl, wg, wr = fwd_w(WL[i, ix]), fwd_w(WG[i, ix]), fwd_w(WR[i, ix])
            ph = _phase(nky, nkz, N, +1)
            for o, c in enumerate((gl * wl, gg * wg, gl * wr + gr * wl + gr * wr)):
                out[o][i, ix] = np.fft.ifftn(c * ph)[:, :, :n].reshape(nk, n)
    f = complex(0.0, dEn / 2.0 / F.PI) / nk
    SL, SG, SR = (o * f for o in out)
    SR = SR.real + 1j * (SG - SL).imag / 2.0
    return SL, SG, SR


def _inputs(nij, nx, nk, n, k, seed):
    rng = np.random.default_rng(seed)
    return [rng.normal(size=(nij, nx, nk, n)) + 1j * rng.normal(size=(nij, nx, nk, n)) for _ in range(k)]


@pytest.mark.parametrize("nky,nkz,n", [(1, 1, 8), (2, 2, 12), (1, 4, 10), (3, 2, 8)])
def test_gpu_formulation_reproduces_the_oracle(nky, nkz, n):
    nm, ndiag, first_ij = 3, 1, 2
    nij, nx, nk = 6, 2, nky * nkz
    GL, GG, GR, GLt, GGt = _inputs(nij, nx, nk, n, 5, 1)
    want = F.gw_polarization_fft(GL, GG, GR, GLt, GGt, nky, nkz, nm, ndiag, first_ij, 0.01, 2.0)
    got = polarization_3d(GL, GG, GR, GLt, GGt, nky, nkz, nm, ndiag, first_ij, 0.01, 2.0)
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    WL, WG, WR = _inputs(nij, nx, nk, n, 3, 2)
    want = F.gw_self_energy_fft(GL, GG, GR, WL, WG, WR, nky, nkz, nm, ndiag, first_ij, 0.01)
    got = self_energy_3d(GL, GG, GR, WL, WG, WR, nky, nkz, nm, ndiag, first_ij, 0.01)
    for a, b in zip(got, want):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    # local elements 1 and 5 are (row 3, col 1) and (row 1, col 3): outside the band, zero
    assert not F.in_band(1, first_ij, nm, ndiag) and not F.in_band(5, first_ij, nm, ndiag)
    for a in got:
        assert not np.any(a[1]) and not np.any(a[5])
