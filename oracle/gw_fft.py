"""Oracle of the FFT-form GW convolutions (test infrastructure only; the
library never imports it).

The production GW loop with MPI energy <-> (i,j) redistribution,
green_rgf_solve_gw_ephoton_3d_ijs (src/green_rgf.f90:1009-2059), forms the
polarization (:1397-1468) and the GW self-energy (:1598-1672) per (i,j)
element as energy correlations / convolutions by FFT: corr1d2 and conv1d2
with method 'fft' (src/fft_mod.f90:56-89, :175-212), each a circular
convolution of length 2n - 1 by do_mkl_dfti_conv (:214-234; forward DFTs,
pointwise product, backward DFT divided by the length).  MKL's DFT is
restated with numpy's FFT (same transform; rounding differs at the 1e-16
level).

What the 'fft' paths compute (derived from the padding and windows, and
checked against the explicit sums below in tests/test_gw_fft_oracle.py):
  corr1d2:  Z(p) = sum_ie X(ie) Y(ie - b),   b = p - 1 - n/2,  p = 1..n
  conv1d2:  Z(e) = sum_nop X(e - nop) Y(nop + n/2),  |nop| <= n/2 - 1
with terms outside 1..n dropped.  (The routines' explicit-index methods use
b = p - n/2 and a narrower energy range: the 'fft' and explicit methods of
the reference are not the same function; the production loop uses 'fft'.)

Arrays use the NumPy view of the Fortran *_by_blocks layout
(nen, nk, nx, local_Nij): shape (nij, nx, nk, nen), energy fastest, with
ik = ikz + nkz * iky (0-based).  n = nen must be even (the reference's
windows assume it)."""
import numpy as np

PI = 3.14159265359   # the reference's pi (src/green_rgf.f90:23)


def dfti_conv(x, y):
    """do_mkl_dfti_conv (src/fft_mod.f90:214-234): circular convolution of
    two length-N sequences, backward transform divided by N."""
    return np.fft.ifft(np.fft.fft(x) * np.fft.fft(y))


def corr1d2_fft(X, Y):
    """corr1d2(n, X, Y, 'fft') (src/fft_mod.f90:56-89)."""
    n = len(X)
    N = 2 * n - 1
    Xp = np.zeros(N, complex)
    Yp = np.zeros(N, complex)
    Xp[:n] = X
    Yp[:n] = Y[::-1]
    return dfti_conv(Xp, Yp)[n - n // 2 - 1:n + n // 2 - 1]


def conv1d2_fft(X, Y):
    """conv1d2(n, X, Y, 'fft') (src/fft_mod.f90:175-212)."""
    n = len(X)
    N = 2 * n - 1
    Xp = np.zeros(N, complex)
    Yp = np.zeros(N, complex)
    Xp[:n] = X
    Yp[:n // 2] = Y[n // 2 - 1:n - 1]
    if n // 2 - 1 > 0:
        Yp[N - (n // 2 - 1):] = Y[:n // 2 - 1]
    return dfti_conv(Yp, Xp)[:n]


def corr1d2_sum(X, Y):
    """corr1d2 'fft' as the explicit sum it equals (small n)."""
    n = len(X)
    Z = np.zeros(n, complex)
    for p in range(n):
        b = p - n // 2
        for e in range(n):
            if 0 <= e - b < n:
                Z[p] += X[e] * Y[e - b]
    return Z


def conv1d2_sum(X, Y):
    """conv1d2 'fft' as the explicit sum it equals (small n)."""
    n = len(X)
    Z = np.zeros(n, complex)
    for e in range(n):
        for nop in range(-(n // 2 - 1), n // 2):
            if 0 <= e - nop < n:
                Z[e] += X[e - nop] * Y[nop + n // 2 - 1]
    return Z


def kd_index(ik, iq, nky, nkz):
    """0-based ikd of the k - q loops (src/green_rgf.f90:1413-1426)."""
    iky, ikz = divmod(ik, nkz)
    iqy, iqz = divmod(iq, nkz)
    ikzd = (ikz - iqz + nkz // 2 - 1) % nkz if nkz > 1 else 0
    ikyd = (iky - iqy + nky // 2 - 1) % nky if nky > 1 else 0
    return ikzd + ikyd * nkz


def in_band(i_local, first_ij, nm, ndiag):
    """The banded-element test of the loops (src/green_rgf.f90:1401-1408):
    local index i_local (0-based), first_ij the 1-based global index of the
    rank's first (i,j)."""
    g = i_local + first_ij
    col = (g - 1) // nm + 1
    row = (g - 1) % nm + 1
    return max(row - ndiag, 1) <= col <= min(nm, row + ndiag)


def gw_polarization_fft(GL, GG, GR, GLt, GGt, nky, nkz, nm, ndiag, first_ij, dEn, spindeg, corr=corr1d2_fft):
    """P^<, P^>, P^R buffers of the ijs loop (src/green_rgf.f90:1397-1468)
    times dE = -i dEn / (2 pi) * spindeg / nk (:1470-1473).  GLt / GGt are the
    transposed G^< / G^> (element (j,i)) in the same layout."""
    nij, nx, nk, nen = GL.shape
    PL, PG, PR = (np.zeros_like(GL) for _ in range(3))
    for i in range(nij):
        if not in_band(i, first_ij, nm, ndiag):
            continue
        for ix in range(nx):
            for iq in range(nk):
                for ik in range(nk):
                    kd = kd_index(ik, iq, nky, nkz)
                    PL[i, ix, iq] += corr(GL[i, ix, ik], GGt[i, ix, kd])
                    PG[i, ix, iq] += corr(GG[i, ix, ik], GLt[i, ix, kd])
                    PR[i, ix, iq] += corr(GL[i, ix, ik], np.conj(GR[i, ix, kd])) + corr(GR[i, ix, ik],
                                                                                      GLt[i, ix, kd])
    f = complex(0.0, -1.0 * dEn / 2.0 / PI) * spindeg / nk
    return PL * f, PG * f, PR * f


def gw_self_energy_fft(GL, GG, GR, WL, WG, WR, nky, nkz, nm, ndiag, first_ij, dEn, conv=conv1d2_fft):
    """Sigma^<, Sigma^>, Sigma^R buffers of the ijs loop (src/green_rgf.f90:
    1598-1672) times dE = i dEn / (2 pi) / nk, Sigma^R's imaginary part
    replaced by Im(Sigma^> - Sigma^<) / 2 (:1674-1678)."""
    nij, nx, nk, nen = GL.shape
    SL, SG, SR = (np.zeros_like(GL) for _ in range(3))
    for i in range(nij):
        if not in_band(i, first_ij, nm, ndiag):
            continue
        for ix in range(nx):
            for ik in range(nk):
                for iq in range(nk):
                    kd = kd_index(ik, iq, nky, nkz)
                    SL[i, ix, ik] += conv(GL[i, ix, kd], WL[i, ix, iq])
                    SG[i, ix, ik] += conv(GG[i, ix, kd], WG[i, ix, iq])
                    SR[i, ix, ik] += (conv(GL[i, ix, kd], WR[i, ix, iq]) + conv(GR[i, ix, kd], WL[i, ix, iq])
                                      + conv(GR[i, ix, kd], WR[i, ix, iq]))
    f = complex(0.0, dEn / 2.0 / PI) / nk
    SL, SG, SR = SL * f, SG * f, SR * f
    SR = SR.real + 1j * (SG - SL).imag / 2.0
    return SL, SG, SR
