"""CPU oracle for the RGF hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline / ``--impl
reference`` legs of bench.py import this module, and only as the checker or
the timed CPU baseline.  The product library never calls it.

Parity status: *unpinned by reference outputs*.  The reference (Fortran 90 +
MKL) cannot be built here and ships no tests or golden outputs.  The oracle
is pinned instead by known answers (dense inverse of the whole device,
Sancho fixed point, integer transmission of a uniform chain, current
conservation) and by the two restatements agreeing with each other:

* ``rgf_oracle.cpp`` (C++ + OpenBLAS), the fast one, built into
  ``oracle/_build/librgf_oracle.so``;
* ``rgf_numpy`` below, an independent NumPy restatement of the same
  reference routines, for small cases.

Reference routines followed (paths relative to the liteQT tree):
``green_RGF_RS`` src/green_rgf.f90:3950-4164, ``sancho`` :4451-4537,
``invert`` :4421-4441, ``ferm`` :4444-4447, Caroli T(E) src/green.f90:2571-2580,
``calc_n_electron`` src/green_rgf.f90:3920-3945.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "librgf_oracle.so")

# Constants of the reference (src/green_rgf.f90:16-24, :3968; src/parameters.f90:38)
BOLTZ_RGF_RS = 8.61734e-05
BOLTZ_RGF_G = 8.617333262e-05
E0 = 1.6022e-19
HBAR = 1.0546e-34
PI = 3.14159265359
TPI = 3.14159265359 * 2.0

ST_SINGULAR = 1
ST_SANCHO_NC = 2
ST_BAD_ARGS = 4


class OracleOpts(ctypes.Structure):
    _fields_ = [
        ("eta_dev", ctypes.c_double),
        ("eta_lead", ctypes.c_double),
        ("boltz", ctypes.c_double),
        ("sancho_tol", ctypes.c_double),
        ("sancho_nmax", ctypes.c_int32),
        ("consistent", ctypes.c_int32),
        ("want_T", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


class OracleStat(ctypes.Structure):
    _fields_ = [
        ("sancho_iters_left", ctypes.c_int32),
        ("sancho_iters_right", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("n_gemm", ctypes.c_int32),
        ("n_inv", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


STAT_DTYPE = np.dtype([("sancho_iters_left", "<i4"), ("sancho_iters_right", "<i4"),
                       ("status", "<i4"), ("n_gemm", "<i4"), ("n_inv", "<i4"), ("pad", "<i4")])


@dataclass
class Opts:
    """Mirror of the reference's behaviour switches.

    Defaults reproduce green_RGF_RS exactly: device eta 0 (z = dcmplx(E,0.0d-6),
    green_rgf.f90:3974), lead eta 1e-3 (:4474), BOLTZ 8.61734e-5 (:3968),
    Sancho TOL 1e-100 (:4457) and nmax 100 (:4473), reference H1i indexing in
    the backward sweep (consistent=False).
    """
    eta_dev: float = 0.0
    eta_lead: float = 1e-3
    boltz: float = BOLTZ_RGF_RS
    sancho_tol: float = 1e-100
    sancho_nmax: int = 100
    consistent: bool = False
    want_T: bool = True

    def c(self) -> OracleOpts:
        return OracleOpts(self.eta_dev, self.eta_lead, self.boltz, self.sancho_tol,
                          int(self.sancho_nmax), int(self.consistent), int(self.want_T), 0)


def blas_path() -> str:
    import scipy
    pats = [os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "libscipy_openblas*.so")]
    for p in pats:
        hits = sorted(glob.glob(p))
        if hits:
            return os.path.abspath(hits[0])
    raise RuntimeError("scipy's bundled OpenBLAS was not found")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "rgf_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "_build/librgf_oracle.so"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_init.argtypes = [ctypes.c_char_p]
        L.oracle_init.restype = ctypes.c_int
        rc = L.oracle_init(blas_path().encode())
        if rc != 0:
            raise RuntimeError(f"oracle_init failed ({rc})")
        P = ctypes.c_void_p
        L.oracle_rgf_energy.argtypes = [ctypes.POINTER(OracleOpts), ctypes.c_int64, ctypes.c_int64,
                                        ctypes.c_double] + [P] * 17 + [ctypes.POINTER(OracleStat)]
        L.oracle_rgf_energy.restype = ctypes.c_int
        L.oracle_rgf_batch.argtypes = [ctypes.POINTER(OracleOpts), ctypes.c_int64, ctypes.c_int64,
                                       ctypes.c_int64] + [P] * 19 + [ctypes.c_int, ctypes.c_int]
        L.oracle_rgf_batch.restype = ctypes.c_int
        L.oracle_rgf_w_batch.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64] + [P] * 10 + \
            [ctypes.c_int, ctypes.c_int]
        L.oracle_rgf_w_batch.restype = ctypes.c_int
        I64 = ctypes.c_int64
        L.oracle_gw_polarization.argtypes = [I64] * 6 + [ctypes.c_double, ctypes.c_double, ctypes.c_int] + \
            [P] * 6 + [ctypes.c_int]
        L.oracle_gw_polarization.restype = None
        L.oracle_gw_self_energy.argtypes = [I64] * 6 + [ctypes.c_double, ctypes.c_double, ctypes.c_int] + \
            [P] * 9 + [ctypes.c_int]
        L.oracle_gw_self_energy.restype = None
        L.oracle_calc_n_electron.argtypes = [P, P, ctypes.c_int64, P, ctypes.c_int64,
                                             ctypes.c_int64, ctypes.c_int64, P, P, P]
        L.oracle_calc_n_electron.restype = None
        L.oracle_calc_block_current.argtypes = [P, P, ctypes.c_int64, P, ctypes.c_double,
                                                ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                                ctypes.c_int64, P, P, P]
        L.oracle_calc_block_current.restype = None
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _fortran3(a, nm, nx, dtype=np.complex128):
    """Return a C-contiguous (nx, nm, nm) array whose memory is the Fortran
    (nm, nm, nx) column-major layout: element (i, j, l) at i + j*nm + l*nm^2."""
    a = np.ascontiguousarray(a, dtype=dtype)
    assert a.shape[-3:] == (nx, nm, nm), a.shape
    return a


def rgf_batch(Hii, H1i, E, mu, temp, opts: Opts | None = None, sig_lesser=None, sig_r=None,
              outputs=("ldos", "ndens", "pdens", "cur", "GRi1"), threads: int | None = None,
              extended: bool = False, Sii=None):
    """Run the C++ oracle over a batch of energies.

    Sii=None: green_RGF_RS (S = I).  Sii given (same layout as Hii):
    green_RGF_CMS (green_rgf.f90:4167-4383).  outputs may also name "GLi1"
    and "GGi1".

    extended=False: FP64 with OpenBLAS, the reference's arithmetic.
    extended=True: the same algorithm in x87 80-bit long double with plain
    loops (ground truth for accuracy statements; small cases only).

    Arrays use the *block-major* NumPy view of the Fortran layout: shape
    (nx, nm, nm) with the last two axes (col, row) -- i.e. ``X[l].T`` is the
    mathematical block.  Use ``to_blocks`` / ``from_blocks`` to convert.
    Returns a dict of outputs plus 'tr', 'tre', 'T', 'stats'.
    """
    opts = opts or Opts()
    nx, nm, _ = Hii.shape
    E = np.ascontiguousarray(E, dtype=np.float64)
    nE = E.shape[0]
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    temp = np.ascontiguousarray(temp, dtype=np.float64)
    Hii = _fortran3(Hii, nm, nx)
    H1i = _fortran3(H1i, nm, nx)
    sl = None if sig_lesser is None else np.ascontiguousarray(sig_lesser, dtype=np.complex128)
    sr = None if sig_r is None else np.ascontiguousarray(sig_r, dtype=np.complex128)
    Sii = None if Sii is None else _fortran3(Sii, nm, nx)
    out = {}
    for name in ("ldos", "ndens", "pdens", "GRi1", "GLi1", "GGi1"):
        out[name] = np.zeros((nE, nx, nm, nm), np.complex128) if name in outputs else None
    out["cur"] = np.zeros((nE, nx, nm, nm), np.float64) if "cur" in outputs else None
    tr = np.zeros(nE)
    tre = np.zeros(nE)
    T = np.zeros(nE)
    stats = np.zeros(nE, STAT_DTYPE)
    if threads is None:
        threads = os.cpu_count() or 1
    o = opts.c()
    rc = lib().oracle_rgf_batch(ctypes.byref(o), nm, nx, nE, _p(E), _p(mu), _p(temp), _p(Sii),
                                _p(Hii), _p(H1i), _p(sl), _p(sr), _p(out["ndens"]), _p(out["pdens"]),
                                _p(out["ldos"]), _p(tr), _p(tre), _p(out["cur"]), _p(out["GRi1"]),
                                _p(out["GLi1"]), _p(out["GGi1"]), _p(T), _p(stats), int(threads),
                                int(extended))
    out.update(tr=tr, tre=tre, T=T, stats=stats, status=rc)
    return out


def rgf_w_batch(Vii, V1i, PL, PG, PR, threads: int | None = None, extended: bool = False):
    """green_rgf_calc_w / RGF_W (NBC = 0, no off-diagonal P) over a batch.

    Vii, V1i: (nx, nm, nm) Fortran block layout; PL, PG, PR: (nE, nx, nm, nm).
    Returns dict WL, WG, WR, WRi1 (nE, nx, nm, nm; WRi1 block nx zero) and
    'stats'."""
    nx, nm, _ = Vii.shape
    Vii = _fortran3(Vii, nm, nx)
    V1i = _fortran3(V1i, nm, nx)
    PL, PG, PR = (np.ascontiguousarray(a, np.complex128) for a in (PL, PG, PR))
    nE = PL.shape[0]
    out = {k: np.zeros((nE, nx, nm, nm), np.complex128) for k in ("WL", "WG", "WR", "WRi1")}
    stats = np.zeros(nE, STAT_DTYPE)
    rc = lib().oracle_rgf_w_batch(nm, nx, nE, _p(Vii), _p(V1i), _p(PL), _p(PG), _p(PR), _p(out["WL"]),
                                  _p(out["WG"]), _p(out["WR"]), _p(out["WRi1"]), _p(stats),
                                  int(threads or os.cpu_count() or 1), int(extended))
    out.update(stats=stats, status=rc)
    return out


def rgf_w_numpy(Vb, V1b, PLb, PGb, PRb):
    """One W solve of green_rgf_calc_w (NBC = 0, no off-diagonal P) on
    mathematical blocks (l = 0..nx-1; V1b[l] is V1i(:,:,l+1) = V_{l+1,l})."""
    nx, nm, _ = Vb.shape
    I = np.eye(nm)
    M = [I - Vb[i] @ PRb[i] for i in range(nx)]
    M1i = [-V1b[i] @ PRb[i] for i in range(nx - 1)]
    Mi1 = [-V1b[i].conj().T @ PRb[i + 1] for i in range(nx - 1)]
    xlr = [None] * nx
    Wlr = [None] * nx
    xlr[-1] = np.linalg.inv(M[-1])
    Wlr[-1] = xlr[-1] @ Vb[-1]
    for i in range(nx - 2, -1, -1):
        B = Mi1[i] @ xlr[i + 1]
        xlr[i] = np.linalg.inv(M[i] - B @ M1i[i])
        Wlr[i] = xlr[i] @ (Vb[i] - B @ V1b[i])
    WR = [None] * nx
    Wo = [None] * (nx - 1)
    WR[0] = Wlr[0]
    Wo[0] = (V1b[0].T - WR[0] @ M1i[0].T) @ xlr[1].T
    for i in range(1, nx):
        WR[i] = Wlr[i] - xlr[i] @ M1i[i - 1] @ Wo[i - 1]
        if i < nx - 1:
            Wo[i] = (V1b[i].T - WR[i] @ M1i[i].T) @ xlr[i + 1].T
    Wi = [1j * w.imag for w in Wo]
    WL, WG = [], []
    for P, out in ((PLb, WL), (PGb, WG)):
        for i in range(nx):
            jo, jp = (i, i + 1) if i < nx - 1 else (nx - 2, nx - 1)
            m = max(i - 1, 0)
            out.append(WR[i] @ P[i] @ WR[i].conj().T + Wi[jo] @ P[jp] @ (-Wi[jo]).T
                       + Wi[m].T @ P[m] @ (-Wi[m]))
    return dict(WR=np.array(WR), WRi1=np.array(Wo), WL=np.array(WL), WG=np.array(WG))


def dense_w(Vb, V1b, PRb):
    """Known answer: W^R = (I - V P^R)^-1 V of the whole (truncated) device,
    V block-tridiagonal with V_{l+1,l} = V1b[l], V_{l,l+1} = V1b[l]^H and
    P^R block-diagonal."""
    nx, nm, _ = Vb.shape
    N = nx * nm
    V = np.zeros((N, N), complex)
    P = np.zeros((N, N), complex)
    for l in range(nx):
        s = slice(l * nm, (l + 1) * nm)
        V[s, s] = Vb[l]
        P[s, s] = PRb[l]
        if l < nx - 1:
            s1 = slice((l + 1) * nm, (l + 2) * nm)
            V[s1, s] = V1b[l]
            V[s, s1] = V1b[l].conj().T
    return np.linalg.solve(np.eye(N) - V @ P, V)


def gw_polarization(GL, GG, GR, nky, nkz, ndiag, dE, spindeg, imag_only=True, threads=None):
    """P^<, P^>, P^R of green_rgf_solve_gw_3d (green_rgf.f90:2944-2999).
    G arrays (nk, nen, nx, nm, nm): the NumPy view of the Fortran
    (nm,nm,nx,nen,nk) layout.  Returns (PL, PG, PR) in the same layout."""
    GL, GG, GR = (np.ascontiguousarray(a, np.complex128) for a in (GL, GG, GR))
    nk, nen, nx, nm, _ = GL.shape
    out = [np.zeros_like(GL) for _ in range(3)]
    lib().oracle_gw_polarization(nm, nx, nen, nky, nkz, ndiag, float(dE), float(spindeg), int(imag_only),
                                 _p(GL), _p(GG), _p(GR), _p(out[0]), _p(out[1]), _p(out[2]),
                                 int(threads or os.cpu_count() or 1))
    return tuple(out)


def gw_self_energy(GL, GG, GR, WL, WG, WR, SL, SG, SR, nky, nkz, ndiag, dE, alpha_mix, imag_only=True,
                   threads=None):
    """New GW self-energies, Sigma^R's imaginary part, symmetrisation, mixing
    into SL / SG / SR (updated in place) and the edge copies
    (green_rgf.f90:3020-3092).  Same layout as gw_polarization."""
    GL, GG, GR, WL, WG, WR = (np.ascontiguousarray(a, np.complex128) for a in (GL, GG, GR, WL, WG, WR))
    for a in (SL, SG, SR):
        assert a.flags["C_CONTIGUOUS"] and a.dtype == np.complex128
    nk, nen, nx, nm, _ = GL.shape
    lib().oracle_gw_self_energy(nm, nx, nen, nky, nkz, ndiag, float(dE), float(alpha_mix), int(imag_only),
                                _p(GL), _p(GG), _p(GR), _p(WL), _p(WG), _p(WR), _p(SL), _p(SG), _p(SR),
                                int(threads or os.cpu_count() or 1))


def _kd(ik, iq, nky, nkz):
    """0-based k - q index with the reference's nk/2 shift (green_rgf.f90:2968-2977)."""
    iky, ikz = divmod(ik, nkz)
    iqy, iqz = divmod(iq, nkz)
    ikzd = (ikz - iqz + nkz // 2 - 1) % nkz if nkz > 1 else 0
    ikyd = (iky - iqy + nky // 2 - 1) % nky if nky > 1 else 0
    return ikzd + ikyd * nkz


def gw_polarization_numpy(GLm, GGm, GRm, nky, nkz, ndiag, dE, spindeg):
    """Independent vectorised restatement (small cases).  Arrays indexed
    [ik, ie, ix, i, j] with mathematical (row i, column j) blocks; real
    parts already zeroed by the caller."""
    nk, nen, nx, nm, _ = GLm.shape
    nopmax = nen // 2 - 10
    i, j = np.indices((nm, nm))
    band = np.abs(i - j) <= ndiag
    PL, PG, PR = (np.zeros_like(GLm) for _ in range(3))
    T = lambda X: np.swapaxes(X, -1, -2)
    for nop in range(-nopmax, nopmax + 1):
        iop = nop + nen // 2 - 1
        lo, hi = max(nop + 1, 1) - 1, min(nen, nen + nop)   # 0-based ie range [lo, hi)
        for iq in range(nk):
            for ik in range(nk):
                kd = _kd(ik, iq, nky, nkz)
                a = slice(lo, hi)
                b = slice(lo - nop, hi - nop)
                PL[iq, iop] += np.sum(GLm[ik, a] * T(GGm[kd, b]), axis=0)
                PG[iq, iop] += np.sum(GGm[ik, a] * T(GLm[kd, b]), axis=0)
                PR[iq, iop] += np.sum(GLm[ik, a] * np.conj(GRm[kd, b]) + GRm[ik, a] * T(GLm[kd, b]), axis=0)
    f = complex(0.0, -dE / 2.0 / 3.14159265359) * spindeg / nk
    return tuple(np.where(band, X, 0) * f for X in (PL, PG, PR))


def gw_self_energy_numpy(GLm, GGm, GRm, WLm, WGm, WRm, SLm, SGm, SRm, nky, nkz, ndiag, dE, alpha_mix):
    """Independent vectorised restatement of gw_self_energy on [ik, ie, ix,
    i, j] mathematical blocks (G real parts already zeroed).  Returns the
    updated (SL, SG, SR)."""
    nk, nen, nx, nm, _ = GLm.shape
    nopmax = nen // 2 - 10
    i, j = np.indices((nm, nm))
    band = np.abs(i - j) <= ndiag
    nL, nG, nR = (np.zeros_like(GLm) for _ in range(3))
    for ie in range(1, nen + 1):
        for ik in range(nk):
            for nop in range(-nopmax, nopmax + 1):
                if not (ie > max(nop, 1) and ie < nen + nop):
                    continue
                iop = nop + nen // 2 - 1
                for iq in range(nk):
                    kd = _kd(ik, iq, nky, nkz)
                    g, gg, gr = GLm[kd, ie - nop - 1], GGm[kd, ie - nop - 1], GRm[kd, ie - nop - 1]
                    nL[ik, ie - 1] += g * WLm[iq, iop]
                    nG[ik, ie - 1] += gg * WGm[iq, iop]
                    nR[ik, ie - 1] += g * WRm[iq, iop] + gr * WLm[iq, iop] + gr * WRm[iq, iop]
    f = complex(0.0, dE / 2.0 / 3.14159265359) / nk
    nL, nG, nR = (np.where(band, X, 0) * f for X in (nL, nG, nR))
    nR = nR.real + 1j * (nG - nL).imag / 2.0
    sym = lambda X: (X + np.swapaxes(X, -1, -2)) / 2.0
    nL, nG, nR = sym(nL), sym(nG), sym(nR)
    out = []
    for S, N in ((SLm, nL), (SGm, nG), (SRm, nR)):
        S = S + alpha_mix * (N - S)
        S[:, :, 0] = S[:, :, 2]
        S[:, :, 1] = S[:, :, 2]
        S[:, :, nx - 1] = S[:, :, nx - 3]
        S[:, :, nx - 2] = S[:, :, nx - 3]
        out.append(S)
    return tuple(out)


def calc_n_electron(G_lesser, G_greater, E, midgap):
    """calc_n_electron (green_rgf.f90:3920-3945).  G arrays: (nk, nen, nx, nm, nm)
    block-major views of the Fortran (nm,nm,nx,nen,nk) arrays."""
    nk, nen, nx, nm, _ = G_lesser.shape
    gl = np.ascontiguousarray(G_lesser, dtype=np.complex128)
    gg = np.ascontiguousarray(G_greater, dtype=np.complex128)
    E = np.ascontiguousarray(E, dtype=np.float64)
    midgap = np.ascontiguousarray(midgap, dtype=np.float64)
    ne = np.zeros(nx)
    pe = np.zeros(nx)
    lib().oracle_calc_n_electron(_p(gl), _p(gg), nen, _p(E), nm, nk, nx, _p(ne), _p(pe), _p(midgap))
    return ne, pe


def calc_block_current(H, G_lesser, E, spindeg, nb, ns, jdens=False):
    """calc_block_current (green_rgf.f90:4602-4640).  H: (nx, nm, nm) and
    G_lesser: (nen, nx, nm, nm), Fortran block layouts.  Returns tot_cur,
    tot_ecur (nx*ns, nb, nb) and jdens (nen, nx*ns, nb, nb) or None."""
    nx, nm, _ = H.shape
    nen = G_lesser.shape[0]
    Hc = np.ascontiguousarray(H, np.complex128)
    Gc = np.ascontiguousarray(G_lesser, np.complex128)
    E = np.ascontiguousarray(E, np.float64)
    tc = np.zeros((nx * ns, nb, nb))
    te = np.zeros((nx * ns, nb, nb))
    jd = np.zeros((nen, nx * ns, nb, nb)) if jdens else None
    lib().oracle_calc_block_current(_p(Hc), _p(Gc), nen, _p(E), float(spindeg), nb, ns, nm, nx,
                                    _p(tc), _p(te), _p(jd))
    return tc, te, jd


def terminal_current(tr, dE, spindeg=1.0, nk=1):
    """sum(tr)*(En(2)-En(1))*e0/tpi/hbar*e0*spindeg/nk (green_rgf.f90:2938)."""
    return float(np.sum(tr)) * dE * E0 / TPI / HBAR * E0 * spindeg / nk


# ---------------------------------------------------------------------------
# Layout helpers: NumPy (nx, nm, nm) views of Fortran (nm, nm, nx) data hold
# each block transposed.  to_blocks gives the mathematical blocks.
def to_blocks(X):
    return np.swapaxes(X, -1, -2)


def from_blocks(B):
    return np.ascontiguousarray(np.swapaxes(B, -1, -2))


def ferm(a):
    return 1.0 / (1.0 + np.exp(a))


# ---------------------------------------------------------------------------
# Independent NumPy restatement (mathematical blocks, small cases only).
def _inv(A):
    try:
        return np.linalg.inv(A), 0
    except np.linalg.LinAlgError:
        return np.zeros_like(A), ST_SINGULAR


def sancho_numpy(E, H00, H10, opts: Opts, S00=None):
    """sancho (green_rgf.f90:4451-4537) on mathematical blocks; S00 = I
    unless given (green_RGF_CMS)."""
    nm = H00.shape[0]
    z = complex(E, opts.eta_lead)
    I = np.eye(nm) if S00 is None else S00
    H_BB = H00.copy()
    H_SS = H00.copy()
    H_10 = H10.copy()
    H_01 = H_10.conj().T.copy()
    status = 0
    taken = 0
    for it in range(1, opts.sancho_nmax + 1):
        taken = it
        A, s = _inv(z * I - H_BB)
        status |= s
        B = A @ H_10
        C = H_01 @ B
        H_SS = H_SS + C
        H_BB = H_BB + C
        C = H_10 @ B
        B = A @ H_01
        A = H_10 @ B
        H_10 = C
        H_BB = H_BB + A
        C = H_01 @ B
        H_01 = C
        error = np.sum(np.abs(C))
        if abs(error) < opts.sancho_tol:
            break
        if it == opts.sancho_nmax:
            H_SS = H00.copy()
            H_BB = H00.copy()
            status |= ST_SANCHO_NC
            taken = opts.sancho_nmax + 1
    G00, s1 = _inv(z * I - H_SS)
    GBB, s2 = _inv(z * I - H_BB)
    return G00, GBB, taken, status | s1 | s2


def rgf_numpy(Hb, H1b, E, mu, temp, opts: Opts | None = None, sigl=None, sigr=None, Sb=None):
    """One energy of green_RGF_RS on mathematical blocks Hb[l], H1b[l]
    (l = 0..nx-1; H1b[l] is H1i(:,:,l+1)).  Returns dict of block lists.
    Sb (overlap blocks) given: green_RGF_CMS (green_rgf.f90:4167-4383) --
    z S_ll in place of z I, Sigma^R_ph S and Sigma^<_ph S, Sancho with the end
    blocks' S, and G^> recursed through the never-filled Glp."""
    opts = opts or Opts()
    nx, nm, _ = Hb.shape
    cms = Sb is not None
    Sl = (lambda l: Sb[l]) if cms else (lambda l: np.eye(nm))
    I = np.eye(nm)
    z = complex(E, opts.eta_dev)
    zero = np.zeros((nm, nm), complex)
    if cms:
        sl = (lambda l: sigl[l] @ Sb[l]) if sigl is not None else (lambda l: zero)
        sr = (lambda l: sigr[l] @ Sb[l]) if sigr is not None else (lambda l: zero)
    else:
        sl = (lambda l: sigl[l]) if sigl is not None else (lambda l: zero)
        sr = (lambda l: sigr[l]) if sigr is not None else (lambda l: zero)
    mul, mur = mu
    templ, tempr = temp
    H = lambda X: X.conj().T
    Gl = [None] * nx
    Gln = [None] * nx
    ldos = [None] * nx
    ndens = [None] * nx
    pdens = [None] * nx
    cur = [None] * nx
    GRi1 = [zero.copy() for _ in range(nx)]
    status = 0
    # left contact
    H00 = Hb[0] + sr(0)
    H10 = H1b[0]
    G00, _, itL, s = sancho_numpy(E, H00, H(H10), opts, Sb[0] if cms else None)
    status |= s
    sigmal = H10 @ G00 @ H(H10)
    fl = ferm((E - mul) / (opts.boltz * templ))
    sig = -(sigmal - H(sigmal)) * fl + sl(0)
    A, s = _inv(z * Sl(0) - H00 - sigmal)
    status |= s
    Gl[0] = A
    Gln[0] = A @ sig @ H(A)
    GN1 = A
    for l in range(1, nx - 1):
        H00 = Hb[l] + sr(l)
        H10 = H1b[l]
        A, s = _inv(z * Sl(l) - H00 - H10 @ Gl[l - 1] @ H(H10))
        status |= s
        Gl[l] = A
        Gln[l] = A @ (H10 @ Gln[l - 1] @ H(H10) + sl(l)) @ H(A)
        GN1 = A @ H10 @ GN1
    # right contact
    H00 = Hb[nx - 1] + sr(nx - 1)
    H10 = H1b[nx - 1]
    G00s, _, itR, s = sancho_numpy(E, H00, H10, opts, Sb[nx - 1] if cms else None)
    status |= s
    sigmar = H(H10) @ G00s @ H10
    G00, s = _inv(z * Sl(nx - 1) - H00 - sigmar - H10 @ Gl[nx - 2] @ H(H10))
    status |= s
    ldos[nx - 1] = G00
    fr = ferm((E - mur) / (opts.boltz * templ))
    sig = -(sigmar - H(sigmar)) * fr + H10 @ Gln[nx - 2] @ H(H10) + sl(nx - 1)
    Gn = G00 @ sig @ H(G00)
    ndens[nx - 1] = Gn
    Gp = Gn + (G00 - H(G00))
    pdens[nx - 1] = Gp
    B = (-(sigmar - H(sigmar)) * fr) @ Gp
    C = (-(sigmar - H(sigmar)) * (fr - 1.0)) @ Gn
    tr = -np.real(np.trace(B - C))
    gL = 1j * (sigmal - H(sigmal))
    gR = 1j * (sigmar - H(sigmar))
    X = G00 @ H10 @ GN1
    T = float(np.real(np.trace(gR @ X @ gL @ H(X))))
    # backward sweep
    for l in range(nx - 2, -1, -1):
        H10 = H1b[l + 1] if opts.consistent else H1b[l]
        g = Gl[l]
        gn = Gln[l]
        Glow = Gn @ H10 @ H(g) + G00 @ H10 @ gn         # G<_{l+1,l} (pre-multiplied below)
        c = np.real(H(H10) @ Glow)
        Gup = g @ H(H10) @ Gn + gn @ H(H10) @ H(G00)     # G<_{l,l+1}
        c = c - np.real(H10 @ Gup)
        cur[l] = c
        GN0 = g @ H(H10) @ G00
        GRi1[l] = GN0
        G00 = g + GN0 @ H10 @ g
        ldos[l] = G00
        Gn = gn + g @ H(H10) @ Gn @ H10 @ H(g) + GN0 @ H10 @ gn + gn @ H(H10) @ H(GN0)
        ndens[l] = Gn
        if cms:   # Gp = Glp + g H^H Gp H g^H + (terms with Glp = 0)
            Gp = g @ H(H10) @ Gp @ H10 @ H(g)
            pdens[l] = Gp
        else:
            pdens[l] = Gn + (G00 - H(G00))
    cur[nx - 1] = np.zeros((nm, nm))
    Gp = Gn + (G00 - H(G00))
    fl2 = ferm((E - mul) / (opts.boltz * tempr))
    B = (-(sigmal - H(sigmal)) * fl2) @ Gp
    C = (-(sigmal - H(sigmal)) * (fl2 - 1.0)) @ Gn
    tre = float(np.real(np.trace(B - C)))
    return dict(ldos=np.array(ldos), ndens=np.array(ndens), pdens=np.array(pdens),
                cur=np.array(cur), GRi1=np.array(GRi1), tr=float(tr), tre=tre, T=T,
                iters=(itL, itR), status=status, sigmal=sigmal, sigmar=sigmar)


def dense_green(Hb, H1b, E, sigmal, sigmar, eta_dev=0.0, sigr=None, Sb=None):
    """Known answer: invert the whole device (E S - H - Sigma)^-1 with the
    consistent coupling H_{l,l-1} = H1b[l] and block-diagonal overlap Sb
    (None = I; with Sb the scattering term is sigr[l] Sb[l], as in
    green_RGF_CMS).  Returns the full G^R matrix."""
    nx, nm, _ = Hb.shape
    N = nx * nm
    M = np.zeros((N, N), complex)
    Sfull = np.eye(N, dtype=complex)
    for l in range(nx):
        s = slice(l * nm, (l + 1) * nm)
        sr_l = 0 if sigr is None else (sigr[l] if Sb is None else sigr[l] @ Sb[l])
        M[s, s] = Hb[l] + sr_l
        if Sb is not None:
            Sfull[s, s] = Sb[l]
        if l > 0:
            p = slice((l - 1) * nm, l * nm)
            M[s, p] = H1b[l]
            M[p, s] = H1b[l].conj().T
    M[:nm, :nm] += sigmal
    M[-nm:, -nm:] += sigmar
    return np.linalg.inv(complex(E, eta_dev) * Sfull - M)


# ---------------------------------------------------------------------------
# Adjoint of T(E) (checker for rgf_adjoint_energies).  No counterpart in the
# reference; T is the Caroli transmission of src/green.f90:2571-2580 and the
# parameters are the per-block potential V_l (Hii(:,:,l) += V_l I, the end
# blocks also shifting their leads, which the reference builds from
# Hii(:,:,1) / Hii(:,:,nx)) and the interior coupling scale s
# (H1i(:,:,m) *= s for m = 2..nx-1, 1-based).
def _dgs_dE(g, H10, tol=1e-17, cap=400):
    """dg/dE of g = (z - H00 - H10^H g H10)^-1 by doubling of the Stein
    equation X = -g g + (g H10^H) X (H10 g)."""
    P = g @ H10.conj().T
    R = H10 @ g
    X = -g @ g
    for _ in range(cap):
        D = P @ X @ R
        X = X + D
        if not np.sum(np.abs(D)) > tol * np.sum(np.abs(X)):
            break
        P = P @ P
        R = R @ R
    return X


def adjoint_numpy(Hb, H1b, E, opts: Opts):
    """Returns T, dT/dV (nx), dT/ds on mathematical blocks (ballistic)."""
    H = lambda X: X.conj().T
    nx, nm, _ = Hb.shape
    I = np.eye(nm)
    z = complex(E, opts.eta_dev)
    gL, _, _, _ = sancho_numpy(E, Hb[0], H(H1b[0]), opts)
    gR, _, _, _ = sancho_numpy(E, Hb[-1], H1b[-1], opts)
    SL = H1b[0] @ gL @ H(H1b[0])
    SR = H(H1b[-1]) @ gR @ H1b[-1]
    SpL = -(H1b[0] @ _dgs_dE(gL, H(H1b[0])) @ H(H1b[0]))
    SpR = -(H(H1b[-1]) @ _dgs_dE(gR, H1b[-1]) @ H1b[-1])
    g = [None] * nx
    c = [None] * nx
    g[0] = np.linalg.inv(z * I - Hb[0] - SL)
    c[0] = g[0]
    for l in range(1, nx - 1):
        g[l] = np.linalg.inv(z * I - Hb[l] - H1b[l] @ g[l - 1] @ H(H1b[l]))
        c[l] = g[l] @ H1b[l] @ c[l - 1]
    GNN = np.linalg.inv(z * I - Hb[-1] - SR - H1b[-1] @ g[nx - 2] @ H(H1b[-1]))
    X = GNN @ H1b[-1] @ c[nx - 2]
    GamL = 1j * (SL - H(SL))
    GamR = 1j * (SR - H(SR))
    T = float(np.real(np.trace(GamR @ X @ GamL @ H(X))))
    W = GamL @ H(X) @ GamR
    r = [None] * nx
    k = [None] * nx
    r[-1] = GNN
    k[-1] = X
    for l in range(nx - 2, -1, -1):
        r[l] = r[l + 1] @ H1b[l + 1] @ g[l]
        k[l] = c[l] + g[l] @ H(H1b[l + 1]) @ k[l + 1]
    dV = np.array([2 * np.real(np.trace(k[l] @ W @ r[l])) for l in range(nx)])
    dV[0] += 2 * np.real(np.trace(W @ X @ SpL @ k[0])) + np.real(np.trace(GamR @ X @ (1j * (SpL - H(SpL))) @ H(X)))
    dV[-1] += 2 * np.real(np.trace(W @ r[-1] @ SpR @ X)) + np.real(np.trace((1j * (SpR - H(SpR))) @ X @ GamL @ H(X)))
    ds = 0.0
    for m in range(1, nx - 1):
        ds += 2 * np.real(np.trace(W @ r[m] @ H1b[m] @ k[m - 1]) + np.trace(W @ r[m - 1] @ H(H1b[m]) @ k[m]))
    return T, dV, float(ds)


def fd_gradient(Hii, H1i, E, mu, temp, opts: Opts, h=1e-6):
    """Central finite differences of the C++ oracle's T(E) (the reference
    algorithm in FP64) w.r.t. V_l and s.  Arrays in the Fortran block layout."""
    nx, nm, _ = Hii.shape
    E = np.atleast_1d(np.asarray(E, float))
    o = Opts(**{**opts.__dict__, "want_T": True})
    eye = np.eye(nm, dtype=complex)
    dV = np.zeros((len(E), nx))
    for l in range(nx):
        Hp = Hii.copy()
        Hm = Hii.copy()
        Hp[l] += h * eye
        Hm[l] -= h * eye
        Tp = rgf_batch(Hp, H1i, E, mu, temp, o, outputs=())["T"]
        Tm = rgf_batch(Hm, H1i, E, mu, temp, o, outputs=())["T"]
        dV[:, l] = (Tp - Tm) / (2 * h)
    Sp = H1i.copy()
    Sm = H1i.copy()
    Sp[1:nx - 1] *= (1 + h)
    Sm[1:nx - 1] *= (1 - h)
    ds = (rgf_batch(Hii, Sp, E, mu, temp, o, outputs=())["T"]
          - rgf_batch(Hii, Sm, E, mu, temp, o, outputs=())["T"]) / (2 * h)
    return dV, ds
