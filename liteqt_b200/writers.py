"""The reference's output writers (src/green_rgf.f90:4541-4896, :2937-2939)
through the library (sums on the GPU, Fortran-formatted text on the host).
Arrays use the NumPy view of the Fortran layouts: G (nk, nen, length, nm, nm),
cur (nk, nen, length, NB, NB); host NumPy or device torch arrays."""
from __future__ import annotations

import numpy as np

from . import rgf as R


def _chk(rc):
    if rc != R.RGF_OK:
        raise R.RgfError(rc, R.load().rgf_io_last_error().decode())


def _en(en):
    return np.ascontiguousarray(en, np.float64)


def write_spectrum(ctx, dataset, i, G, en, length, NB, NS, Lx, coeff, nk=1, summed_over_k=False, append=False):
    """write_spectrum / write_spectrum_summed_over_k (:4541, :4771)."""
    e = _en(en)
    c = np.ascontiguousarray(coeff, np.float64)
    _chk(R.load().rgf_write_spectrum(ctx.h, dataset.encode(), int(i), R._ptr(G), len(e), R._ptr(e), int(nk),
                                     int(length), int(NB), int(NS), float(Lx), R._ptr(c), int(summed_over_k),
                                     int(append)))


def write_dos_summed_over_k(ctx, dataset, i, G, en, nk, length, NB, NS, Lx, append=False):
    e = _en(en)
    _chk(R.load().rgf_write_dos(ctx.h, dataset.encode(), int(i), R._ptr(G), len(e), R._ptr(e), int(nk),
                                int(length), int(NB), int(NS), float(Lx), int(append)))


def write_current_spectrum(ctx, dataset, i, cur, en, length, NB, Lx, nk=1, summed_over_kz=False, append=False):
    e = _en(en)
    _chk(R.load().rgf_write_current_spectrum(ctx.h, dataset.encode(), int(i), R._ptr(cur), len(e), R._ptr(e),
                                             int(nk), int(length), int(NB), float(Lx), int(summed_over_kz),
                                             int(append)))


def write_current_summed_over_k(ctx, dataset, i, cur, nx, NB, Lx, nk):
    _chk(R.load().rgf_write_current_summed_over_k(ctx.h, dataset.encode(), int(i), R._ptr(cur), int(nx), int(NB),
                                                  float(Lx), int(nk)))


def write_transmission_spectrum(dataset, i, tr, en, nk=0, append=False):
    e = _en(en)
    t = np.ascontiguousarray(tr, np.float64)
    _chk(R.load().rgf_write_transmission_spectrum(dataset.encode(), int(i), R._ptr(t), len(e), R._ptr(e),
                                                  int(nk), int(append)))


def write_id_iteration(path, it, current_left, current_right):
    _chk(R.load().rgf_write_id_iteration(path.encode(), int(it), float(current_left), float(current_right)))


def read_ham_dat(path, axis=None):
    """w90_load_from_file (src/wannierHam.f90:68-130).  Returns (info dict,
    Hr) with Hr the NumPy view (ny, nx, nb, nb) of Hr(nb,nb,nx,ny)."""
    L = R.load()
    info = R.c_ham_info()
    ax = None if axis is None else (R.ctypes.c_int32 * 3)(*[int(a) for a in axis])
    axp = None if ax is None else R.ctypes.addressof(ax)
    _chk(L.rgf_read_ham_dat(path.encode(), axp, R.ctypes.byref(info), None))
    Hr = np.zeros((info.ny, info.nx, info.nb, info.nb), np.complex128)
    _chk(L.rgf_read_ham_dat(path.encode(), axp, R.ctypes.byref(info), Hr.ctypes.data))
    d = {k: getattr(info, k) for k, _ in R.c_ham_info._fields_ if k not in ("cell", "b1", "b2")}
    d["cell"] = np.array(info.cell[:]).reshape(3, 3)   # rows: alpha, beta, gamm
    d["b1"], d["b2"] = np.array(info.b1[:]), np.array(info.b2[:])
    return d, Hr
