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
