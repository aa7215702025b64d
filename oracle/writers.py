"""Oracle of the reference's output writers (test infrastructure only):
src/green_rgf.f90:4541-4896 and :2937-2939 restated with NumPy sums in each
routine's loop order and Python formatting of Fortran's Ew.d / Iw."""
import math

import numpy as np


def fE(v, w, d):
    """Fortran Ew.d: 0.d..dE+ee (E dropped for 3-digit exponents), right-justified."""
    v = float(v)
    if math.isnan(v) or math.isinf(v):
        body = "NaN" if math.isnan(v) else ("-Infinity" if v < 0 else "Infinity")
    else:
        mant, ex = f"{abs(v):.{d - 1}e}".split("e")
        digits = mant.replace(".", "")
        ex = 0 if v == 0 else int(ex) + 1
        exp = f"E{'-' if ex < 0 else '+'}{abs(ex):02d}" if abs(ex) <= 99 else f"{'-' if ex < 0 else '+'}{abs(ex):03d}"
        body = ("-" if math.copysign(1.0, v) < 0 else "") + "0." + digits + exp
    return "*" * w if len(body) > w else body.rjust(w)


def fI(v, w):
    s = str(int(v))
    return "*" * w if len(s) > w else s.rjust(w)


def STRING(i):
    return f"{i:04d}"


def spectrum_text(G, en, length, NB, NS, Lx, coeff, nk=1, summed_over_k=False):
    """G: (nk, nen, length, nm, nm) NumPy view of G(nm,nm,length,nen,nk)."""
    lines = []
    for ie in range(len(en)):
        for j in range(length):
            for k in range(NS):
                tr = 0j
                for ik in range(nk):
                    for ib in range(NB):
                        d = ib + k * NB
                        tr = tr + G[ik, ie, j, d, d]
                if summed_over_k:
                    tr = tr / nk
                x = j * Lx * NS + k * Lx
                lines.append(fE(x, 18, 4) + fE(en[ie], 18, 4) + fE(tr.real * coeff[0], 18, 4) +
                             fE(tr.imag * coeff[1], 18, 4))
        lines.append("")
    return "\n".join(lines) + "\n"


def dos_text(G, en, nk, length, NB, NS, Lx):
    lines = []
    for ie in range(len(en)):
        tr = 0j
        for j in range(length):
            for k in range(NS):
                for ik in range(nk):
                    for ib in range(NB):
                        d = ib + k * NB
                        tr = tr + G[ik, ie, j, d, d]
        im = tr.imag / nk / length / NS / Lx
        lines.append(fE(en[ie], 18, 4) + fE(im * (-2.0), 18, 4))
    return "\n".join(lines) + "\n"


def current_spectrum_text(cur, en, length, NB, Lx, nk=1, summed_over_kz=False):
    """cur: (nk, nen, length, NB, NB) view of cur(NB,NB,length,nen,nk)."""
    lines = []
    for ie in range(len(en)):
        for j in range(length - 1 if summed_over_kz else length):
            tr = 0.0
            for ik in range(nk if summed_over_kz else 1):
                for ib in range(NB):
                    for jb in range(NB):
                        tr = tr + cur[ik, ie, j, jb, ib]
            if summed_over_kz:
                tr = tr / nk
            lines.append(fE(j * Lx, 18, 4) + fE(en[ie], 18, 4) + fE(tr, 18, 4))
        lines.append("")
    return "\n".join(lines) + "\n"


def current_summed_over_k_text(cur, nx, NB, Lx, nk):
    """cur: (nk, nx, NB, NB) view of cur(NB,NB,nx,nk)."""
    lines = []
    for ii in range(nx - 1):
        tr = 0.0
        for ib in range(NB):
            for jb in range(NB):
                for ik in range(nk):
                    tr = tr + cur[ik, ii, jb, ib]
        lines.append(fE(ii * Lx, 18, 4) + fE(tr / nk, 18, 4))
    return "\n".join(lines) + "\n"


def transmission_text(tr, en, nk=0):
    """tr: (nen,) or (nk, nen) view of tr(nen,nk)."""
    lines = []
    for ie in range(len(en)):
        if nk:
            s = 0.0
            for ik in range(nk):
                s = s + tr[ik, ie]
            v = s / nk
        else:
            v = tr[ie]
        lines.append(fE(en[ie], 18, 4) + fE(v, 18, 4))
    return "\n".join(lines) + "\n"


def id_iteration_line(it, a, b):
    return fI(it, 4) + fE(a, 16, 6) + fE(b, 16, 6) + "\n"
