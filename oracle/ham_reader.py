"""Oracle of w90_load_from_file (src/wannierHam.f90:68-130), test
infrastructure only: Fortran list-directed reads of the Wannier Hamiltonian
file restated in Python, and the derived cell quantities."""
import math

import numpy as np


def _values(path):
    recs = []
    with open(path) as f:
        for line in f:
            recs.append(line.replace(",", " ").split())
    return recs


def read(path, axis=None):
    recs = _values(path)
    pos = [0]

    def read_n(n):           # one READ statement: starts at a new record
        out = []
        while len(out) < n:
            out.extend(recs[pos[0]])
            pos[0] += 1
        return out[:n]

    num = lambda s: float(s.replace("d", "e").replace("D", "e"))
    nvb, spin = (int(x) for x in read_n(2))
    read_n(1)
    cell = np.array([[num(x) for x in read_n(3)] for _ in range(3)])   # rows alpha, beta, gamm
    read_n(1)
    if axis is not None:
        cell = cell[[a - 1 for a in axis]]
    n = int(read_n(1)[0])
    ham = np.array([[num(x) for x in read_n(7)] for _ in range(n)])
    if axis is not None:
        ham[:, 0:3] = ham[:, [a - 1 for a in axis]]
    xmin, xmax = int(ham[:, 0].min()), int(ham[:, 0].max())
    ymin, ymax = int(ham[:, 1].min()), int(ham[:, 1].max())
    nb = int(ham[:, 3].max())
    nx, ny = xmax - xmin + 1, ymax - ymin + 1
    alpha, beta, gamm = cell
    xhat = alpha / np.linalg.norm(alpha)
    yhat = -np.cross(xhat, gamm)
    yhat = yhat / np.linalg.norm(yhat)
    info = dict(nvb=nvb, spin_deg=spin, nb=nb, nx=nx, ny=ny, xmin=xmin, xmax=xmax, ymin=ymin, ymax=ymax,
                n_entries=n, Lx=abs(alpha @ xhat), Ly=abs(beta @ yhat), Lz=np.linalg.norm(gamm),
                b1=np.cross(beta, gamm) / (alpha @ np.cross(beta, gamm)),
                b2=np.cross(gamm, alpha) / (beta @ np.cross(gamm, alpha)), cell=cell)
    Hr = np.zeros((ny, nx, nb, nb), complex)          # view of Hr(nb,nb,nx,ny): [y, x, n, m]
    for r in ham:
        Hr[math.floor(r[1]) - ymin, math.floor(r[0]) - xmin, math.floor(r[4]) - 1, math.floor(r[3]) - 1] = \
            complex(r[5], r[6])
    return info, Hr
