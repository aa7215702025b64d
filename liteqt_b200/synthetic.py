"""Seeded synthetic tight-binding devices for the RGF benchmarks and tests.

No public dataset is involved: the inputs are random block-tridiagonal
Hamiltonians with the distributions the benchmark configurations state.

* H_ll: Hermitian, diagonal U[-0.5, 0.5] eV, off-diagonal complex N(0, 0.1) eV
  (real and imaginary parts each N(0, 0.1)), Hermitised.
* H_{l,l-1} = -2.7 eV * (I + P_l) with P_l real N(0, 0.05) entries.
* The leads are the semi-infinite continuation of the end blocks, which is
  what the RGF entry point does with Hii(:,:,1), H1i(:,:,1) and Hii(:,:,nx),
  H1i(:,:,nx) (green_rgf.f90:3991-3995, :4032-4035).
* Energies: the liteQT grid en(i) = i/nen*(emax-emin)+emin, i = 1..nen
  (main3d.f90:658).

All arrays are returned in the Fortran layout the C ABI takes: complex128,
column-major (nm, nm, nx), exposed to NumPy as C-contiguous (nx, nm, nm)
arrays whose last two axes are (column, row).  ``H1i[l]`` is the coupling
block H_{l,l-1} (the forward-sweep meaning of H1i(:,:,l)).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Device:
    nm: int
    nx: int
    Hii: np.ndarray   # (nx, nm, nm) complex128, Fortran block layout
    H1i: np.ndarray   # (nx, nm, nm) complex128, Fortran block layout
    seed: int


def _to_fortran_blocks(B: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.swapaxes(B, -1, -2))


def make_device(nm: int, nx: int, seed: int = 1234, onsite=(-0.5, 0.5), offdiag_sigma=0.1,
                hop=-2.7, hop_sigma=0.05, uniform_coupling=False, potential=None) -> Device:
    """Random chain of ``nx`` blocks of ``nm`` orbitals.

    ``potential`` (length nx) is added to the diagonal of each H_ll (the
    per-block on-site potential V_l of the adjoint benchmark).
    ``uniform_coupling`` makes every H1i block the same (the situation every
    reference driver produces, main3d.f90:437-446).
    """
    rng = np.random.default_rng(seed)
    Hb = np.empty((nx, nm, nm), np.complex128)
    for l in range(nx):
        X = rng.normal(0.0, offdiag_sigma, (nm, nm)) + 1j * rng.normal(0.0, offdiag_sigma, (nm, nm))
        U = np.triu(X, 1)
        M = U + U.conj().T
        M[np.diag_indices(nm)] = rng.uniform(onsite[0], onsite[1], nm)
        if potential is not None:
            M[np.diag_indices(nm)] += potential[l]
        Hb[l] = M
    H1b = np.empty((nx, nm, nm), np.complex128)
    P0 = rng.normal(0.0, hop_sigma, (nm, nm))
    for l in range(nx):
        P = P0 if uniform_coupling else rng.normal(0.0, hop_sigma, (nm, nm))
        H1b[l] = hop * (np.eye(nm) + P)
    return Device(nm, nx, _to_fortran_blocks(Hb), _to_fortran_blocks(H1b), seed)


def make_overlap(nm: int, nx: int, seed: int = 4321, sigma: float = 0.05) -> np.ndarray:
    """Overlap blocks S_ll of a non-orthogonal basis (green_RGF_CMS's Sii):
    I + a Hermitian perturbation with complex N(0, sigma/sqrt(nm))
    off-diagonal and real N(0, sigma) diagonal entries.  The 1/sqrt(nm)
    keeps the perturbation's spectral radius near 2*sqrt(2)*sigma whatever
    the block size, so S stays positive definite (a physical overlap).
    Fortran block layout (nx, nm, nm) like Hii."""
    rng = np.random.default_rng(seed)
    Sb = np.empty((nx, nm, nm), np.complex128)
    so = sigma / np.sqrt(nm)
    for l in range(nx):
        X = rng.normal(0.0, so, (nm, nm)) + 1j * rng.normal(0.0, so, (nm, nm))
        U = np.triu(X, 1)
        M = U + U.conj().T
        M[np.diag_indices(nm)] = 1.0 + rng.normal(0.0, sigma, nm)
        Sb[l] = M
    return _to_fortran_blocks(Sb)


def make_coulomb(nm: int, nx: int, seed: int = 99, a: float = 0.3, cell: float = 0.5,
                 width: float = 2.0, e2: float = 1.44) -> tuple[np.ndarray, np.ndarray]:
    """Bare Coulomb interaction of the GW workloads as block-tridiagonal
    blocks: orbital positions seeded uniformly in cells of `cell` nm along the
    chain (block l at x in [l*cell, (l+1)*cell)) and `width` nm across,
    V_ij = e2 / (|r_i - r_j| + a) eV (e2 = e^2/(4 pi eps0) = 1.44 eV nm,
    a = 0.3 nm), truncated to the diagonal blocks and the first
    off-diagonal blocks.  Returns (Vii, V1i) in the Fortran block layout;
    V1i[l] is V_{l+1,l} (zero for l = nx-1), real, so V is real symmetric."""
    rng = np.random.default_rng(seed)
    pos = np.empty((nx, nm, 3))
    for l in range(nx):
        pos[l, :, 0] = rng.uniform(l * cell, (l + 1) * cell, nm)
        pos[l, :, 1:] = rng.uniform(0.0, width, (nm, 2))

    def block(p, q):
        r = np.linalg.norm(p[:, None, :] - q[None, :, :], axis=-1)
        return e2 / (r + a)
    Vb = np.array([block(pos[l], pos[l]) for l in range(nx)], dtype=np.complex128)
    V1b = np.zeros((nx, nm, nm), np.complex128)
    for l in range(nx - 1):
        V1b[l] = block(pos[l + 1], pos[l])
    return _to_fortran_blocks(Vb), _to_fortran_blocks(V1b)


def make_polarization(nm: int, nx: int, nen: int, seed: int = 7, scale: float = 0.05):
    """Seeded polarization blocks (PL, PG, PR), each (nen, nx, nm, nm) in the
    Fortran block layout, with the symmetries of the physical P: P^R complex
    symmetric with a negative-semidefinite imaginary part, P^< and P^>
    anti-Hermitian and complex symmetric (i times a real symmetric matrix,
    P^< with a non-negative, P^> with a non-positive spectrum)."""
    rng = np.random.default_rng(seed)
    out = [np.empty((nen, nx, nm, nm), np.complex128) for _ in range(3)]
    for e in range(nen):
        for l in range(nx):
            X = rng.normal(0.0, 1.0, (nm, nm))
            Y = rng.normal(0.0, 1.0, (nm, nm))
            A = (X + X.T) / np.sqrt(2 * nm)
            B = Y @ Y.T / nm                       # real symmetric PSD
            f = rng.uniform(0.0, 1.0)
            out[2][e, l] = scale * (A - 1j * B)    # P^R
            out[0][e, l] = 1j * scale * 2 * f * B   # P^<
            out[1][e, l] = -1j * scale * 2 * (1 - f) * B  # P^>
    return tuple(out)


def uniform_chain(nm: int, nx: int, t: float = -1.0, eps: float = 0.0) -> Device:
    """nm decoupled identical 1D chains: H_ll = eps*I, H_{l,l-1} = t*I.
    Its exact transmission is nm inside the band |E - eps| < 2|t|."""
    Hb = np.broadcast_to(eps * np.eye(nm, dtype=np.complex128), (nx, nm, nm)).copy()
    H1b = np.broadcast_to(t * np.eye(nm, dtype=np.complex128), (nx, nm, nm)).copy()
    return Device(nm, nx, _to_fortran_blocks(Hb), _to_fortran_blocks(H1b), 0)


def energy_grid(nen: int, emin: float = -3.0, emax: float = 3.0) -> np.ndarray:
    """en(i) = i/nen*(emax-emin)+emin, i = 1..nen (main3d.f90:658)."""
    return np.arange(1, nen + 1, dtype=np.float64) / float(nen) * (emax - emin) + emin


def temperature_for_kT(kT: float, boltz: float = 8.61734e-05) -> float:
    return kT / boltz


def lead_band_edges(Hii: np.ndarray, H1i: np.ndarray, block: int = 0, nk: int = 512) -> np.ndarray:
    """Subband edges (eV) of the semi-infinite lead that continues block
    ``block`` of a device (Hii, H1i in the Fortran block layout): the extrema
    over k of every eigenvalue band of the Bloch Hamiltonian
    H(k) = H00 + T e^{ik} + T^H e^{-ik}, with H00 the block and T its coupling
    H1i(:,:,block+1).  Bands are sampled on nk points of [-pi, pi) and each
    extremum is refined by the parabola through its sample and the two
    neighbours.  Returns the sorted band minima and maxima."""
    H00 = np.asarray(Hii[block]).T
    T = np.asarray(H1i[block]).T
    k = -np.pi + 2.0 * np.pi * np.arange(nk) / nk
    ev = np.empty((nk, H00.shape[0]))
    for i, kk in enumerate(k):
        Hk = H00 + T * np.exp(1j * kk) + T.conj().T * np.exp(-1j * kk)
        ev[i] = np.linalg.eigvalsh(0.5 * (Hk + Hk.conj().T))
    edges = []
    for n in range(ev.shape[1]):
        band = ev[:, n]
        for i0 in (int(np.argmin(band)), int(np.argmax(band))):
            y0, y1, y2 = band[(i0 - 1) % nk], band[i0], band[(i0 + 1) % nk]
            den = y0 - 2.0 * y1 + y2
            edges.append(y1 - 0.125 * (y2 - y0) ** 2 / den if den != 0.0 else y1)
    return np.sort(np.array(edges))


def band_edge_energy_grid(nen: int, edges: np.ndarray, emin: float = -3.0, emax: float = 3.0,
                          frac: float = 0.1, width: float = 1e-3, seed: int = 5) -> np.ndarray:
    """Energies for the band-edge workload: round(frac*nen) points placed
    within `width` eV of band edges in [emin, emax] (edges drawn uniformly
    with replacement, offsets uniform in [-width, width]), the rest on the
    uniform liteQT grid of [emin, emax]; sorted."""
    rng = np.random.default_rng(seed)
    n_edge = int(round(frac * nen))
    inside = edges[(edges > emin + width) & (edges < emax - width)]
    grid = energy_grid(nen - n_edge, emin, emax)
    if n_edge == 0 or inside.size == 0:
        return energy_grid(nen, emin, emax)
    near = rng.choice(inside, n_edge) + rng.uniform(-width, width, n_edge)
    return np.sort(np.concatenate([grid, near]))
