import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def random_sigma(nm, nx, nen, seed, scale=0.02):
    """Scattering self-energies for the tests, in the Fortran block layout
    (nen, nx, nm, nm): sigma^R = Hermitian part - i * PSD broadening,
    sigma^< = i * PSD (anti-Hermitian), as a physical Sigma^R / Sigma^< pair."""
    rng = np.random.default_rng(seed)
    sr = np.empty((nen, nx, nm, nm), np.complex128)
    sl = np.empty((nen, nx, nm, nm), np.complex128)
    for e in range(nen):
        for l in range(nx):
            X = rng.normal(size=(nm, nm)) + 1j * rng.normal(size=(nm, nm))
            Y = rng.normal(size=(nm, nm)) + 1j * rng.normal(size=(nm, nm))
            Bm = Y @ Y.conj().T / nm
            A = 0.5 * (X + X.conj().T)
            f = rng.uniform(0.0, 1.0)
            sr[e, l] = (scale * A - 1j * scale * Bm).T
            sl[e, l] = (1j * f * 2 * scale * Bm).T
    return sl, sr


def perturbed_inputs(Hii, H1i, seed, eps=2.0 ** -52):
    """Hii, H1i with every element scaled by (1 + eps*u), u uniform in
    [-1, 1]: one rounding of the input.  Each diagonal block stays Hermitian
    (the perturbed upper triangle is mirrored, the diagonal kept real)."""
    rng = np.random.default_rng(10_000 + seed)
    P = np.array(Hii, np.complex128) * (1 + eps * rng.uniform(-1, 1, np.shape(Hii)))
    up = np.triu(P, 1)
    P = up + np.conj(np.swapaxes(up, -1, -2))
    n = P.shape[-1]
    P[..., range(n), range(n)] = (np.asarray(Hii)[..., range(n), range(n)].real
                                  * (1 + eps * rng.uniform(-1, 1, P.shape[:-2] + (n,))))
    Q = np.array(H1i, np.complex128) * (1 + eps * rng.uniform(-1, 1, np.shape(H1i)))
    return P, Q


def rel_err(a, b, scale=None):
    a = np.asarray(a)
    b = np.asarray(b)
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / s)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
