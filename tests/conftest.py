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


# GPU-vs-oracle parity rule (the FP64 tolerance and the noise-floor fallback
# are explained in test_gpu_parity.py's module docstring).
def errors(g, r, nm, H1i, skip_last_gri1=True):
    """Per-output relative errors of g against r; outputs absent from g
    (not requested from the GPU) are skipped."""
    errs = {}
    errs["ldos"] = rel_err(g["ldos"], r["ldos"])
    errs["ndens"] = rel_err(g["ndens"], r["ndens"])
    if g.get("pdens") is not None:
        errs["pdens"] = rel_err(g["pdens"], r["pdens"], scale=max(np.max(np.abs(r["ldos"])),
                                                                    np.max(np.abs(r["ndens"]))))
    sl = slice(0, -1) if skip_last_gri1 else slice(None)
    for k in ("GRi1", "GLi1", "GGi1"):
        if g.get(k) is not None:
            errs[k] = rel_err(g[k][:, sl], r[k][:, sl])
    if g.get("cur") is not None:
        cur_scale = nm * np.max(np.abs(H1i)) * np.max(np.abs(r["ndens"]))
        errs["cur"] = rel_err(g["cur"], r["cur"], scale=cur_scale)
    trs = max(np.max(np.abs(r["tr"])), np.max(np.abs(r["tre"])), np.max(np.abs(r["T"])), 1e-300)
    errs["tr"] = float(np.max(np.abs(g["tr"] - r["tr"])) / trs)
    errs["tre"] = float(np.max(np.abs(g["tre"] - r["tre"])) / trs)
    errs["T"] = float(np.max(np.abs(g["T"] - r["T"]) / np.maximum(1.0, np.abs(r["T"]))))
    return errs


def compare(g, r, nm, H1i, tol=1e-10, truth=None, skip_last_gri1=True, floor=()):
    """g: GPU outputs, r: FP64 oracle outputs, truth: 80-bit oracle outputs,
    floor: FP64 oracle outputs on perturbed inputs (noise floor)."""
    e_go = errors(g, r, nm, H1i, skip_last_gri1)
    if truth is None:
        bad = {k: v for k, v in e_go.items() if not v <= tol}
        assert not bad, f"errors above {tol}: {bad} (all: {e_go})"
        return e_go
    e_gt = errors(g, truth, nm, H1i, skip_last_gri1)
    e_rt = errors(r, truth, nm, H1i, skip_last_gri1)
    for f in floor:
        e_ft = errors(f, truth, nm, H1i, skip_last_gri1)
        e_rt = {k: max(e_rt[k], e_ft[k]) for k in e_rt}
    bad = {k: (e_go[k], e_gt[k], e_rt[k]) for k in e_go
           if not (e_go[k] <= tol or e_gt[k] <= 8.0 * e_rt[k] + 1e-12) or not e_gt[k] < 1e-6}
    assert not bad, f"(gpu-oracle, gpu-exact, oracle-exact) failing: {bad}"
    return e_go


def compare_spread(g, r, floors, nm, H1i, tol=1e-10, factor=8.0, skip_last_gri1=True):
    """Parity rule for the full-size configurations, where the 80-bit
    evaluation takes minutes: every output within `tol` of the FP64 oracle r,
    or within `factor` times the FP64 spread of the problem -- the largest
    distance between r and the FP64 oracle run on inputs perturbed by one
    rounding (floors).  The spread is the problem's own conditioning: a
    200-block disordered chain near a resonance moves its G^R by 1e-4
    (relative) under one rounding of the input, so no absolute cap applies.
    Returns the errors and the spread."""
    e_go = errors(g, r, nm, H1i, skip_last_gri1)
    spread = {k: 0.0 for k in e_go}
    for f in floors:
        e_f = errors({k: f[k] for k in f if k in g or k in ("tr", "tre", "T")}, r, nm, H1i,
                     skip_last_gri1)
        spread = {k: max(spread[k], e_f.get(k, 0.0)) for k in spread}
    bad = {k: (e_go[k], spread[k]) for k in e_go
           if not (e_go[k] <= tol or e_go[k] <= factor * spread[k] + 1e-12)}
    assert not bad, f"(gpu-oracle, fp64 spread) failing: {bad}"
    return e_go, spread



@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
