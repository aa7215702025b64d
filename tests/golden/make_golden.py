"""Generate the golden fixtures in this directory with the CPU oracle.

    python tests/golden/make_golden.py

Each fixture holds seeded inputs (Fortran block layout, see oracle/oracle.py),
the FP64 oracle's outputs and, as exact_*, the same algorithm evaluated in
x87 80-bit precision.  They pin the oracle against regressions and give
the GPU parity tests a reference that needs no oracle at run time.  The
reference (Fortran + MKL) cannot be run in this environment, so these are
outputs of the restatement, not of the reference itself.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import random_sigma  # noqa: E402
from liteqt_b200 import synthetic as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = [
    # name, nm, nx, nen, consistent, sigma, eta_dev, eta_lead, boltz, overlap (green_RGF_CMS)
    ("compat_nm8_nx4", 8, 4, 5, False, False, 0.0, 1e-3, O.BOLTZ_RGF_RS, False),
    ("compat_sigma_nm8_nx5", 8, 5, 4, False, True, 0.0, 1e-3, O.BOLTZ_RGF_RS, False),
    ("consistent_nm16_nx3", 16, 3, 3, True, True, 1e-5, 1e-5, O.BOLTZ_RGF_RS, False),
    ("rgfg_nm8_nx2", 8, 2, 3, False, False, 0.0, 1e-3, O.BOLTZ_RGF_G, False),
    ("cms_sigma_nm8_nx4", 8, 4, 4, False, True, 0.0, 1e-3, O.BOLTZ_RGF_RS, True),
]


def main(names=None):
    """Writes every fixture, or only those named on the command line."""
    mu = np.array([0.1, -0.1])
    temp = np.array([S.temperature_for_kT(0.025)] * 2)
    for name, nm, nx, nen, cons, sig, eta_dev, eta_lead, boltz, ovl in CASES:
        if names and name not in names:
            continue
        d = S.make_device(nm, nx, seed=1000 + nm * 10 + nx)
        E = S.energy_grid(nen, -3.0, 3.0)
        sl, sr = random_sigma(nm, nx, nen, seed=99) if sig else (None, None)
        Sii = S.make_overlap(nm, nx, seed=77) if ovl else None
        opts = O.Opts(eta_dev=eta_dev, eta_lead=eta_lead, consistent=cons, boltz=boltz)
        r = O.rgf_batch(d.Hii, d.H1i, E, mu, temp, opts, sig_lesser=sl, sig_r=sr, threads=1, Sii=Sii)
        x = O.rgf_batch(d.Hii, d.H1i, E, mu, temp, opts, sig_lesser=sl, sig_r=sr, threads=1,
                        extended=True, Sii=Sii)
        extra = {"has_overlap": True, "Sii": Sii} if ovl else {}
        exact = {"exact_" + k: x[k] for k in ("ldos", "ndens", "pdens", "GRi1", "cur", "tr", "tre", "T")}
        empty = np.zeros((0,), np.complex128)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), Hii=d.Hii, H1i=d.H1i, E=E, mu=mu, temp=temp,
            has_sigma=sig, sig_lesser=sl if sig else empty, sig_r=sr if sig else empty,
            consistent=cons, eta_dev=eta_dev, eta_lead=eta_lead, boltz=boltz,
            ldos=r["ldos"], ndens=r["ndens"], pdens=r["pdens"], GRi1=r["GRi1"], cur=r["cur"],
            tr=r["tr"], tre=r["tre"], T=r["T"],
            sancho_iters=np.stack([r["stats"]["sancho_iters_left"], r["stats"]["sancho_iters_right"]]),
            **exact, **extra)
        print(name, os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")


if __name__ == "__main__":
    main(sys.argv[1:])
