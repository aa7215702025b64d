"""GPU tests of the output writers: files written through the library
(sums on the GPU) equal, byte for byte, the oracle's text of the same
reference routines (src/green_rgf.f90:4541-4896, :2937-2939)."""
import os

import numpy as np
import pytest

from oracle import writers as OW

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rgf():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf as R
    build.build()
    R.load()
    return R


def _read(path):
    with open(path) as f:
        return f.read()


@pytest.mark.parametrize("NB,NS,length,nen,nk", [(3, 2, 4, 5, 2), (5, 3, 7, 9, 3)])
def test_writers_match_oracle_text(rgf, tmp_path, NB, NS, length, nen, nk):
    """Small sizes, and sizes whose ordered sums span several 32-term warp
    chunks with a ragged last one (DOS: 315 terms, current: 75)."""
    from liteqt_b200 import writers as W
    rng = np.random.default_rng(0)
    Lx = 0.5
    nm = NB * NS
    en = np.linspace(-1.0, 1.0, nen)
    G = rng.normal(size=(nk, nen, length, nm, nm)) + 1j * rng.normal(size=(nk, nen, length, nm, nm))
    cur = rng.normal(size=(nk, nen, length, NB, NB))
    cur4 = np.ascontiguousarray(cur[0])
    curk = rng.normal(size=(nk, length, NB, NB))
    tr = rng.normal(size=(nk, nen))
    d = str(tmp_path) + os.sep
    with rgf.Context(rgf.Options()) as ctx:
        W.write_spectrum(ctx, d + "ldos", 3, np.ascontiguousarray(G[:1]), en, length, NB, NS, Lx, (1.0, -2.0))
        W.write_spectrum(ctx, d + "gw_ldos", 3, G, en, length, NB, NS, Lx, (1.0, -2.0), nk=nk, summed_over_k=True)
        W.write_dos_summed_over_k(ctx, d + "dos", 1, G, en, nk, length, NB, NS, Lx)
        W.write_current_spectrum(ctx, d + "Jdens", 2, cur4, en, length, NB, Lx)
        W.write_current_spectrum(ctx, d + "gw_Jdens", 2, cur, en, length, NB, Lx, nk=nk, summed_over_kz=True)
        W.write_current_summed_over_k(ctx, d + "gw_I", 2, curk, length, NB, Lx, nk)
    W.write_transmission_spectrum(d + "tr", 4, tr[0], en)
    W.write_transmission_spectrum(d + "gw_trR", 4, tr, en, nk=nk)
    W.write_id_iteration(d + "gw_Id_iteration.dat", 1, 1.25e-6, -3.5e-7)
    W.write_id_iteration(d + "gw_Id_iteration.dat", 2, 1.5e-6, -2.5e-7)
    assert _read(d + "ldos0003.dat") == OW.spectrum_text(G[:1], en, length, NB, NS, Lx, (1.0, -2.0))
    assert _read(d + "gw_ldos0003.dat") == OW.spectrum_text(G, en, length, NB, NS, Lx, (1.0, -2.0), nk=nk,
                                                            summed_over_k=True)
    assert _read(d + "dos0001.dat") == OW.dos_text(G, en, nk, length, NB, NS, Lx)
    assert _read(d + "Jdens_0002.dat") == OW.current_spectrum_text(cur[:1], en, length, NB, Lx)
    assert _read(d + "gw_Jdens0002.dat") == OW.current_spectrum_text(cur, en, length, NB, Lx, nk=nk,
                                                                     summed_over_kz=True)
    assert _read(d + "gw_I_0002.dat") == OW.current_summed_over_k_text(curk, length, NB, Lx, nk)
    assert _read(d + "tr_0004.dat") == OW.transmission_text(tr[0], en)
    assert _read(d + "gw_trR0004.dat") == OW.transmission_text(tr, en, nk=nk)
    assert _read(d + "gw_Id_iteration.dat") == OW.id_iteration_line(1, 1.25e-6, -3.5e-7) + \
        OW.id_iteration_line(2, 1.5e-6, -2.5e-7)
