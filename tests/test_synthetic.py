"""CPU tests of the seeded workload generators: the liteQT energy grid
(main3d.f90:658, i = 1..nen), the lead subband edges of the band-edge
workload and its energy grid with a fraction of points near the edges."""
import numpy as np
import pytest

from liteqt_b200 import synthetic as S


def test_energy_grid_is_the_reference_grid():
    E = S.energy_grid(8, -3.0, 3.0)
    assert E.shape == (8,)
    assert E[0] == pytest.approx(-3.0 + 6.0 / 8) and E[-1] == 3.0   # i = 1 .. nen, not 0 .. nen-1
    assert np.allclose(np.diff(E), 6.0 / 8)


@pytest.mark.parametrize("nm,eps,t", [(4, 0.0, -1.0), (3, 0.25, 0.7)])
def test_band_edges_of_a_uniform_chain(nm, eps, t):
    """H00 = eps I, T = t I: every band is eps + 2 t cos k, edges eps -+ 2|t|."""
    d = S.uniform_chain(nm, 3, t=t, eps=eps)
    edges = S.lead_band_edges(d.Hii, d.H1i, 0, nk=64)
    want = np.sort(np.r_[np.full(nm, eps - 2 * abs(t)), np.full(nm, eps + 2 * abs(t))])
    assert np.allclose(edges, want, atol=1e-12)


def test_band_edges_of_a_random_lead_bound_the_spectrum():
    d = S.make_device(16, 3, seed=2)
    edges = S.lead_band_edges(d.Hii, d.H1i, 0, nk=128)
    assert edges.shape == (32,) and np.all(np.diff(edges) >= 0)
    H00, T = d.Hii[0].T, d.H1i[0].T
    for k in np.linspace(-np.pi, np.pi, 7):
        ev = np.linalg.eigvalsh(H00 + T * np.exp(1j * k) + T.conj().T * np.exp(-1j * k))
        assert ev.min() >= edges[0] - 1e-9 and ev.max() <= edges[-1] + 1e-9


def test_band_edge_grid_places_the_fraction_near_edges():
    edges = np.array([-2.5, -1.0, 0.4, 2.9])
    nen, frac, width = 400, 0.1, 1e-3
    E = S.band_edge_energy_grid(nen, edges, -3.0, 3.0, frac=frac, width=width, seed=3)
    assert E.shape == (nen,) and np.all(np.diff(E) >= 0)
    near = np.min(np.abs(E[:, None] - edges[None, :]), axis=1) <= width
    uniform = S.energy_grid(nen - round(frac * nen), -3.0, 3.0)
    assert near.sum() >= round(frac * nen)
    assert np.all(np.isin(uniform, E))
