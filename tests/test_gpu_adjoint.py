"""GPU tests of the adjoint RGF (rgf_adjoint_energies): T(E), dT/dV_l, dT/ds
and the Landauer current's derivatives, against the analytic adjoint of the
oracle (oracle.adjoint_numpy) and central finite differences of the FP64
oracle (the reference algorithm) at dV = 1e-6 eV."""
import numpy as np
import pytest

from liteqt_b200 import synthetic as S

pytestmark = pytest.mark.gpu

MU = (0.1, -0.1)


def _temp():
    return (S.temperature_for_kT(0.025),) * 2


@pytest.fixture(scope="module")
def rgf():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf as R
    build.build()
    R.load()
    return R


def gpu_adjoint(R, d, E, opts, spindeg=2.0):
    nen = len(E)
    T = np.zeros(nen)
    dTdV = np.zeros((nen, d.nx))
    dTds = np.zeros(nen)
    info = np.zeros(nen, R.INFO_DTYPE)
    with R.Context(opts) as ctx:
        dIdV, dIds = ctx.adjoint_energies(d.Hii, d.H1i, np.asarray(E, float), MU, _temp(), T=T,
                                          dTdV=dTdV, dTds=dTds, spindeg=spindeg, info=info)
    return T, dTdV, dTds, dIdV, dIds, info


@pytest.mark.parametrize("nm,nx", [(8, 2), (8, 5), (16, 20), (32, 40)])
def test_adjoint_matches_analytic_adjoint(rgf, nm, nx):
    """nx >= 18 runs the sqrt(nx)-checkpointed reverse sweep (segments)."""
    from oracle import oracle as O
    d = S.make_device(nm, nx, seed=500 + nm + nx)
    E = np.array([-1.7, -0.2, 0.9])
    opts = rgf.Options()
    T, dTdV, dTds, _, _, info = gpu_adjoint(rgf, d, E, opts)
    assert np.all(info["status"] == 0)
    Hb, H1b = O.to_blocks(d.Hii), O.to_blocks(d.H1i)
    for ie, e in enumerate(E):
        Tr, dVr, dsr = O.adjoint_numpy(Hb, H1b, e, O.Opts())
        assert abs(T[ie] - Tr) < 1e-10 * max(1.0, abs(Tr))
        scale = np.max(np.abs(dVr))
        assert np.max(np.abs(dTdV[ie] - dVr)) < 1e-9 * scale, (ie, np.max(np.abs(dTdV[ie] - dVr)) / scale)
        assert abs(dTds[ie] - dsr) < 1e-9 * max(abs(dsr), 1.0)


def test_adjoint_matches_finite_differences_of_reference_rgf(rgf):
    """Central differences of the FP64 CPU restatement of green_RGF_RS's T(E).
    Interior blocks and the coupling scale at dV = 1e-6 eV.  The two end
    blocks also move the Sancho-Rubio leads, whose decimation amplifies
    rounding (T carries ~1e-11 of noise), so central differences at 1e-6 eV
    there are noise-limited to ~1e-5; they are checked at dV = 1e-4 eV, where
    the O(dV^2) truncation is ~1e-7."""
    from oracle import oracle as O
    nm, nx = 16, 12
    d = S.make_device(nm, nx, seed=44, potential=np.random.default_rng(1).uniform(-0.2, 0.2, 12))
    E = np.array([-0.8, 0.3])
    opts = rgf.Options()
    T, dTdV, dTds, _, _, _ = gpu_adjoint(rgf, d, E, opts)
    fdV, fds = O.fd_gradient(d.Hii, d.H1i, E, MU, _temp(), O.Opts(), h=1e-6)
    scale = np.max(np.abs(fdV))
    assert np.max(np.abs(dTdV[:, 1:-1] - fdV[:, 1:-1])) < 1e-6 * scale
    assert np.max(np.abs(dTds - fds)) < 1e-6 * max(np.max(np.abs(fds)), 1.0)
    fdV4, _ = O.fd_gradient(d.Hii, d.H1i, E, MU, _temp(), O.Opts(), h=1e-4)
    ends = [0, nx - 1]
    assert np.max(np.abs(dTdV[:, ends] - fdV4[:, ends])) < 1e-5 * scale


def test_adjoint_current_derivatives(rgf):
    from oracle import oracle as O
    nm, nx = 8, 6
    d = S.make_device(nm, nx, seed=3)
    E = S.energy_grid(64, -0.5, 0.5)
    opts = rgf.Options()
    T, dTdV, dTds, dIdV, dIds, _ = gpu_adjoint(rgf, d, E, opts, spindeg=2.0)
    fl = O.ferm((E - MU[0]) / (O.BOLTZ_RGF_RS * _temp()[0]))
    fr = O.ferm((E - MU[1]) / (O.BOLTZ_RGF_RS * _temp()[1]))
    w = (fl - fr) * (E[1] - E[0]) * O.E0 / O.TPI / O.HBAR * O.E0 * 2.0
    ref = w @ dTdV
    assert np.allclose(dIdV, ref, rtol=1e-12, atol=1e-30)
    assert abs(dIds - w @ dTds) <= 1e-12 * abs(w @ dTds)
    # the current itself, from the same T: I = sum_e w_e T(E_e)
    assert np.all(T > 0)
