"""CPU tests of the oracle (test infrastructure): the C++ restatement of
green_RGF_RS against the independent NumPy restatement, and both against
known answers (dense inverse, Sancho fixed point, uniform chain, current
conservation, Hermiticity) and the committed golden fixtures."""
import glob
import os

import numpy as np
import pytest

from conftest import random_sigma, rel_err
from liteqt_b200 import synthetic as S

MU = (0.1, -0.1)


def _temp():
    return (S.temperature_for_kT(0.025),) * 2


@pytest.mark.parametrize("consistent", [False, True])
@pytest.mark.parametrize("nm,nx,scatter", [(8, 5, False), (8, 2, True), (12, 4, True), (16, 3, False)])
def test_cpp_matches_numpy_restatement(oracle_mod, consistent, nm, nx, scatter):
    O = oracle_mod
    d = S.make_device(nm, nx, seed=nm * 100 + nx)
    E = np.array([-2.2, -0.45, 0.02, 0.9, 2.7])
    sl = sr = None
    if scatter:
        sl, sr = random_sigma(nm, nx, len(E), seed=7)
    opts = O.Opts(consistent=consistent)
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), opts, sig_lesser=sl, sig_r=sr, threads=2)
    Hb, H1b = O.to_blocks(d.Hii), O.to_blocks(d.H1i)
    for ie, e in enumerate(E):
        t = O.rgf_numpy(Hb, H1b, e, MU, _temp(), opts,
                        sigl=None if sl is None else O.to_blocks(sl[ie]),
                        sigr=None if sr is None else O.to_blocks(sr[ie]))
        g_scale = np.max(np.abs(t["ldos"]))
        for k in ("ldos", "ndens", "GRi1"):
            assert rel_err(O.to_blocks(r[k][ie]), t[k]) < 1e-9, k
        assert rel_err(O.to_blocks(r["pdens"][ie]), t["pdens"], scale=g_scale) < 1e-9
        cur_scale = nm * np.max(np.abs(H1b)) * np.max(np.abs(t["ndens"]))
        assert rel_err(O.to_blocks(r["cur"][ie]), t["cur"], scale=cur_scale) < 1e-9
        assert abs(r["T"][ie] - t["T"]) < 1e-9 * max(1.0, abs(t["T"]))
        tr_scale = max(np.max(np.abs(r["tr"])), 1e-300)
        assert abs(r["tr"][ie] - t["tr"]) < 1e-8 * tr_scale + 1e-14 * nm
        assert abs(r["tre"][ie] - t["tre"]) < 1e-8 * tr_scale + 1e-14 * nm
        assert tuple(r["stats"][ie][["sancho_iters_left", "sancho_iters_right"]]) == t["iters"]


def test_gemm_inverse_counts_follow_reference_formula(oracle_mod):
    """N_gemm = 28 Nx - 18 + 6 (nL + nR) and N_inv = Nx + 4 + nL + nR for a
    call with GRi1 only (green_rgf.f90:2920), plus 2 (Nx-2) + 4 T(E) products."""
    O = oracle_mod
    nm, nx = 8, 7
    d = S.make_device(nm, nx, seed=5)
    r = O.rgf_batch(d.Hii, d.H1i, np.array([0.3]), MU, _temp(), O.Opts(), threads=1)
    st = r["stats"][0]
    nl, nr = st["sancho_iters_left"], st["sancho_iters_right"]
    assert st["n_gemm"] == 28 * nx - 18 + 6 * (nl + nr) + 2 * (nx - 2) + 4
    assert st["n_inv"] == nx + 4 + nl + nr


@pytest.mark.parametrize("nm,nx", [(4, 2), (6, 5), (8, 7)])
def test_dense_inverse_known_answer(oracle_mod, nm, nx):
    """Consistent mode equals the inverse of the whole device matrix."""
    O = oracle_mod
    d = S.make_device(nm, nx, seed=11 + nm)
    Hb, H1b = O.to_blocks(d.Hii), O.to_blocks(d.H1i)
    E = np.array([-1.3, 0.4, 2.1])
    sl, sr = random_sigma(nm, nx, len(E), seed=3)
    opts = O.Opts(consistent=True, eta_dev=1e-4)
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), opts, sig_lesser=sl, sig_r=sr, threads=1)
    for ie, e in enumerate(E):
        t = O.rgf_numpy(Hb, H1b, e, MU, _temp(), opts, sigl=O.to_blocks(sl[ie]), sigr=O.to_blocks(sr[ie]))
        srb = O.to_blocks(sr[ie])
        G = O.dense_green(Hb, H1b, e, t["sigmal"], t["sigmar"], eta_dev=opts.eta_dev, sigr=srb)
        ldos = O.to_blocks(r["ldos"][ie])
        gri1 = O.to_blocks(r["GRi1"][ie])
        for l in range(nx):
            s = slice(l * nm, (l + 1) * nm)
            assert rel_err(ldos[l], G[s, s], scale=np.max(np.abs(G))) < 1e-10
            if l < nx - 1:
                s1 = slice((l + 1) * nm, (l + 2) * nm)
                assert rel_err(gri1[l], G[s, s1], scale=np.max(np.abs(G))) < 1e-10
        # G^< = G Sigma^< G^H with the lead and scattering Sigma^<
        N = nm * nx
        Sl = np.zeros((N, N), complex)
        fl = O.ferm((e - MU[0]) / (opts.boltz * _temp()[0]))
        fr = O.ferm((e - MU[1]) / (opts.boltz * _temp()[0]))
        Sl[:nm, :nm] = -(t["sigmal"] - t["sigmal"].conj().T) * fl
        Sl[-nm:, -nm:] = -(t["sigmar"] - t["sigmar"].conj().T) * fr
        slb = O.to_blocks(sl[ie])
        for l in range(nx):
            Sl[l * nm:(l + 1) * nm, l * nm:(l + 1) * nm] += slb[l]
        Gless = G @ Sl @ G.conj().T
        nd = O.to_blocks(r["ndens"][ie])
        for l in range(nx):
            s = slice(l * nm, (l + 1) * nm)
            assert rel_err(nd[l], Gless[s, s], scale=np.max(np.abs(Gless))) < 1e-10
        # Caroli te(L,R) = Re Tr[Gamma_L G^A Gamma_R G^R] (green.f90:2571-2580)
        gL = 1j * (t["sigmal"] - t["sigmal"].conj().T)
        gR = 1j * (t["sigmar"] - t["sigmar"].conj().T)
        GN1 = G[-nm:, :nm]
        T = np.real(np.trace(gL @ GN1.conj().T @ gR @ GN1))
        assert abs(r["T"][ie] - T) < 1e-10 * max(1.0, abs(T))


def test_sancho_fixed_point(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(3)
    nm = 6
    X = rng.normal(size=(nm, nm)) + 1j * rng.normal(size=(nm, nm))
    H00 = 0.1 * (X + X.conj().T)
    H10 = -1.0 * (np.eye(nm) + 0.1 * rng.normal(size=(nm, nm)))
    opts = O.Opts()
    for E in (-0.7, 0.3, 1.1):
        G, _, it, st = O.sancho_numpy(E, H00, H10, opts)
        assert st == 0 and it < opts.sancho_nmax
        z = complex(E, opts.eta_lead)
        R = G - np.linalg.inv(z * np.eye(nm) - H00 - H10.conj().T @ G @ H10)
        assert np.linalg.norm(R) < 1e-8 * np.linalg.norm(G)


def test_uniform_chain_integer_transmission(oracle_mod):
    O = oracle_mod
    nm = 4
    d = S.uniform_chain(nm, 6, t=-1.0)
    E = np.array([-1.5, -0.5, 0.05, 0.5, 1.9, 2.5])
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(eta_lead=1e-6, consistent=True), threads=2)
    inside = np.abs(E) < 2.0
    assert np.allclose(r["T"][inside], nm, atol=1e-8)
    assert np.all(np.abs(r["T"][~inside]) < 1e-8)
    fl = O.ferm((E - MU[0]) / (O.BOLTZ_RGF_RS * _temp()[0]))
    fr = O.ferm((E - MU[1]) / (O.BOLTZ_RGF_RS * _temp()[0]))
    expect = r["T"] * (fl - fr)
    scale = np.max(np.abs(expect))
    assert np.max(np.abs(r["tr"] - expect)) < 1e-9 * scale
    assert np.max(np.abs(r["tre"] - expect)) < 1e-9 * scale


def test_invariants_and_current_conservation(oracle_mod):
    O = oracle_mod
    nm, nx = 8, 6
    d = S.make_device(nm, nx, seed=21)
    E = S.energy_grid(9, -1.0, 1.0)
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(consistent=True), threads=2)
    g = O.to_blocks(r["ndens"])
    assert np.max(np.abs(g + np.swapaxes(g.conj(), -1, -2))) < 1e-10 * np.max(np.abs(g))
    ldos = O.to_blocks(r["ldos"])
    diag = np.diagonal(ldos, axis1=-2, axis2=-1)
    assert np.all(diag.imag <= 1e-12)
    scale = np.max(np.abs(r["tr"]))
    assert np.max(np.abs(r["tr"] - r["tre"])) < 1e-8 * scale


def test_singular_block_gives_zero_and_status(oracle_mod):
    """invert's zero-matrix fallback (green_rgf.f90:4429-4437): H = E*I, no coupling."""
    O = oracle_mod
    nm, nx, E = 8, 3, 0.25
    Hii = O.from_blocks(np.broadcast_to(E * np.eye(nm), (nx, nm, nm)).astype(complex))
    H1i = np.zeros_like(Hii)
    r = O.rgf_batch(Hii, H1i, np.array([E]), MU, _temp(), O.Opts(), threads=1)
    assert r["stats"][0]["status"] & O.ST_SINGULAR
    assert np.all(np.isfinite(r["ldos"]))


def test_sancho_cap_drops_lead_and_sets_status(oracle_mod):
    O = oracle_mod
    d = S.make_device(8, 3, seed=2)
    opts = O.Opts(sancho_nmax=3)
    r = O.rgf_batch(d.Hii, d.H1i, np.array([0.1]), MU, _temp(), opts, threads=1)
    assert r["stats"][0]["status"] & O.ST_SANCHO_NC
    assert r["stats"][0]["sancho_iters_left"] == 4
    t = O.rgf_numpy(O.to_blocks(d.Hii), O.to_blocks(d.H1i), 0.1, MU, _temp(), opts)
    assert rel_err(O.to_blocks(r["ldos"][0]), t["ldos"]) < 1e-10


def test_calc_n_electron_matches_loop(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(0)
    nk, nen, nx, nm = 2, 5, 3, 4
    Gl = rng.normal(size=(nk, nen, nx, nm, nm)) + 1j * rng.normal(size=(nk, nen, nx, nm, nm))
    Gg = rng.normal(size=(nk, nen, nx, nm, nm)) + 1j * rng.normal(size=(nk, nen, nx, nm, nm))
    E = np.linspace(-1, 1, nen)
    mid = np.array([-0.2, 0.0, 0.3])
    ne, pe = O.calc_n_electron(Gl, Gg, E, mid)
    dE = (E[1] - E[0]) / (2.0 * O.PI)
    dK = 2.0 * O.PI / nk
    ne2 = np.zeros(nx)
    pe2 = np.zeros(nx)
    for i in range(nen):
        for ik in range(nk):
            for ix in range(nx):
                for j in range(nm):
                    if E[i] > mid[ix]:
                        ne2[ix] += Gl[ik, i, ix, j, j].imag * dE * dK
                    else:
                        pe2[ix] -= Gg[ik, i, ix, j, j].imag * dE * dK
    assert np.allclose(ne, ne2, rtol=1e-13, atol=1e-15)
    assert np.allclose(pe, pe2, rtol=1e-13, atol=1e-15)


GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_reproduces_golden(oracle_mod, path):
    O = oracle_mod
    z = np.load(path)
    opts = O.Opts(eta_dev=float(z["eta_dev"]), eta_lead=float(z["eta_lead"]),
                  consistent=bool(z["consistent"]), boltz=float(z["boltz"]))
    sl = z["sig_lesser"] if z["has_sigma"] else None
    sr = z["sig_r"] if z["has_sigma"] else None
    Sii = z["Sii"] if "has_overlap" in z.files else None
    r = O.rgf_batch(z["Hii"], z["H1i"], z["E"], z["mu"], z["temp"], opts, sig_lesser=sl, sig_r=sr,
                    threads=2, Sii=Sii)
    for k in ("ldos", "ndens", "GRi1"):
        assert rel_err(r[k], z[k]) < 1e-12, k
    assert rel_err(r["pdens"], z["pdens"], scale=np.max(np.abs(z["ldos"]))) < 1e-12
    assert rel_err(r["T"], z["T"]) < 1e-12
    assert rel_err(r["tr"], z["tr"]) < 1e-10


def test_adjoint_restatement_matches_finite_differences(oracle_mod):
    """The analytic adjoint of T(E) (checker of rgf_adjoint_energies) against
    central differences of the C++ FP64 oracle, including the lead shift of
    the end blocks and the interior coupling scale."""
    O = oracle_mod
    nm, nx = 6, 5
    d = S.make_device(nm, nx, seed=7)
    Hb, H1b = O.to_blocks(d.Hii), O.to_blocks(d.H1i)
    opts = O.Opts(eta_dev=0.0, eta_lead=1e-3)
    E = np.array([-1.3, 0.4])
    fdV, fds = O.fd_gradient(d.Hii, d.H1i, E, MU, _temp(), opts, h=1e-5)
    for ie, e in enumerate(E):
        T, dV, ds = O.adjoint_numpy(Hb, H1b, e, opts)
        scale = np.max(np.abs(dV))
        assert np.max(np.abs(dV - fdV[ie])) < 1e-6 * scale
        assert abs(ds - fds[ie]) < 1e-6 * max(abs(ds), 1.0)


def test_calc_block_current_loops(oracle_mod):
    """calc_block_current against a direct transcription of its loops."""
    O = oracle_mod
    rng = np.random.default_rng(0)
    nb, ns, nx, nen = 3, 3, 2, 4
    nm = nb * ns
    H = rng.normal(size=(nx, nm, nm)) + 1j * rng.normal(size=(nx, nm, nm))
    G = rng.normal(size=(nen, nx, nm, nm)) + 1j * rng.normal(size=(nen, nx, nm, nm))
    E = np.linspace(-1, 1, nen)
    tc, te, jd = O.calc_block_current(H, G, E, 2.0, nb, ns, jdens=True)
    Hm, Gm = O.to_blocks(H), O.to_blocks(G)
    scale = (E[1] - E[0]) * O.E0 / 6.28318530718 / O.HBAR * O.E0 * 2.0
    ref = np.zeros((nx * ns, nb, nb))
    for ie in range(nen):
        for ix in range(nx):
            B = np.zeros((nb, nb))
            for ib in range(ns - 1):
                for io in range(nb):
                    for jo in range(nb):
                        i, j = io + ib * nb, jo + (ib + 1) * nb
                        B[io, jo] = ((Hm[ix][i, j] * Gm[ie, ix][j, i] - Hm[ix][j, i] * Gm[ie, ix][i, j]) * scale).real
                ref[ix * ns + ib] += B
            ref[ix * ns + ns - 1] += B
    assert np.allclose(O.to_blocks(tc), ref, rtol=1e-13, atol=1e-25)


def test_perturbed_inputs_stay_hermitian_and_close():
    from conftest import perturbed_inputs
    d = S.make_device(8, 3, seed=2)
    P, Q = perturbed_inputs(d.Hii, d.H1i, 0)
    for l in range(3):
        assert np.array_equal(P[l], P[l].conj().T)
    assert np.max(np.abs(P - d.Hii) / np.maximum(np.abs(d.Hii), 1e-300)) <= 2.0 ** -51
    assert np.max(np.abs(Q - d.H1i) / np.maximum(np.abs(d.H1i), 1e-300)) <= 2.0 ** -51
    assert not np.array_equal(P, d.Hii)


# ---------------------------------------------------------------- green_RGF_CMS
@pytest.mark.parametrize("consistent", [False, True])
@pytest.mark.parametrize("nm,nx,scatter", [(8, 5, True), (12, 3, False), (6, 2, True)])
def test_cms_cpp_matches_numpy_restatement(oracle_mod, consistent, nm, nx, scatter):
    O = oracle_mod
    d = S.make_device(nm, nx, seed=nm * 10 + nx)
    Sii = S.make_overlap(nm, nx, seed=nx)
    E = np.array([-1.9, -0.3, 0.6, 2.2])
    sl = sr = None
    if scatter:
        sl, sr = random_sigma(nm, nx, len(E), seed=17)
    opts = O.Opts(consistent=consistent)
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), opts, sig_lesser=sl, sig_r=sr, threads=2, Sii=Sii)
    Hb, H1b, Sb = O.to_blocks(d.Hii), O.to_blocks(d.H1i), O.to_blocks(Sii)
    for ie, e in enumerate(E):
        t = O.rgf_numpy(Hb, H1b, e, MU, _temp(), opts,
                        sigl=None if sl is None else O.to_blocks(sl[ie]),
                        sigr=None if sr is None else O.to_blocks(sr[ie]), Sb=Sb)
        for k in ("ldos", "ndens", "GRi1"):
            assert rel_err(O.to_blocks(r[k][ie]), t[k]) < 1e-9, k
        assert rel_err(O.to_blocks(r["pdens"][ie]), t["pdens"],
                       scale=max(np.max(np.abs(t["ldos"])), np.max(np.abs(t["ndens"])))) < 1e-9
        cur_scale = nm * np.max(np.abs(H1b)) * np.max(np.abs(t["ndens"]))
        assert rel_err(O.to_blocks(r["cur"][ie]), t["cur"], scale=cur_scale) < 1e-9
        assert abs(r["T"][ie] - t["T"]) < 1e-9 * max(1.0, abs(t["T"]))
        tr_scale = max(np.max(np.abs(r["tr"])), 1e-300)
        assert abs(r["tr"][ie] - t["tr"]) < 1e-8 * tr_scale + 1e-14 * nm
        assert abs(r["tre"][ie] - t["tre"]) < 1e-8 * tr_scale + 1e-14 * nm
        assert tuple(r["stats"][ie][["sancho_iters_left", "sancho_iters_right"]]) == t["iters"]


def test_cms_with_unit_overlap_is_rs_except_the_greater_recursion(oracle_mod):
    """With S = I, green_RGF_CMS computes what green_RGF_RS computes (bit for
    bit: the overlap products are exact), except G^>_ll for l < nx, which it
    recurses through the never-filled Glp instead of using the identity
    G^> = G^< + G^R - G^A, and GGi1, which uses that running G^>."""
    O = oracle_mod
    nm, nx = 8, 5
    d = S.make_device(nm, nx, seed=5)
    Sii = S._to_fortran_blocks(np.broadcast_to(np.eye(nm, dtype=complex), (nx, nm, nm)).copy())
    E = np.array([-0.8, 0.35])
    sl, sr = random_sigma(nm, nx, len(E), seed=2)
    outs = ("ldos", "ndens", "pdens", "cur", "GRi1", "GLi1", "GGi1")
    rs = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(), sig_lesser=sl, sig_r=sr, outputs=outs)
    cms = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), O.Opts(), sig_lesser=sl, sig_r=sr, outputs=outs,
                      Sii=Sii)
    for k in ("ldos", "ndens", "cur", "GRi1", "GLi1", "tr", "tre", "T"):
        assert np.array_equal(rs[k], cms[k]), k
    assert np.array_equal(rs["pdens"][:, -1], cms["pdens"][:, -1])
    assert not np.allclose(rs["pdens"][:, :-1], cms["pdens"][:, :-1])
    assert np.array_equal(rs["GGi1"][:, -2], cms["GGi1"][:, -2])  # both use the closure's G^> there


@pytest.mark.parametrize("nm,nx", [(4, 2), (6, 4)])
def test_cms_dense_inverse_known_answer(oracle_mod, nm, nx):
    """Consistent-mode CMS equals (E S - H - Sigma)^-1 of the whole device."""
    O = oracle_mod
    d = S.make_device(nm, nx, seed=21 + nm)
    Sii = S.make_overlap(nm, nx, seed=3)
    Hb, H1b, Sb = O.to_blocks(d.Hii), O.to_blocks(d.H1i), O.to_blocks(Sii)
    E = np.array([-1.1, 0.7])
    sl, sr = random_sigma(nm, nx, len(E), seed=4)
    opts = O.Opts(consistent=True, eta_dev=1e-4)
    r = O.rgf_batch(d.Hii, d.H1i, E, MU, _temp(), opts, sig_lesser=sl, sig_r=sr, threads=1, Sii=Sii)
    for ie, e in enumerate(E):
        t = O.rgf_numpy(Hb, H1b, e, MU, _temp(), opts, sigl=O.to_blocks(sl[ie]),
                        sigr=O.to_blocks(sr[ie]), Sb=Sb)
        G = O.dense_green(Hb, H1b, e, t["sigmal"], t["sigmar"], eta_dev=opts.eta_dev,
                          sigr=O.to_blocks(sr[ie]), Sb=Sb)
        ldos, gri1 = O.to_blocks(r["ldos"][ie]), O.to_blocks(r["GRi1"][ie])
        for l in range(nx):
            s = slice(l * nm, (l + 1) * nm)
            assert rel_err(ldos[l], G[s, s], scale=np.max(np.abs(G))) < 1e-10
            if l < nx - 1:
                s1 = slice((l + 1) * nm, (l + 2) * nm)
                assert rel_err(gri1[l], G[s, s1], scale=np.max(np.abs(G))) < 1e-10
        N = nm * nx
        Sl = np.zeros((N, N), complex)
        fl = O.ferm((e - MU[0]) / (opts.boltz * _temp()[0]))
        fr = O.ferm((e - MU[1]) / (opts.boltz * _temp()[0]))
        Sl[:nm, :nm] = -(t["sigmal"] - t["sigmal"].conj().T) * fl
        Sl[-nm:, -nm:] = -(t["sigmar"] - t["sigmar"].conj().T) * fr
        slb = O.to_blocks(sl[ie])
        for l in range(nx):
            Sl[l * nm:(l + 1) * nm, l * nm:(l + 1) * nm] += slb[l] @ Sb[l]
        Gless = G @ Sl @ G.conj().T
        nd = O.to_blocks(r["ndens"][ie])
        for l in range(nx):
            s = slice(l * nm, (l + 1) * nm)
            assert rel_err(nd[l], Gless[s, s], scale=np.max(np.abs(Gless))) < 1e-10
        gL = 1j * (t["sigmal"] - t["sigmal"].conj().T)
        gR = 1j * (t["sigmar"] - t["sigmar"].conj().T)
        GN1 = G[-nm:, :nm]
        T = np.real(np.trace(gL @ GN1.conj().T @ gR @ GN1))
        assert abs(r["T"][ie] - T) < 1e-10 * max(1.0, abs(T))


def test_cms_sancho_fixed_point_with_overlap(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(8)
    nm = 6
    X = rng.normal(size=(nm, nm)) + 1j * rng.normal(size=(nm, nm))
    H00 = 0.1 * (X + X.conj().T)
    H10 = -1.0 * (np.eye(nm) + 0.1 * rng.normal(size=(nm, nm)))
    S00 = O.to_blocks(S.make_overlap(nm, 1, seed=9))[0]
    opts = O.Opts()
    for E in (-0.7, 0.3, 1.1):
        G, _, it, st = O.sancho_numpy(E, H00, H10, opts, S00)
        assert st == 0 and it < opts.sancho_nmax
        z = complex(E, opts.eta_lead)
        R = G - np.linalg.inv(z * S00 - H00 - H10.conj().T @ G @ H10)
        assert np.linalg.norm(R) < 1e-8 * np.linalg.norm(G)


# ---------------------------------------------------------------- RGF_W
def _rand_blocks(rng, nx, nm, scale):
    return np.array([rng.normal(0, scale, (nm, nm)) + 1j * rng.normal(0, scale, (nm, nm)) for _ in range(nx)])


@pytest.mark.parametrize("nm,nx", [(6, 2), (6, 5), (10, 4)])
def test_w_cpp_matches_numpy_restatement(oracle_mod, nm, nx):
    """General (non-symmetric) inputs: the C++ and NumPy restatements of
    green_rgf_calc_w agree, transposes and quirks included."""
    O = oracle_mod
    rng = np.random.default_rng(nm + nx)
    Vb = np.array([np.eye(nm) + b + b.conj().T for b in _rand_blocks(rng, nx, nm, 0.15)])
    V1b = _rand_blocks(rng, nx, nm, 0.2)
    nE = 3
    P = [np.array([_rand_blocks(rng, nx, nm, 0.2) for _ in range(nE)]) for _ in range(3)]
    F = lambda a: np.array([O.from_blocks(x) for x in a]) if a.ndim == 4 else O.from_blocks(a)
    r = O.rgf_w_batch(F(Vb), F(V1b), F(P[0]), F(P[1]), F(P[2]), threads=2)
    for e in range(nE):
        t = O.rgf_w_numpy(Vb, V1b, P[0][e], P[1][e], P[2][e])
        for k in ("WR", "WL", "WG"):
            assert rel_err(O.to_blocks(r[k][e]), t[k]) < 1e-12, k
        assert rel_err(O.to_blocks(r["WRi1"][e])[:-1], t["WRi1"]) < 1e-12
        assert np.all(r["WRi1"][e][-1] == 0)
    st = r["stats"][0]
    # S blocks 3 nx - 2, right-to-left 4 (nx - 1) + 1, left-to-right 4 (nx - 1), W^< / W^> 12 nx
    assert st["n_inv"] == nx and st["n_gemm"] == 23 * nx - 9


@pytest.mark.parametrize("nm,nx", [(5, 3), (8, 6)])
def test_w_dense_known_answer(oracle_mod, nm, nx):
    """Coulomb V (real symmetric) and complex-symmetric P^R, the case the
    routine's transposes assume: W^R_ll and W^R_{l,l+1} equal the blocks of
    (I - V P^R)^-1 V of the whole device."""
    O = oracle_mod
    Vii, V1i = S.make_coulomb(nm, nx, seed=nm)
    PL, PG, PR = S.make_polarization(nm, nx, 2, seed=nx)
    r = O.rgf_w_batch(Vii, V1i, PL, PG, PR, threads=1)
    Vb, V1b = O.to_blocks(Vii), O.to_blocks(V1i)
    for e in range(2):
        W = O.dense_w(Vb, V1b, O.to_blocks(PR[e]))
        WR, Wo = O.to_blocks(r["WR"][e]), O.to_blocks(r["WRi1"][e])
        sc = np.max(np.abs(W))
        for l in range(nx):
            s = slice(l * nm, (l + 1) * nm)
            assert np.max(np.abs(WR[l] - W[s, s])) < 1e-12 * sc
            if l < nx - 1:
                s1 = slice((l + 1) * nm, (l + 2) * nm)
                assert np.max(np.abs(Wo[l] - W[s, s1])) < 1e-12 * sc


def test_w_lesser_formula_and_symmetry(oracle_mod):
    """W^< from the routine's formula: with the off-diagonal blocks' real part
    zeroed, WL_ll = WR P^< WR^H + neighbour terms; for anti-Hermitian P^< the
    result is anti-Hermitian."""
    O = oracle_mod
    nm, nx = 6, 4
    Vii, V1i = S.make_coulomb(nm, nx, seed=3)
    PL, PG, PR = S.make_polarization(nm, nx, 1, seed=5)
    r = O.rgf_w_batch(Vii, V1i, PL, PG, PR, threads=1)
    WL = O.to_blocks(r["WL"][0])
    for l in range(nx):
        assert np.max(np.abs(WL[l] + WL[l].conj().T)) < 1e-12 * np.max(np.abs(WL[l]))


# ------------------------------------------------------------ GW convolutions
def _gw_inputs(rng, nk, nen, nx, nm, n):
    return [rng.normal(size=(nk, nen, nx, nm, nm)) + 1j * rng.normal(size=(nk, nen, nx, nm, nm))
            for _ in range(n)]


def _swap(X):
    return np.ascontiguousarray(np.swapaxes(X, -1, -2))


@pytest.mark.parametrize("nky,nkz,ndiag", [(1, 1, 0), (2, 2, 2), (1, 3, 1), (3, 1, 4)])
def test_gw_polarization_cpp_matches_numpy(oracle_mod, nky, nkz, ndiag):
    O = oracle_mod
    rng = np.random.default_rng(nky * 10 + nkz)
    nk, nen, nx, nm = nky * nkz, 30, 3, 5
    G = _gw_inputs(rng, nk, nen, nx, nm, 3)
    P = O.gw_polarization(*[_swap(g) for g in G], nky, nkz, ndiag, 0.01, 2.0, imag_only=True, threads=2)
    Pn = O.gw_polarization_numpy(*[1j * g.imag for g in G], nky, nkz, ndiag, 0.01, 2.0)
    for a, b in zip(P, Pn):
        assert rel_err(_swap(a), b) < 1e-13


@pytest.mark.parametrize("nky,nkz,ndiag,nx", [(1, 2, 1, 6), (2, 1, 3, 4), (1, 1, 0, 3)])
def test_gw_self_energy_cpp_matches_numpy(oracle_mod, nky, nkz, ndiag, nx):
    O = oracle_mod
    rng = np.random.default_rng(nx + ndiag)
    nk, nen, nm = nky * nkz, 28, 4
    G = _gw_inputs(rng, nk, nen, nx, nm, 3)
    W = _gw_inputs(rng, nk, nen, nx, nm, 3)
    S = [np.zeros((nk, nen, nx, nm, nm), complex) for _ in range(3)]
    Sf = [_swap(s) for s in S]
    O.gw_self_energy(*[_swap(g) for g in G], *[_swap(w) for w in W], *Sf, nky, nkz, ndiag, 0.02, 0.7,
                     imag_only=True, threads=2)
    Sn = O.gw_self_energy_numpy(*[1j * g.imag for g in G], *W, *S, nky, nkz, ndiag, 0.02, 0.7)
    for a, b in zip(Sf, Sn):
        assert rel_err(_swap(a), b) < 1e-13
        assert np.max(np.abs(b)) > 0
