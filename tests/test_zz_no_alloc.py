"""The allocation-free entry point rgf_solve_energies_noalloc.

Some callers cannot let the library allocate device memory: host codes that
hand all of HBM to their own memory pool at start-up, or that call the
solver inside a loop where cudaMalloc's implicit device synchronisation is
not acceptable.  rgf_solve_energies_noalloc works only on the caller's
device arrays and on a fixed scratch array built into the library.  This
test calls it through the C ABI twice in a row and checks each result
against the allocating entry point rgf_solve_energies on the same inputs,
with the tolerance of the other GPU parity tests.  It lives in a file of its
own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest

from liteqt_b200 import synthetic as S

pytestmark = pytest.mark.gpu

TOL = 1e-10
MU = (0.1, -0.1)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf
    build.build()
    L = rgf.load()
    P = ctypes.c_void_p
    L.rgf_solve_energies_noalloc.argtypes = [ctypes.POINTER(rgf.c_opts), ctypes.POINTER(rgf.c_device),
                                             ctypes.c_int64] + [P] * 13
    L.rgf_solve_energies_noalloc.restype = ctypes.c_int
    L.rgf_noalloc_last_error.restype = ctypes.c_char_p
    return L


def _device_problem(nm, nx, nen, seed, emin, emax):
    import torch
    d = S.make_device(nm, nx, seed=seed)
    dev = torch.device("cuda:0")
    Hii = torch.from_numpy(d.Hii).to(dev)
    H1i = torch.from_numpy(d.H1i).to(dev)
    E = S.energy_grid(nen, emin, emax)
    return d, Hii, H1i, E


def _outputs(nen, nx, nm):
    import torch
    dev = torch.device("cuda:0")
    shape = (nen, nx, nm, nm)
    return dict(ldos=torch.full(shape, 7.0, dtype=torch.complex128, device=dev),
                ndens=torch.full(shape, 7.0, dtype=torch.complex128, device=dev),
                T=torch.full((nen,), 7.0, dtype=torch.float64, device=dev),
                tr=torch.full((nen,), 7.0, dtype=torch.float64, device=dev))


def _call_noalloc(L, opts, nm, nx, Hii, H1i, E, out):
    from liteqt_b200 import rgf
    d = rgf.c_device()
    d.nm, d.nx = nm, nx
    d.Hii, d.H1i = Hii.data_ptr(), H1i.data_ptr()
    d.mu[0], d.mu[1] = MU
    d.temp[0] = d.temp[1] = S.temperature_for_kT(0.025)
    o = opts.c()
    info = np.zeros(len(E), rgf.INFO_DTYPE)
    rc = L.rgf_solve_energies_noalloc(ctypes.byref(o), ctypes.byref(d), len(E), E.ctypes.data, None,
                                      None, out["ldos"].data_ptr(), out["ndens"].data_ptr(), None,
                                      None, None, out["tr"].data_ptr(), None, out["T"].data_ptr(),
                                      info.ctypes.data, None)
    return rc, info


def test_no_alloc_matches_allocating_entry_point_twice(lib):
    import torch
    from liteqt_b200 import rgf
    nm, nx, nen = 32, 12, 40
    opts = rgf.Options(eta_dev=0.0, eta_lead=1e-3)
    for call, (seed, emin, emax) in enumerate(((11, -3.0, 3.0), (12, -1.0, 2.0))):
        d, Hii, H1i, E = _device_problem(nm, nx, nen, seed, emin, emax)
        ref = _outputs(nen, nx, nm)
        with rgf.Context(opts) as ctx:
            ctx.solve_energies(Hii, H1i, E, MU, (S.temperature_for_kT(0.025),) * 2, ldos=ref["ldos"],
                               ndens=ref["ndens"], tr=ref["tr"], T=ref["T"])
        got = _outputs(nen, nx, nm)
        rc, info = _call_noalloc(lib, opts, nm, nx, Hii, H1i, E, got)
        assert rc == 0, lib.rgf_noalloc_last_error().decode()
        assert np.all(info["status"] == 0)
        torch.cuda.synchronize()
        for k in ("ldos", "ndens", "T", "tr"):
            a = got[k].cpu().numpy()
            b = ref[k].cpu().numpy()
            assert _rel(a, b) <= TOL, (call, k, _rel(a, b))


def test_no_alloc_rejects_oversized_problem_and_host_arrays(lib):
    import torch
    from liteqt_b200 import rgf
    opts = rgf.Options()
    # nm = 256, nx = 200: one solver slot alone is (2*200 + 32) * 256^2 * 16 B = 453 MB
    nm, nx = 256, 200
    dev = torch.device("cuda:0")
    Hii = torch.zeros((nx, nm, nm), dtype=torch.complex128, device=dev)
    out = _outputs(1, 2, 8)
    rc, _ = _call_noalloc(lib, opts, nm, nx, Hii, Hii, np.array([0.1]), out)
    assert rc == rgf.RGF_E_ARG
    assert "too large" in lib.rgf_noalloc_last_error().decode()
    # host arrays are refused (they would need staging buffers)
    d = S.make_device(8, 3, seed=1)
    o = opts.c()
    cd = rgf.c_device()
    cd.nm, cd.nx = 8, 3
    cd.Hii, cd.H1i = d.Hii.ctypes.data, d.H1i.ctypes.data
    cd.temp[0] = cd.temp[1] = 290.0
    E = np.array([0.1])
    rc = lib.rgf_solve_energies_noalloc(ctypes.byref(o), ctypes.byref(cd), 1, E.ctypes.data,
                                        *([None] * 12))
    assert rc == rgf.RGF_E_ARG
    assert "device memory" in lib.rgf_noalloc_last_error().decode()


def test_no_alloc_nb128_matches_allocating_entry_point(lib):
    """nb = 128 with a chain of 24 blocks: one solver slot is 15 MB, so the
    256 MiB scratch holds 16 slots and the launch runs 16 CTAs; the results
    must still equal the allocating entry point's."""
    import torch
    from liteqt_b200 import rgf
    nm, nx, nen = 128, 24, 20
    opts = rgf.Options(eta_dev=1e-5, eta_lead=1e-5)
    d, Hii, H1i, E = _device_problem(nm, nx, nen, 21, -2.5, 2.5)
    ref = _outputs(nen, nx, nm)
    with rgf.Context(opts) as ctx:
        ctx.solve_energies(Hii, H1i, E, MU, (S.temperature_for_kT(0.025),) * 2, ldos=ref["ldos"],
                           ndens=ref["ndens"], tr=ref["tr"], T=ref["T"])
    got = _outputs(nen, nx, nm)
    rc, info = _call_noalloc(lib, opts, nm, nx, Hii, H1i, E, got)
    assert rc == 0, lib.rgf_noalloc_last_error().decode()
    assert np.all(info["status"] == 0)
    torch.cuda.synchronize()
    for k in ("ldos", "ndens", "T", "tr"):
        a = got[k].cpu().numpy()
        b = ref[k].cpu().numpy()
        assert _rel(a, b) <= TOL, (k, _rel(a, b))
