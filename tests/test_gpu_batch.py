"""GPU tests of uneven batches: devices of different block sizes nb and chain
lengths Nx in ONE persistent launch (rgf_solve_batch), the same task list as
a CUDA-graph plan (rgf_plan_*), and the autotuner (rgf_autotune).

Every task's outputs must be bit-identical to solving its device alone (a
task's arithmetic does not depend on what else is in the launch), and within
the FP64 tolerance of the CPU oracle."""
import numpy as np
import pytest

from conftest import compare, perturbed_inputs, random_sigma, rel_err
from liteqt_b200 import synthetic as S

pytestmark = pytest.mark.gpu

MU = (0.1, -0.1)
TOL = 1e-10


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


# (nb, nx, energies, scattering)
MIXED = [(32, 7, 5, False), (128, 3, 3, True), (48, 4, 4, False), (64, 9, 4, True),
         (32, 20, 3, False), (256, 2, 2, False), (24, 5, 3, False)]


def _batch(R, torch, dev):
    """Device-resident inputs / outputs of the mixed batch."""
    devices, tasks, keep, meta = [], [], [], []
    for di, (nb, nx, nen, scat) in enumerate(MIXED):
        d = S.make_device(nb, nx, seed=900 + di)
        E = S.energy_grid(nen, -2.5, 2.5) + 0.013 * di
        Hii = torch.from_numpy(d.Hii).to(dev)
        H1i = torch.from_numpy(d.H1i).to(dev)
        sl = sr = None
        if scat:
            sl_h, sr_h = random_sigma(nb, nx, nen, seed=di)
            sl, sr = torch.from_numpy(sl_h).to(dev), torch.from_numpy(sr_h).to(dev)
        cd = R.c_device()
        cd.nm, cd.nx = nb, nx
        cd.Hii, cd.H1i = Hii.data_ptr(), H1i.data_ptr()
        cd.mu[0], cd.mu[1] = MU
        cd.temp[0], cd.temp[1] = _temp()
        devices.append(cd)
        out = dict(ldos=torch.zeros((nen, nx, nb, nb), dtype=torch.complex128, device=dev))
        out["ndens"] = torch.zeros_like(out["ldos"])
        out["pdens"] = torch.zeros_like(out["ldos"])
        out["GRi1"] = torch.zeros_like(out["ldos"])
        out["cur"] = torch.zeros((nen, nx, nb, nb), dtype=torch.float64, device=dev)
        out["tr"] = torch.zeros(nen, dtype=torch.float64, device=dev)
        out["tre"] = torch.zeros_like(out["tr"])
        out["T"] = torch.zeros_like(out["tr"])
        for e in range(nen):
            t = R.c_task()
            t.device = di
            t.E = float(E[e])
            if scat:
                t.sigma_lesser, t.sigma_r = sl[e].data_ptr(), sr[e].data_ptr()
            for k in ("ldos", "ndens", "pdens", "GRi1", "cur"):
                setattr(t, k, out[k][e].data_ptr())
            for k in ("tr", "tre", "T"):
                setattr(t, k, out[k][e:e + 1].data_ptr())
            tasks.append(t)
        keep.append((Hii, H1i, sl, sr))
        meta.append(dict(d=d, E=E, out=out, sl=sl, sr=sr))
    return devices, tasks, keep, meta


def _alone(R, ctx, m):
    """The same device solved alone through rgf_solve_energies (host arrays)."""
    d, E = m["d"], m["E"]
    nen, nx, nb = len(E), d.nx, d.nm
    shape = (nen, nx, nb, nb)
    o = dict(ldos=np.zeros(shape, complex), ndens=np.zeros(shape, complex), pdens=np.zeros(shape, complex),
             GRi1=np.zeros(shape, complex), cur=np.zeros(shape), tr=np.zeros(nen), tre=np.zeros(nen),
             T=np.zeros(nen))
    sl = m["sl"].cpu().numpy() if m["sl"] is not None else None
    sr = m["sr"].cpu().numpy() if m["sr"] is not None else None
    ctx.solve_energies(d.Hii, d.H1i, E, MU, _temp(), sigma_lesser=sl, sigma_r=sr, **o)
    return o


def _check_parity(got, d, E, sl=None, sr=None):
    """GPU outputs against the FP64 oracle; where FP64 itself limits the
    agreement, against the 80-bit evaluation with the perturbed-input floor."""
    from oracle import oracle as O

    def orc(Hii, H1i, extended=False):
        return O.rgf_batch(Hii, H1i, E, MU, _temp(), O.Opts(), sig_lesser=sl, sig_r=sr, extended=extended)
    r = orc(d.Hii, d.H1i)
    try:
        compare(got, r, d.nm, d.H1i)
    except AssertionError:
        x = orc(d.Hii, d.H1i, extended=True)
        floor = [orc(*perturbed_inputs(d.Hii, d.H1i, seed)) for seed in range(2)]
        compare(got, r, d.nm, d.H1i, truth=x, floor=floor)


def _host(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


def test_mixed_block_sizes_in_one_launch(rgf):
    import torch
    dev = torch.device("cuda", 0)
    devices, tasks, keep, meta = _batch(rgf, torch, dev)
    info = np.zeros(len(tasks), rgf.INFO_DTYPE)
    with rgf.Context(rgf.Options()) as ctx:
        n0 = ctx.stats()["launches"]
        ctx.solve_batch(devices, tasks, info=info)
        torch.cuda.synchronize()
        assert ctx.stats()["launches"] - n0 == 1, "an uneven batch must run as one launch"
        assert np.all(info["status"] == 0)
        for m in meta:
            got = _host(m["out"])
            alone = _alone(rgf, ctx, m)
            for k in alone:
                assert np.array_equal(got[k], alone[k]), (m["d"].nm, m["d"].nx, k)
            sl = m["sl"].cpu().numpy() if m["sl"] is not None else None
            sr = m["sr"].cpu().numpy() if m["sr"] is not None else None
            _check_parity(got, m["d"], m["E"], sl, sr)


def test_plan_replays_and_reads_inputs_at_execution(rgf):
    import torch
    dev = torch.device("cuda", 0)
    devices, tasks, keep, meta = _batch(rgf, torch, dev)
    info = np.zeros(len(tasks), rgf.INFO_DTYPE)
    with rgf.Context(rgf.Options()) as ctx:
        ctx.solve_batch(devices, tasks, info=info)
        torch.cuda.synchronize()
        ref = [_host(m["out"]) for m in meta]
        for m in meta:
            for v in m["out"].values():
                v.zero_()
        with ctx.plan(devices, tasks) as plan:
            for rep in range(2):
                plan.execute(info=info)
                torch.cuda.synchronize()
                assert np.all(info["status"] == 0)
                for m, r in zip(meta, ref):
                    got = _host(m["out"])
                    for k in r:
                        assert np.array_equal(got[k], r[k]), (rep, m["d"].nm, k)
            # new scattering self-energies written in place are picked up by the replay
            m = meta[1]
            m["sl"].mul_(0.5)
            plan.execute()
            torch.cuda.synchronize()
            got = _host(m["out"])
            fresh = _alone(rgf, ctx, m)
            for k in ("ndens", "pdens", "tr"):
                assert np.array_equal(got[k], fresh[k]), k
            assert not np.array_equal(got["ndens"], ref[1]["ndens"])


def test_plan_rejects_host_arrays(rgf):
    d = S.make_device(32, 3, seed=1)
    cd = rgf.c_device()
    cd.nm, cd.nx = 32, 3
    cd.Hii, cd.H1i = d.Hii.ctypes.data, d.H1i.ctypes.data
    cd.temp[0] = cd.temp[1] = 300.0
    t = rgf.c_task()
    t.E = 0.1
    with rgf.Context(rgf.Options()) as ctx:
        with pytest.raises(rgf.RgfError, match="device memory"):
            ctx.plan([cd], [t])


@pytest.mark.parametrize("nb", [32, 48])
def test_autotune_picks_a_valid_variant_and_keeps_parity(rgf, nb):
    d = S.make_device(nb, 6, seed=31 + nb)
    E = S.energy_grid(6, -2.0, 2.0)
    with rgf.Context(rgf.Options()) as ctx:
        res = ctx.autotune(d.Hii, d.H1i, MU, _temp())
        assert res["nb"] == nb and res["ctas_per_sm"] >= 1
        names = [c[0] for c in res["candidates"]]
        assert res["variant"] in names
        expect = {"generic1x1", "generic1x2", "generic2x2"} | ({"staged32"} if nb == 32 else set())
        assert set(names) == expect
        best = min(c[2] for c in res["candidates"])
        assert [c for c in res["candidates"] if c[0] == res["variant"] and c[1] == res["ctas_per_sm"]][0][2] == best
        got = _alone(rgf, ctx, dict(d=d, E=E, sl=None, sr=None))
    _check_parity(got, d, E)


def test_T_only_solve_skips_nothing_it_needs(rgf):
    """A solve that asks only for T and tr (no block outputs) skips the
    backward sweep; T and tr are bit-identical to the full solve's."""
    d = S.make_device(64, 8, seed=12)
    E = S.energy_grid(5, -2.0, 2.0)
    shape = (len(E), d.nx, 64, 64)
    full = dict(ldos=np.zeros(shape, complex), ndens=np.zeros(shape, complex), T=np.zeros(len(E)),
                tr=np.zeros(len(E)), tre=np.zeros(len(E)))
    part = dict(T=np.zeros(len(E)), tr=np.zeros(len(E)))
    info_f = np.zeros(len(E), rgf.INFO_DTYPE)
    info_p = np.zeros(len(E), rgf.INFO_DTYPE)
    with rgf.Context(rgf.Options()) as ctx:
        ctx.solve_energies(d.Hii, d.H1i, E, MU, _temp(), info=info_f, **full)
        ctx.solve_energies(d.Hii, d.H1i, E, MU, _temp(), info=info_p, **part)
    assert np.array_equal(part["T"], full["T"]) and np.array_equal(part["tr"], full["tr"])
    assert np.all(info_p["n_gemm"] < info_f["n_gemm"])


def test_pipelined_calls_match_synchronous_calls(rgf):
    """rgf_opts.pipelined: calls return once queued, outputs staged in two
    alternating device buffers and copied on the context's copy stream, the
    blocks of the backward sweep as the kernel reports them written; after
    rgf_ctx_synchronize every pinned host output (block outputs of both
    element types, the untouched last block of GRi1, the scalars) equals
    the synchronous call's, bit for bit (three calls in a row, the first and
    third into the same arrays), and the statistics are those of the last
    call."""
    import torch
    from liteqt_b200 import synthetic as S
    nm, nx, nen = 32, 12, 40
    d = S.make_device(nm, nx, seed=31)
    temp = (S.temperature_for_kT(0.025),) * 2
    Es = [S.energy_grid(nen, -2.5, 2.5) + 0.01 * k for k in range(3)]

    def pinned():
        o = {k: torch.zeros((nen, nx, nm, nm), dtype=torch.complex128).pin_memory()
             for k in ("ldos", "ndens", "pdens", "GRi1")}
        o["GRi1"].fill_(complex(3.0, -1.0))   # block nx is left untouched
        o["cur"] = torch.zeros((nen, nx, nm, nm), dtype=torch.float64).pin_memory()
        o.update({k: torch.zeros(nen, dtype=torch.float64).pin_memory() for k in ("T", "tr", "tre")})
        return o
    want = []
    with rgf.Context(rgf.Options(eta_dev=1e-5, eta_lead=1e-5)) as ctx:
        for E in Es:
            o = pinned()
            ctx.solve_energies(d.Hii, d.H1i, E, (0.1, -0.1), temp, **{k: v.numpy() for k, v in o.items()})
            want.append({k: v.numpy().copy() for k, v in o.items()})
    A, B = pinned(), pinned()
    outs = [A, B, A]
    with rgf.Context(rgf.Options(eta_dev=1e-5, eta_lead=1e-5, pipelined=True)) as ctx:
        got = []
        for k, E in enumerate(Es):
            ctx.solve_energies(d.Hii, d.H1i, E, (0.1, -0.1), temp, **{n: v.numpy() for n, v in outs[k].items()})
            if k == 1:   # the second call's outputs are final once the context is synchronised
                ctx.synchronize()
                got.append({n: v.numpy().copy() for n, v in B.items()})
        ctx.synchronize()
        got.append({n: v.numpy().copy() for n, v in A.items()})
        st = ctx.stats()
    for g, w in zip(got, (want[1], want[2])):
        for n in w:
            assert np.array_equal(g[n], w[n]), n
    assert st["last_tasks"] == nen and st["last_kernel_ms"] > 0 and st["last_flops"] > 0


def test_pageable_host_arrays_match_device_arrays(rgf):
    """Pageable (not page-locked) host inputs and outputs go through the
    library's bounce copier (pinned slots of 8 MB, a landing thread, host
    side split over a thread pool) in both directions.  With per-energy
    Sigma^R / Sigma^< and every output kind about 126 MB per array -- many
    passes over the sixteen slots -- a synchronous call and a pipelined call
    on pageable NumPy arrays, and a synchronous call on page-locked arrays
    with zero copy off (outputs copied by DMA as their blocks are written),
    give bit for bit the outputs of the same solve on device-resident arrays,
    and block nx of GRi1, which the solver never writes, keeps its host value
    in all of them."""
    import torch
    nm, nx, nen = 64, 40, 48
    d = S.make_device(nm, nx, seed=41)
    E = S.energy_grid(nen, -2.5, 2.5)
    rng = np.random.default_rng(5)
    shape = (nen, nx, nm, nm)
    eye = np.eye(nm)
    sig_r = np.ascontiguousarray(np.broadcast_to(-0.01j * eye, shape)
                                 + 1e-3 * (rng.normal(size=shape) + 1j * rng.normal(size=shape)))
    sig_l = np.ascontiguousarray(np.broadcast_to(0.004j * eye, shape)
                                 + 1e-4 * (rng.normal(size=shape) + 1j * rng.normal(size=shape)))
    kinds = ("ldos", "ndens", "pdens", "GRi1")

    def host_outs():
        o = {k: np.zeros(shape, complex) for k in kinds}
        o["GRi1"][:] = complex(3.0, -1.0)
        o["cur"] = np.zeros(shape)
        o.update({k: np.zeros(nen) for k in ("tr", "tre")})
        return o
    opts = dict(eta_dev=1e-5, eta_lead=1e-5)
    dev = {k: torch.full(shape, complex(3.0, -1.0), dtype=torch.complex128, device="cuda") for k in kinds}
    dev["cur"] = torch.zeros(shape, dtype=torch.float64, device="cuda")
    dev.update({k: torch.zeros(nen, dtype=torch.float64, device="cuda") for k in ("tr", "tre")})
    with rgf.Context(rgf.Options(**opts)) as ctx:
        ctx.solve_energies(torch.from_numpy(d.Hii).cuda(), torch.from_numpy(d.H1i).cuda(), E, MU, _temp(),
                           sigma_lesser=torch.from_numpy(sig_l).cuda(), sigma_r=torch.from_numpy(sig_r).cuda(),
                           **dev)
        torch.cuda.synchronize()
        want = {k: v.cpu().numpy() for k, v in dev.items()}
        sync = host_outs()
        ctx.solve_energies(d.Hii, d.H1i, E, MU, _temp(), sigma_lesser=sig_l, sigma_r=sig_r, **sync)
    with rgf.Context(rgf.Options(pipelined=True, **opts)) as ctx:
        pipe = host_outs()
        ctx.solve_energies(d.Hii, d.H1i, E, MU, _temp(), sigma_lesser=sig_l, sigma_r=sig_r, **pipe)
        ctx.synchronize()
    # page-locked outputs staged (zero_copy off): a synchronous call copies
    # them by DMA as the kernel reports their blocks written
    pinned = {k: torch.from_numpy(v).pin_memory() for k, v in host_outs().items()}
    with rgf.Context(rgf.Options(zero_copy=False, **opts)) as ctx:
        ctx.solve_energies(d.Hii, d.H1i, E, MU, _temp(), sigma_lesser=sig_l, sigma_r=sig_r,
                           **{k: v.numpy() for k, v in pinned.items()})
    pin = {k: v.numpy() for k, v in pinned.items()}
    assert np.all(want["GRi1"][:, -1] == complex(3.0, -1.0))
    for got in (sync, pipe, pin):
        for k in want:
            assert np.array_equal(got[k], want[k]), k
