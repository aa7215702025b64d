#!/usr/bin/env python
"""RGF throughput benchmark: energy points per second on B200.

Workload (``rgf_nb128_nx100``): one seeded synthetic tight-binding chain
(nb = 128 orbitals per block, Nx = 100 blocks, H_ll Hermitian with diagonal
U[-0.5,0.5] eV and off-diagonal N(0,0.1) eV, H_{l,l-1} = -2.7 eV (I + N(0,0.05))),
semi-infinite leads by Sancho-Rubio, eta = 1e-5 eV in device and leads,
mu = (+0.1, -0.1) eV, kT = 0.025 eV, energies on the uniform grid of
[-3, 3] eV.  One step = one batched solve of --nen energies per GPU producing
G^R_ll, G^<_ll (all diagonal blocks), T(E) and the contact current spectra
tr / tre.  Synthetic data: no dataset is involved.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  ``value`` is measured with inputs resident in HBM
(CUDA events on the solver's stream, L2 flushed between steps); ``e2e`` is the
same metric through the public C ABI with pinned host buffers, host<->device
copies inside the timed region.  ``--impl reference`` times the CPU oracle
(the C++ restatement of the reference's green_RGF_RS, one energy per host
thread with single-threaded OpenBLAS, as the reference's `!$omp do ie`).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RGF energy-pts/s (G^R,G^<,T) mixed vs plain FP64 on 1 B200 at rel err ≤1e-8"
UNIT = "energy-pts/s"
MU = (0.1, -0.1)
KT = 0.025
ETA = 1e-5


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--nb", type=int, default=128)
    p.add_argument("--nx", type=int, default=100)
    p.add_argument("--nen", type=int, default=296, help="energies per GPU per step")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                   help="form of the headline value: fp64 (default), the plain drop-in form; mixed, "
                        "split-integer block products on the int8 tensor cores (nb = 128).  The other form "
                        "is timed beside it on the same workload (mixed_vs_plain)")
    p.add_argument("--no-other", action="store_true", help="skip timing the other precision form")
    p.add_argument("--full-outputs", action="store_true",
                   help="request the reference's full output set per energy (G^R_ll, G^<_ll, G^>_ll, the bond "
                        "current cur, G^R_{l,l+1}, tr, tre, T) instead of G^R_ll, G^<_ll, T, tr, tre")
    p.add_argument("--consistent", action="store_true",
                   help="the consistent backward coupling H1i(:,:,l+1) instead of the reference's H1i(:,:,l)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-threads", type=int, default=0)
    p.add_argument("--adjoint", action="store_true",
                   help="time the adjoint (dT/dV_l, dT/ds, dI/dV_l) against forward solves on the "
                        "adjoint workload (nb=64, Nx=200, per-block potential U[-0.2,0.2] eV)")
    p.add_argument("--w", action="store_true",
                   help="time the screened-interaction solve (green_rgf_calc_w) on the GW workload "
                        "(nb=64, Nx=40, Coulomb V, 2048 polarization sets per step)")
    p.add_argument("--gw", action="store_true",
                   help="time the GW-loop convolutions (polarization, self-energy) on a 2x2 k-grid, "
                        "nen=512, nx=10, nm=16, ndiag=3")
    p.add_argument("--blocks", action="store_true",
                   help="time the building blocks alone (FP64 and split-integer products, FP64 and refined FP32 "
                        "inverses) on 1480 blocks of 128 x 128, one CTA per SM")
    p.add_argument("--gw-fft", action="store_true",
                   help="time the FFT form of the GW convolutions (rgf_gw_polarization_fft / "
                        "rgf_gw_self_energy_fft) at nk=16, nen=4096, nx=40, nm=64 on one rank's (i,j) slice")
    p.add_argument("--dropin", action="store_true",
                   help="time the per-energy drop-in green_RGF_RS called from every host thread at once, "
                        "each on its own energies (the reference's `!$omp do` loop), against the batched "
                        "entry point on the same energies and outputs")
    p.add_argument("--per-thread", type=int, default=2,
                   help="energies each host thread solves in --dropin (the thread count is --cpu-threads, "
                        "default every host thread; OMP_NUM_THREADS plays that role for the reference's loop)")
    p.add_argument("--uneven", action="store_true",
                   help="uneven batch: 64 devices, Nx in {20..200}, nb in {32,64,128}, one graph-replayed "
                        "persistent launch (--nen energies per device per step; default 32)")
    p.add_argument("--band-edge", action="store_true",
                   help="band-edge workload: nb=256, Nx=64, eta=1e-6, 10%% of a 4096-point grid within 1e-3 eV "
                        "of lead subband edges (--nen sampled energies per step)")
    p.add_argument("--aux", action="store_true",
                   help="time the routines around the solve (redistribution transpose, calc_n_electron, "
                        "calc_block_current, the writers' GPU sums) on arrays of the output size")
    p.add_argument("--single", action="store_true",
                   help="one device-resident solve and exit (for profiler captures; prints no JSON)")
    return p.parse_args()


def workload(args, world=1):
    from liteqt_b200 import synthetic as S
    d = S.make_device(args.nb, args.nx, seed=1)
    E_all = S.energy_grid(args.nen * world, -3.0, 3.0)
    temp = (S.temperature_for_kT(KT),) * 2
    return d, E_all, temp


def config(args, world):
    return {"workload": f"rgf_nb{args.nb}_nx{args.nx}", "nb": args.nb, "nx": args.nx,
            "energies_per_gpu_per_step": args.nen, "energy_range_eV": [-3.0, 3.0], "eta_eV": ETA,
            "mu_eV": list(MU), "kT_eV": KT,
            "outputs": (["G^R_ll", "G^<_ll", "G^>_ll", "cur", "G^R_l,l+1", "T", "tr", "tre"]
                        if args.full_outputs else ["G^R_ll", "G^<_ll", "T", "tr", "tre"]),
            "precision": args.precision, "parallelism": f"energy-sharded x{world}",
            "backward_coupling": "H1i(l+1) (consistent)" if args.consistent else "H1i(l) (the reference's)",
            "l2": "flushed between timed steps (256 MiB write)", "seed": 1}


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(parts)
            except ValueError:
                pass
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------- helpers
def zgemm_peak_tflops(torch, dev):
    """Measured FP64 complex GEMM throughput (cuBLAS ZGEMM 4096^3) on this GPU:
    the roofline denominator of the FP64 tensor pipe."""
    a = torch.randn(4096, 4096, dtype=torch.complex128, device=dev)
    b = torch.randn_like(a)
    best = 1e30
    for _ in range(4):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 8.0 * 4096 ** 3 / (best * 1e-3) / 1e12


def int8_peak_tops():
    """Dense int8 tensor peak: twice the measured dense bf16 burst (the
    B200's int8 MMA rate is twice its bf16 rate per clock)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    bf16 = 1590.0   # the recipe's fallback when the measured file is absent
    if os.path.exists(path):
        bf16 = float(json.load(open(path)).get("bf16_tflops", bf16))
    return 2.0 * bf16


def traffic_from_profiles(args):
    """Per-task DRAM bytes of the solver kernel (the form --precision names)
    from the committed ncu summary, scaled to a launch of --nen tasks (None if
    no summary exists or the output set is not the summary's)."""
    if args.full_outputs:
        return None
    path = os.path.join(ROOT, "profiles", f"rgf_{args.precision}_nb{args.nb}_nx{args.nx}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_task:"):
            return float(line.split(":")[1].split()[0]) * args.nen
    return None


def cpu_baseline(args, d, E, temp, threads, min_seconds=10.0):
    """The CPU oracle on a bounded sample of the workload: rounds of one energy
    per host thread (single-threaded OpenBLAS per call) until at least
    min_seconds of wall time have been spent."""
    from oracle import oracle as O
    opts = O.Opts(eta_dev=ETA, eta_lead=ETA)
    O.lib()
    done, dt, r = 0, 0.0, 0
    while dt < min_seconds and r < 64:
        idx = (np.arange(threads) * 37 + r * threads) % len(E)
        t0 = time.perf_counter()
        O.rgf_batch(d.Hii, d.H1i, E[idx], MU, temp, opts, outputs=("ldos", "ndens"), threads=threads)
        dt += time.perf_counter() - t0
        done += threads
        r += 1
    return {"value": done / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{done} energies of rgf_nb{args.nb}_nx{args.nx} (eta=1e-5) in {r} rounds of one per "
                      f"host thread, full green_RGF_RS work + T(E), {dt:.1f} s wall"}


def host_threads(args):
    if args.cpu_threads > 0:
        return args.cpu_threads
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, n)


# --------------------------------------------------------------------- arms
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    d, E, temp = workload(args)
    threads = host_threads(args)
    opts = O.Opts(eta_dev=ETA, eta_lead=ETA)
    O.lib()
    idx_all = np.arange(len(E))
    times = []
    n_per = threads
    for step in range(args.warmup + args.steps):
        idx = idx_all[(step * n_per + np.arange(n_per)) % len(E)]
        t0 = time.perf_counter()
        O.rgf_batch(d.Hii, d.H1i, E[idx], MU, temp, opts, outputs=("ldos", "ndens"), threads=threads)
        if step >= args.warmup:
            times.append(time.perf_counter() - t0)
    total = sum(times)
    value = n_per * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config(args, 1),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n_per} energies per step of rgf_nb{args.nb}_nx{args.nx}, one per "
                                       "host thread (oracle: C++ restatement of green_RGF_RS + "
                                       "single-threaded OpenBLAS; the Fortran reference cannot be "
                                       "compiled here)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    from liteqt_b200 import rgf

    d, E_all, temp = workload(args, world)
    E = np.ascontiguousarray(E_all[rank * args.nen:(rank + 1) * args.nen])
    nen, nx, nb = args.nen, args.nx, args.nb
    mixed = args.precision == "mixed"
    opts = rgf.Options(device=local, eta_dev=ETA, eta_lead=ETA, consistent=args.consistent,
                       precision=rgf.RGF_PREC_MIXED if mixed else rgf.RGF_PREC_FP64)
    ctx = rgf.Context(opts)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream

    # device-resident inputs and outputs
    Hii = torch.from_numpy(d.Hii).to(dev)
    H1i = torch.from_numpy(d.H1i).to(dev)
    shape = (nen, nx, nb, nb)
    ldos = torch.empty(shape, dtype=torch.complex128, device=dev)
    ndens = torch.empty_like(ldos)
    T = torch.empty(nen, dtype=torch.float64, device=dev)
    tr = torch.empty_like(T)
    tre = torch.empty_like(T)
    extra = {}
    if args.full_outputs:
        extra = dict(pdens=torch.empty_like(ldos), GRi1=torch.empty_like(ldos),
                     cur=torch.empty(shape, dtype=torch.float64, device=dev))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    peak = zgemm_peak_tflops(torch, dev)

    def step_dev():
        ctx.solve_energies(Hii, H1i, E, MU, temp, ldos=ldos, ndens=ndens, tr=tr, tre=tre, T=T,
                           stream=sh, **extra)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step_dev()
    clocks = ClockSampler(local)
    launches0 = ctx.stats()["launches"]
    barrier()
    clocks.start()
    step_ms = []
    kern_ms = []
    flops = []
    int8_ops = []
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.fill_(1.0)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            step_dev()
            e.record(stream)
            e.synchronize()
            step_ms.append(s.elapsed_time(e))
            st = ctx.stats()
            kern_ms.append(st["last_kernel_ms"])
            flops.append(st["last_flops"])
            int8_ops.append(st["last_int8_ops"])
    barrier()
    clk = clocks.stop()
    launches = ctx.stats()["launches"] - launches0


    t_dev = sum(step_ms) / 1e3
    if world > 1:
        tt = torch.tensor([t_dev], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_dev = float(tt.item())
    value = nen * world * args.steps / t_dev

    # algorithmic work of the launch: the reference algorithm's operation count
    # per energy, 8 nb^3 (N_gemm + N_inv) with N_gemm = 28 Nx - 18 + 6 (nL + nR)
    # and N_inv = Nx + 4 + nL + nR (nL, nR = Sancho-Rubio iterations of the
    # task, identical to the reference's), summed over the launch's energies.
    info = np.zeros(nen, rgf.INFO_DTYPE)
    ctx.solve_energies(Hii, H1i, E, MU, temp, ldos=ldos, ndens=ndens, tr=tr, tre=tre, T=T,
                       info=info, stream=sh, **extra)
    torch.cuda.synchronize(dev)
    nsum = info["sancho_iters_left"].astype(np.float64) + info["sancho_iters_right"]
    alg_flops = float(np.sum(8.0 * nb ** 3 * ((28 * nx - 18 + 6 * nsum) + (nx + 4 + nsum))))
    kern_s = float(np.mean(kern_ms)) * 1e-3
    achieved = alg_flops / kern_s / 1e12
    fp64_exec = float(np.mean(flops))
    if not mixed:
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": traffic_from_profiles(args),
                    "peak_source": "cuBLAS ZGEMM 4096^3 measured live on this GPU (FP64 tensor pipe; "
                                   "MEASURED_PEAKS.json holds no FP64 figure)",
                    "algorithmic_flops_per_launch": alg_flops, "kernel_ms": 1e3 * kern_s,
                    "executed_flops_per_launch": fp64_exec,
                    "executed_tflops": fp64_exec / kern_s / 1e12,
                    "executed_frac": fp64_exec / kern_s / 1e12 / peak}
    else:
        # The mixed form's kernel runs two tensor pipes: int8 for the split-
        # integer products, FP64 DMMA for the lead decimation and the FP64
        # fallbacks.  Its roofline time is the sum of the two executed works
        # at their peaks; `peak` is the algorithmic rate the kernel would
        # reach in that time, so frac = (t_int8 + t_fp64) at peak / t_kernel.
        i8 = float(np.mean(int8_ops))
        i8_peak = int8_peak_tops()
        t_min = i8 / (i8_peak * 1e12) + fp64_exec / (peak * 1e12)
        roofline = {"bound": "tensor", "achieved": achieved, "peak": alg_flops / t_min / 1e12,
                    "unit": "TFLOP/s", "frac": t_min / kern_s, "traffic": traffic_from_profiles(args),
                    "peak_source": "int8 tensor: 2 x the measured dense bf16 burst of MEASURED_PEAKS.json "
                                   "(the B200 int8 rate is twice bf16 per clock); FP64 tensor: cuBLAS ZGEMM "
                                   "4096^3 measured live",
                    "algorithmic_flops_per_launch": alg_flops, "kernel_ms": 1e3 * kern_s,
                    "int8_ops_per_launch": i8, "int8_tops": i8 / kern_s / 1e12, "int8_peak_tops": i8_peak,
                    "int8_frac": i8 / kern_s / 1e12 / i8_peak,
                    "fp64_flops_per_launch": fp64_exec, "fp64_tflops": fp64_exec / kern_s / 1e12,
                    "fp64_peak_tflops": peak, "fp64_frac": fp64_exec / kern_s / 1e12 / peak}

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        Hii_h = torch.from_numpy(d.Hii).pin_memory()
        H1i_h = torch.from_numpy(d.H1i).pin_memory()
        ldos_h = torch.empty(shape, dtype=torch.complex128).pin_memory()
        ndens_h = torch.empty(shape, dtype=torch.complex128).pin_memory()
        T_h = torch.empty(nen, dtype=torch.float64).pin_memory()
        tr_h = torch.empty_like(T_h).pin_memory()
        tre_h = torch.empty_like(T_h).pin_memory()
        arrs = dict(ldos=ldos_h.numpy(), ndens=ndens_h.numpy(), T=T_h.numpy(), tr=tr_h.numpy(),
                    tre=tre_h.numpy())
        extra_h = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in extra.items()}
        arrs.update({k: v.numpy() for k, v in extra_h.items()})

        # (a) one synchronous call per step (outputs written through their
        # device mapping while the solve runs)
        def step_host():
            ctx.solve_energies(Hii_h.numpy(), H1i_h.numpy(), E, MU, temp, stream=sh, **arrs)
        step_host()
        barrier()
        ms = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            step_host()
            ms.append((time.perf_counter() - t0) * 1e3)
        barrier()
        t_sync = sum(ms) / 1e3
        # parity spot check of the e2e outputs against the device-resident run
        assert np.array_equal(arrs["T"], T.cpu().numpy())
        # (b) pipelined calls (rgf_opts.pipelined): each call returns once its
        # solve and output copies are queued; the copy engine takes one
        # step's 15.5 GB to the host while the next step solves; the timed
        # region ends with rgf_ctx_synchronize, when every output is on the host
        popts = rgf.Options(device=local, eta_dev=ETA, eta_lead=ETA, consistent=args.consistent,
                            precision=opts.precision, pipelined=True)
        pctx = rgf.Context(popts)

        def step_pipe():
            pctx.solve_energies(Hii_h.numpy(), H1i_h.numpy(), E, MU, temp, stream=sh, **arrs)
        for _ in range(2):
            step_pipe()
        pctx.synchronize()
        barrier()
        T_h.zero_()
        with torch.cuda.stream(stream):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                flush.fill_(1.0)
                step_pipe()
            pctx.synchronize()
            t_e2e = time.perf_counter() - t0
        barrier()
        assert np.array_equal(arrs["T"], T.cpu().numpy())
        # (c) the same pipelined calls on pageable NumPy arrays, as a Fortran
        # caller passes them: the library moves them through its pinned
        # bounce slots (pool of host threads for the pageable side).  One
        # GPU only: every rank would hold another 15.5 GB of host arrays
        t_pg = None
        if world == 1:
            pg = {k: np.empty(v.shape, v.dtype) for k, v in arrs.items()}
            Hii_p, H1i_p = np.array(d.Hii), np.array(d.H1i)

            def step_pageable():
                pctx.solve_energies(Hii_p, H1i_p, E, MU, temp, stream=sh, **pg)
            for _ in range(2):
                step_pageable()
            pctx.synchronize()
            with torch.cuda.stream(stream):
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                for _ in range(args.steps):
                    flush.fill_(1.0)
                    step_pageable()
                pctx.synchronize()
                t_pg = time.perf_counter() - t0
            assert np.array_equal(pg["T"], T.cpu().numpy())
            del pg
        pctx.close()
        if world > 1:
            tt = torch.tensor([t_e2e, t_sync], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t_e2e, t_sync = float(tt[0].item()), float(tt[1].item())
        bi = Hii_h.numel() * 16 + H1i_h.numel() * 16
        bo = (ldos_h.numel() + ndens_h.numel()) * 16 + 3 * nen * 8 + \
            sum(v.numel() * v.element_size() for v in extra_h.values())
        e2e = {"value": nen * world * args.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": bi,
               "d2h_bytes_per_step": bo, "ms_per_step": 1e3 * t_e2e / args.steps,
               "api": "rgf_solve_energies (C ABI) with pinned host arrays, rgf_opts.pipelined = 1, "
                      "rgf_ctx_synchronize at the end of the timed steps",
               "one_call_per_step": {"value": nen * world * args.steps / t_sync,
                                     "ms_per_step": 1e3 * t_sync / args.steps,
                                     "api": "synchronous rgf_solve_energies per step, outputs written "
                                            "through their device mapping"},
               "pageable": None if t_pg is None else {
                   "value": nen * world * args.steps / t_pg, "ms_per_step": 1e3 * t_pg / args.steps,
                   "api": "pipelined rgf_solve_energies on pageable NumPy arrays (as Fortran passes them), "
                          "copied through the library's pinned bounce slots"}}

    # the other precision form on the same workload and timing, for the ratio
    # the metric names (mixed vs plain FP64)
    other = None
    if not args.no_other and nb == 128 and not args.full_outputs:
        oprec = rgf.RGF_PREC_FP64 if mixed else rgf.RGF_PREC_MIXED
        ctx2 = rgf.Context(rgf.Options(device=local, eta_dev=ETA, eta_lead=ETA, precision=oprec,
                                       consistent=args.consistent))
        with torch.cuda.stream(stream):
            for _ in range(max(1, args.warmup)):
                ctx2.solve_energies(Hii, H1i, E, MU, temp, ldos=ldos, ndens=ndens, tr=tr, tre=tre, T=T,
                                    stream=sh)
            torch.cuda.synchronize(dev)
            oms, okms = [], []
            for _ in range(args.steps):
                flush.fill_(1.0)
                s = torch.cuda.Event(enable_timing=True)
                e = torch.cuda.Event(enable_timing=True)
                s.record(stream)
                ctx2.solve_energies(Hii, H1i, E, MU, temp, ldos=ldos, ndens=ndens, tr=tr, tre=tre, T=T,
                                    stream=sh)
                e.record(stream)
                e.synchronize()
                oms.append(s.elapsed_time(e))
                okms.append(ctx2.stats()["last_kernel_ms"])
            ost = ctx2.stats()
        ctx2.close()
        t_o = sum(oms) / 1e3
        if world > 1:
            tt = torch.tensor([t_o], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t_o = float(tt.item())
        other = {"value": nen * world * args.steps / t_o, "unit": UNIT, "ms_per_step": 1e3 * t_o / args.steps,
                 "kernel_ms": float(np.mean(okms)),
                 "form": ("plain FP64 (RGF_PREC_FP64)" if mixed else
                          "mixed (RGF_PREC_MIXED): split-integer products on the int8 tensor cores") +
                         ", same workload, timing and outputs"}
        if not mixed:
            other["int8_tops"] = ost["last_int8_ops"] / (ost["last_kernel_ms"] * 1e-3) / 1e12
            other["fp64_tflops"] = ost["last_flops"] / (ost["last_kernel_ms"] * 1e-3) / 1e12

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, d, E, temp, host_threads(args))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int8 tensor products + f64" if mixed else "f64",
                "data": "synthetic", "config": config(args, world), "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk}
        if other is not None:
            line["mixed" if not mixed else "plain_fp64"] = other
            line["mixed_vs_plain"] = (value / other["value"]) if mixed else (other["value"] / value)
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_single(args):
    """One device-resident batched solve of the workload (profiler captures)."""
    import torch
    from liteqt_b200 import rgf
    d, E, temp = workload(args)
    dev = torch.device("cuda", 0)
    Hii = torch.from_numpy(d.Hii).to(dev)
    H1i = torch.from_numpy(d.H1i).to(dev)
    shape = (args.nen, args.nx, args.nb, args.nb)
    ldos = torch.empty(shape, dtype=torch.complex128, device=dev)
    ndens = torch.empty_like(ldos)
    T = torch.empty(args.nen, dtype=torch.float64, device=dev)
    mixed = args.precision == "mixed"
    opts = rgf.Options(eta_dev=ETA, eta_lead=ETA, precision=rgf.RGF_PREC_MIXED if mixed else rgf.RGF_PREC_FP64)
    with rgf.Context(opts) as ctx:
        ctx.solve_energies(Hii, H1i, E, MU, temp, ldos=ldos, ndens=ndens, T=T)
        st = ctx.stats()
    print(f"single {args.precision} solve nb={args.nb} nx={args.nx} nen={args.nen}: kernel "
          f"{st['last_kernel_ms']:.1f} ms, {st['last_flops'] / st['last_kernel_ms'] / 1e9:.2f} TFLOP/s executed "
          f"in FP64, {st['last_int8_ops'] / st['last_kernel_ms'] / 1e9:.1f} int8 TOP/s")


def run_adjoint(args):
    """Adjoint workload: nb = 64, Nx = 200, on-site potential V_l ~ U[-0.2, 0.2] eV
    per block (seed 2), --nen energies (default 1024) on [-3, 3] eV, eta = 1e-5.
    One step = one rgf_adjoint_energies call (T, dT/dV_l, dT/ds and the
    current's derivatives); it is timed next to forward solves of the same
    energies (T only, and G^R_ll + G^<_ll + T) with CUDA events on the
    library's stream, inputs and outputs resident in HBM."""
    import torch
    from liteqt_b200 import rgf
    from liteqt_b200 import synthetic as S
    nb, nx, nen = 64, 200, (args.nen if args.nen != 296 else 1024)
    pot = np.random.default_rng(2).uniform(-0.2, 0.2, nx)
    d = S.make_device(nb, nx, seed=1, potential=pot)
    E = S.energy_grid(nen, -3.0, 3.0)
    temp = (S.temperature_for_kT(KT),) * 2
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    Hii = torch.from_numpy(d.Hii).to(dev)
    H1i = torch.from_numpy(d.H1i).to(dev)
    T = torch.empty(nen, dtype=torch.float64, device=dev)
    dTdV = torch.empty((nen, nx), dtype=torch.float64, device=dev)
    dTds = torch.empty(nen, dtype=torch.float64, device=dev)
    ldos = torch.empty((nen, nx, nb, nb), dtype=torch.complex128, device=dev)
    ndens = torch.empty_like(ldos)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    ctx = rgf.Context(rgf.Options(eta_dev=ETA, eta_lead=ETA))
    runs = {
        "adjoint": lambda: ctx.adjoint_energies(Hii, H1i, E, MU, temp, T=T, dTdV=dTdV, dTds=dTds,
                                                spindeg=2.0, stream=sh),
        "forward_T": lambda: ctx.solve_energies(Hii, H1i, E, MU, temp, T=T, stream=sh),
        "forward_GR_GL_T": lambda: ctx.solve_energies(Hii, H1i, E, MU, temp, ldos=ldos, ndens=ndens,
                                                      T=T, stream=sh),
    }
    ms = {}
    clocks = ClockSampler(0)
    with torch.cuda.stream(stream):
        for name, fn in runs.items():
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize(dev)
            if name == "adjoint":
                clocks.start()
            t = []
            for _ in range(args.steps):
                flush.fill_(1.0)
                s = torch.cuda.Event(enable_timing=True)
                e = torch.cuda.Event(enable_timing=True)
                s.record(stream)
                fn()
                e.record(stream)
                e.synchronize()
                t.append(s.elapsed_time(e))
            if name == "adjoint":
                clk = clocks.stop()
            ms[name] = float(np.mean(t))
    launches = ctx.stats()["launches"]
    ctx.close()
    line = {"metric": "adjoint RGF energy-pts/s (dT/dV_l, dT/ds, dI/dV_l)", "value": nen / (ms["adjoint"] * 1e-3),
            "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms["adjoint"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"adjoint_nb{nb}_nx{nx}", "nb": nb, "nx": nx, "energies": nen,
                       "eta_eV": ETA, "potential": "U[-0.2,0.2] eV per block, seed 2",
                       "l2": "flushed between timed steps (256 MiB write)"},
            "forward_ms": {"T_only": ms["forward_T"], "GR_GL_T": ms["forward_GR_GL_T"]},
            "cost_vs_forward": {"T_only": ms["adjoint"] / ms["forward_T"],
                                "GR_GL_T": ms["adjoint"] / ms["forward_GR_GL_T"]},
            "gpu_launches_total": int(launches), "clocks": clk}
    print(json.dumps(line), flush=True)


def run_w(args):
    """GW screened-interaction workload: nb = 64, Nx = 40, bare Coulomb V
    (1/(r + 0.3 nm) on a seeded orbital grid, seed 99), seeded physical
    polarizations (P^R complex symmetric, P^< / P^> anti-Hermitian); one step
    = rgf_w_solve_energies over --nen polarization sets (default 2048: the
    energies of one q-point), W^<, W^>, W^R out, device-resident.  Roofline
    numerator: the reference routine's own products for NBC = 0 (46 Nx - 20
    nb^3 products + Nx inversions per solve, including its LL / LG blocks and
    XR recursion, which the GPU skips because nothing returned uses them)."""
    import torch
    from liteqt_b200 import rgf
    from liteqt_b200 import synthetic as S
    nb, nx, nen = 64, 40, (args.nen if args.nen != 296 else 2048)
    Vii, V1i = S.make_coulomb(nb, nx, seed=99)
    # a pool of 64 distinct polarization sets, tiled to nen (the solve cost does
    # not depend on the values)
    pool = S.make_polarization(nb, nx, 64, seed=7)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    reps = (nen + 63) // 64
    P = [torch.from_numpy(np.concatenate([x] * reps)[:nen]).to(dev) for x in pool]
    Vd, V1d = torch.from_numpy(Vii).to(dev), torch.from_numpy(V1i).to(dev)
    W = [torch.empty_like(P[0]) for _ in range(3)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    ctx = rgf.Context(rgf.Options())
    peak = zgemm_peak_tflops(torch, dev)

    def step():
        ctx.w_solve_energies(Vd, V1d, P[0], P[1], P[2], WL=W[0], WG=W[1], WR=W[2], stream=stream.cuda_stream)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(0)
        clocks.start()
        ms, kms = [], []
        for _ in range(args.steps):
            flush.fill_(1.0)
            s0 = torch.cuda.Event(enable_timing=True)
            e0 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            step()
            e0.record(stream)
            e0.synchronize()
            ms.append(s0.elapsed_time(e0))
            kms.append(ctx.stats()["last_kernel_ms"])
        clk = clocks.stop()
    st = ctx.stats()
    ctx.close()
    alg = nen * 8.0 * nb ** 3 * ((46 * nx - 20) + nx)
    kern_s = float(np.mean(kms)) * 1e-3
    line = {"metric": "RGF_W solves/s (W^R, W^<, W^> diagonal blocks)", "value": nen / (np.mean(ms) * 1e-3),
            "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"rgf_w_nb{nb}_nx{nx}", "nb": nb, "nx": nx, "solves_per_step": nen,
                       "V": "Coulomb 1.44/(r+0.3 nm) eV, seed 99", "P": "seeded physical polarizations",
                       "l2": "flushed between timed steps (256 MiB write)"},
            "roofline": {"bound": "tensor", "achieved": alg / kern_s / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": alg / kern_s / 1e12 / peak, "traffic": None,
                         "executed_tflops": st["last_flops"] / kern_s / 1e12,
                         "peak_source": "cuBLAS ZGEMM 4096^3 measured live on this GPU"},
            "gpu_launches_total": int(st["launches"]), "clocks": clk}
    print(json.dumps(line), flush=True)


def _gw_terms(nm, nx, nen, nk, ndiag):
    """Summands of the reference's direct sums: (P terms, Sigma terms)."""
    band = sum(min(nm, i + ndiag) - max(1, i - ndiag) + 1 for i in range(1, nm + 1))
    nopmax = nen // 2 - 10
    p_terms = sum(nen - abs(nop) for nop in range(-nopmax, nopmax + 1)) * nk * nk * nx * band
    s_count = sum(1 for ie in range(1, nen + 1) for nop in range(-nopmax, nopmax + 1)
                  if ie > max(nop, 1) and ie < nen + nop)
    return p_terms, s_count * nk * nk * nx * band


def run_gw(args):
    """GW-loop convolutions (green_rgf.f90:2944-3092) on device-resident
    arrays: 2x2 k-grid, nen = 512, nx = 10, nm = 16, ndiag = 3, seeded complex
    inputs.  One step = rgf_gw_polarization + rgf_gw_self_energy.  Roofline:
    the FP64 pipe (4 complex multiply-adds = 32 flops per P summand, 5 = 40
    per Sigma summand; summand counts of the reference's loops)."""
    import torch
    from liteqt_b200 import rgf
    nky, nkz, nen, nx, nm, ndiag = 2, 2, 512, 10, 16, 3
    nk = nky * nkz
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = torch.Generator(device="cpu").manual_seed(3)
    shape = (nk, nen, nx, nm, nm)

    def rnd():
        return torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                             torch.randn(shape, generator=g, dtype=torch.float64)).to(dev)
    G = [rnd() for _ in range(3)]
    W = [rnd() for _ in range(3)]
    S = [rnd() for _ in range(3)]
    P = [torch.empty_like(G[0]) for _ in range(3)]
    peak = zgemm_peak_tflops(torch, dev)
    stream = torch.cuda.Stream(device=dev)
    ctx = rgf.Context(rgf.Options())
    tp, ts = [], []
    with torch.cuda.stream(stream):
        for it in range(args.warmup + args.steps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            ctx.gw_polarization(*G, PL=P[0], PG=P[1], PR=P[2], nky=nky, nkz=nkz, ndiag=ndiag, dE=0.01,
                                spindeg=2.0, stream=stream.cuda_stream)
            e[1].record(stream)
            ctx.gw_self_energy(*G, *W, SL=S[0], SG=S[1], SR=S[2], nky=nky, nkz=nkz, ndiag=ndiag, dE=0.01,
                               alpha_mix=0.5, stream=stream.cuda_stream)
            e[2].record(stream)
            e[2].synchronize()
            if it >= args.warmup:
                tp.append(e[0].elapsed_time(e[1]))
                ts.append(e[1].elapsed_time(e[2]))
    ctx.close()
    p_terms, s_terms = _gw_terms(nm, nx, nen, nk, ndiag)
    fp, fs = 32.0 * p_terms, 40.0 * s_terms
    mp, ms_ = float(np.mean(tp)), float(np.mean(ts))
    line = {"metric": "GW convolutions: polarization + self-energy steps/s", "value": 1e3 / (mp + ms_),
            "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": mp + ms_, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "gw_conv_nk4_nen512_nx10_nm16_nd3", "nky": nky, "nkz": nkz, "nen": nen,
                       "nx": nx, "nm": nm, "ndiag": ndiag, "array_bytes": 16 * nk * nen * nx * nm * nm},
            "polarization": {"ms": mp, "tflops": fp / (mp * 1e-3) / 1e12, "summands": p_terms},
            "self_energy": {"ms": ms_, "tflops": fs / (ms_ * 1e-3) / 1e12, "summands": s_terms},
            "roofline": {"bound": "fp64", "achieved": (fp + fs) / ((mp + ms_) * 1e-3) / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": (fp + fs) / ((mp + ms_) * 1e-3) / 1e12 / peak,
                         "traffic": None,
                         "peak_source": "cuBLAS ZGEMM 4096^3 measured live (DMMA and DFMA peaks are "
                                        "equal on B200: 37.1 vs 36.5 TFLOP/s in a probe)"}}
    print(json.dumps(line), flush=True)


def run_blocks(args):
    """The solver's building blocks alone, one CTA per SM, 10 blocks per SM
    (1480 seeded 128 x 128 complex blocks): the FP64 DMMA product, the
    split-integer int8 product, the FP64 blocked Gauss-Jordan inverse and the
    refined FP32 inverse, through rgf_block_product / rgf_block_inverse.
    Reported per operation: device time per block per SM in SM cycles (at
    the sampled clock) and the rate in complex-GEMM-equivalent TFLOP/s
    (8 nb^3 per block)."""
    import torch
    from liteqt_b200 import rgf
    nb, count = 128, 1480
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = torch.Generator(device=dev).manual_seed(13)

    def rnd():
        return torch.complex(torch.randn((count, nb, nb), generator=g, device=dev, dtype=torch.float64),
                             torch.randn((count, nb, nb), generator=g, device=dev, dtype=torch.float64))
    A, B = rnd(), rnd()
    C = torch.empty_like(A)
    ctx = rgf.Context(rgf.Options())
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    ops = {
        "product_fp64": lambda: ctx.block_product(A, B, C, precision=rgf.RGF_PREC_FP64),
        "product_int8_split": lambda: ctx.block_product(A, B, C, precision=rgf.RGF_PREC_MIXED),
        "inverse_fp64": lambda: ctx.block_inverse(A, C, precision=rgf.RGF_PREC_FP64),
        "inverse_fp32_refined": lambda: ctx.block_inverse(A, C, precision=rgf.RGF_PREC_MIXED),
    }
    clocks = ClockSampler(0)
    clocks.start()
    out = {}
    for name, fn in ops.items():
        ms = []
        for it in range(args.warmup + args.steps):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            if it >= args.warmup:
                ms.append(s.elapsed_time(e))
        out[name] = float(np.mean(ms))
    clk = clocks.stop()
    ctx.close()
    mhz = clk.get("sm_mhz") or 1965.0
    per_sm = count / sms
    res = {k: {"ms": v, "kcycles_per_block_per_sm": v * 1e-3 * mhz * 1e6 / per_sm / 1e3,
               "tflops_equiv": 8.0 * nb ** 3 * count / (v * 1e-3) / 1e12} for k, v in out.items()}
    peak = zgemm_peak_tflops(torch, dev)
    line = {"metric": "block operations per second (nb 128, one CTA per SM)",
            "value": count / (out["product_fp64"] * 1e-3), "unit": "FP64 products/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["product_fp64"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 / int8", "data": "synthetic",
            "config": {"workload": "block_ops_nb128_x1480", "nb": nb, "blocks": count, "blocks_per_sm": per_sm,
                       "l2": "operands 3 x 388 MB, larger than L2"},
            "ops": res,
            "roofline": {"bound": "tensor", "achieved": res["product_fp64"]["tflops_equiv"], "peak": peak,
                         "unit": "TFLOP/s", "frac": res["product_fp64"]["tflops_equiv"] / peak, "traffic": None,
                         "peak_source": "cuBLAS ZGEMM 4096^3 measured live"},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def run_gw_fft(args):
    """FFT form of the GW convolutions at the GW workload's sizes: 4 x 4
    k-grid, nen = 4096, nx = 40, nm = 64, ndiag = 3, on one rank's slice of
    128 (i,j) elements (columns 30-31 of the 64 x 64 block: 14 banded
    elements, 560 (i,j, block) lines) in the *_by_blocks layout.  One step =
    rgf_gw_polarization_fft + rgf_gw_self_energy_fft on seeded inputs.
    Reported: lines per second and the time of a whole iteration's
    convolutions (all 436 banded elements x 40 blocks = 17 440 lines) at
    that rate.  Roofline: HBM, algorithmic bytes = the banded lines' inputs
    read once (5 + 6 series) plus every output element written once (the
    zeros outside the band included)."""
    import torch
    from liteqt_b200 import rgf
    nky, nkz, nen, nx, nm, ndiag = 4, 4, 4096, 40, 64, 3
    nk = nky * nkz
    nij, first_ij = 128, 29 * nm + 1
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = torch.Generator(device=dev).manual_seed(11)
    shape = (nij, nx, nk, nen)

    def rnd():
        return torch.complex(torch.randn(shape, generator=g, device=dev, dtype=torch.float64),
                             torch.randn(shape, generator=g, device=dev, dtype=torch.float64))
    GL, GG, GR, GLt, GGt, WL, WG, WR = (rnd() for _ in range(8))
    out = [torch.empty_like(GL) for _ in range(3)]
    band = sum(1 for i in range(nij) if max((i + first_ij - 1) % nm + 1 - ndiag, 1) <= (i + first_ij - 1) // nm + 1
               <= min(nm, (i + first_ij - 1) % nm + 1 + ndiag))
    lines = band * nx
    full_lines = (nm * (2 * ndiag + 1) - ndiag * (ndiag + 1)) * nx
    stream = torch.cuda.Stream(device=dev)
    ctx = rgf.Context(rgf.Options())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    tp, ts = [], []
    with torch.cuda.stream(stream):
        for it in range(args.warmup + args.steps):
            flush.fill_(1.0)
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            ctx.gw_polarization_fft(GL, GG, GR, GLt, GGt, PL=out[0], PG=out[1], PR=out[2], nky=nky, nkz=nkz, nm=nm,
                                    ndiag=ndiag, first_ij=first_ij, dEn=8.0 / (nen - 1), spindeg=2.0,
                                    stream=stream.cuda_stream)
            e[1].record(stream)
            ctx.gw_self_energy_fft(GL, GG, GR, WL, WG, WR, SL=out[0], SG=out[1], SR=out[2], nky=nky, nkz=nkz,
                                   nm=nm, ndiag=ndiag, first_ij=first_ij, dEn=8.0 / (nen - 1),
                                   stream=stream.cuda_stream)
            e[2].record(stream)
            e[2].synchronize()
            if it >= args.warmup:
                tp.append(e[0].elapsed_time(e[1]))
                ts.append(e[1].elapsed_time(e[2]))
    ctx.close()
    mp, ms_ = float(np.mean(tp)), float(np.mean(ts))
    series = nk * nen * 16
    alg = lines * series * (5 + 6) + 2 * 3 * nij * nx * series
    peak = None
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        peak = float(json.load(open(path)).get("hbm_gbs"))
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    gbs = alg / ((mp + ms_) * 1e-3) / 1e9
    line = {"metric": "GW FFT convolutions: (i,j,block) lines per second (P + Sigma)",
            "value": lines / ((mp + ms_) * 1e-3), "unit": "lines/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mp + ms_, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c16", "data": "synthetic",
            "config": {"workload": "gw_fft_nk16_nen4096_nx40_nm64_nd3", "nky": nky, "nkz": nkz, "nen": nen,
                       "nx": nx, "nm": nm, "ndiag": ndiag, "nij_slice": nij, "first_ij": first_ij,
                       "banded_in_slice": band, "lines_per_step": lines, "fft_length": 8192,
                       "l2": "flushed before each step (256 MiB write)"},
            "polarization_ms": mp, "self_energy_ms": ms_,
            "full_iteration": {"lines": full_lines, "s": full_lines / (lines / ((mp + ms_) * 1e-3)),
                               "note": "every banded (i,j) element of the 64 x 64 block, 40 blocks"},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "traffic": None, "peak_source": peak_src, "algorithmic_bytes_per_step": alg}}
    print(json.dumps(line), flush=True)


def run_dropin(args):
    """Per-energy drop-in throughput: host threads (all of them, as the
    reference's `!$omp do ie` loop over green_RGF_RS at green_rgf.f90:
    2916-2925) each call rgf_green_rgf_rs for two energies of the
    rgf_nb128_nx100 workload with the reference's output set (ndens, pdens,
    ldos, cur, GRi1, tr, tre) in pageable host memory; no context is passed,
    so concurrent calls are coalesced into shared batches.  Timed by wall
    clock from the first call to the last return, next to
    rgf_solve_energies on the same energies and outputs."""
    import threading
    import torch
    from liteqt_b200 import rgf
    rgf.load()
    d, E_all, temp = workload(args)
    nthr = host_threads(args)
    per = max(1, args.per_thread)
    nen = nthr * per
    E = np.ascontiguousarray(E_all[np.linspace(0, len(E_all) - 1, nen).astype(int)])
    nm, nx = args.nb, args.nx
    mk = lambda: np.zeros((nx, nm, nm), complex)
    outs = [dict(nd=mk(), pd=mk(), ld=mk(), gr=mk(), cur=np.zeros((nx, nm, nm)), tr=np.zeros(1), tre=np.zeros(1))
            for _ in range(nthr)]
    # the drop-in takes no options: both arms run the reference's own
    # settings (device eta 0, lead eta 1e-3)
    start = threading.Barrier(nthr + 1)

    def work(k):
        o = outs[k]
        start.wait()
        for i in range(per):
            e = float(E[k * per + i])
            rgf.green_RGF_RS(temp, nm, nx, e, MU, d.Hii, d.H1i, None, None, None, o["nd"], o["pd"], o["ld"],
                             o["tr"], o["tre"], o["cur"], GRi1=o["gr"])
    # warm-up: one call per thread (contexts, workspace, staging buffers)
    warm = [threading.Thread(target=lambda k=k: rgf.green_RGF_RS(
        temp, nm, nx, float(E[k]), MU, d.Hii, d.H1i, None, None, None, outs[k]["nd"], outs[k]["pd"],
        outs[k]["ld"], outs[k]["tr"], outs[k]["tre"], outs[k]["cur"], GRi1=outs[k]["gr"])) for k in range(nthr)]
    for t in warm:
        t.start()
    for t in warm:
        t.join()
    threads = [threading.Thread(target=work, args=(k,)) for k in range(nthr)]
    for t in threads:
        t.start()
    start.wait()
    t0 = time.perf_counter()
    for t in threads:
        t.join()
    t_drop = time.perf_counter() - t0
    outs.clear()   # the drop-in arrays go before the batched arm's are made (host memory)
    # the batched entry point on the same energies, options and output set
    shape = (nen, nx, nm, nm)
    B = dict(ldos=np.zeros(shape, complex), ndens=np.zeros(shape, complex), pdens=np.zeros(shape, complex),
             GRi1=np.zeros(shape, complex), cur=np.zeros(shape), tr=np.zeros(nen), tre=np.zeros(nen))
    with rgf.Context(rgf.Options(want_T=False)) as ctx:
        ctx.solve_energies(d.Hii, d.H1i, E, MU, temp, **B)
        t1 = time.perf_counter()
        ctx.solve_energies(d.Hii, d.H1i, E, MU, temp, **B)
        t_batch = time.perf_counter() - t1
    line = {"metric": "per-energy drop-in energy-pts/s (green_RGF_RS from every host thread)",
            "value": nen / t_drop, "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "config": {"workload": f"rgf_nb{nm}_nx{nx}", "host_threads": nthr, "energies": nen,
                       "energies_per_thread": per,
                       "options": "the reference's (device eta 0, lead eta 1e-3)",
                       "outputs": ["ndens", "pdens", "ldos", "cur", "GRi1", "tr", "tre"],
                       "memory": "pageable host arrays, as Fortran passes them"},
            "batched_same_energies": {"value": nen / t_batch, "unit": UNIT,
                                      "api": "rgf_solve_energies, host arrays"},
            "dropin_vs_batched": t_batch / t_drop}
    print(json.dumps(line), flush=True)


def _timed_steps(torch, fn, steps, warmup, flush, stream):
    """Device time (ms) of each of `steps` calls of fn after `warmup` calls,
    CUDA events on `stream`, L2 flushed before each timed call."""
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            flush.fill_(1.0)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            ms.append(s.elapsed_time(e))
    return ms


def run_uneven(args):
    """Uneven batch in one persistent launch: 64 seeded devices with Nx
    uniform in {20..200} and nb uniform in {32, 64, 128} (the H construction
    of the main workload), --nen energies per device per step on the uniform
    grid of [-3, 3] eV (the configuration's 2048 per device are 32 such
    steps), eta = 1e-5, outputs G^R_ll, G^<_ll, T, tr, tre in HBM.  The
    context is autotuned for the three block sizes first; one step replays
    a CUDA-graph plan of the whole launch."""
    import torch
    from liteqt_b200 import rgf, synthetic as S
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(2)
    ndev = 64
    nxs = rng.integers(20, 201, ndev)
    nbs = rng.choice([32, 64, 128], ndev)
    nen = args.nen if args.nen != 296 else 32
    temp = (S.temperature_for_kT(KT),) * 2
    ctx = rgf.Context(rgf.Options(eta_dev=ETA, eta_lead=ETA))
    keep, cdevs, ctasks, tuned = [], [], [], {}
    for i in range(ndev):
        d = S.make_device(int(nbs[i]), int(nxs[i]), seed=1000 + i)
        if d.nm not in tuned:
            tuned[d.nm] = ctx.autotune(d.Hii, d.H1i, MU, temp)
        Hii, H1i = torch.from_numpy(d.Hii).to(dev), torch.from_numpy(d.H1i).to(dev)
        cd = rgf.c_device()
        cd.nm, cd.nx = d.nm, d.nx
        cd.Hii, cd.H1i = Hii.data_ptr(), H1i.data_ptr()
        cd.mu[0], cd.mu[1] = MU
        cd.temp[0], cd.temp[1] = temp
        cdevs.append(cd)
        o = {k: torch.empty((nen, d.nx, d.nm, d.nm), dtype=torch.complex128, device=dev)
             for k in ("ldos", "ndens")}
        for k in ("tr", "tre", "T"):
            o[k] = torch.empty(nen, dtype=torch.float64, device=dev)
        keep += [Hii, H1i, o]
        E = S.energy_grid(nen, -3.0, 3.0)
        for ie in range(nen):
            t = rgf.c_task()
            t.device, t.E = i, float(E[ie])
            t.ldos, t.ndens = o["ldos"][ie].data_ptr(), o["ndens"][ie].data_ptr()
            t.tr, t.tre, t.T = o["tr"][ie:].data_ptr(), o["tre"][ie:].data_ptr(), o["T"][ie:].data_ptr()
            ctasks.append(t)
    plan = ctx.plan(cdevs, ctasks)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    ms = _timed_steps(torch, lambda: plan.execute(stream=stream.cuda_stream), args.steps, max(3, args.warmup),
                      flush, stream)
    clk = clocks.stop()
    info = np.zeros(len(ctasks), rgf.INFO_DTYPE)
    plan.execute(info=info, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    plan.close()
    ntask = len(ctasks)
    nb_t = np.repeat(nbs, nen).astype(np.float64)
    nx_t = np.repeat(nxs, nen).astype(np.float64)
    nsum = info["sancho_iters_left"].astype(np.float64) + info["sancho_iters_right"]
    alg = float(np.sum(8.0 * nb_t ** 3 * ((28 * nx_t - 18 + 6 * nsum) + (nx_t + 4 + nsum))))
    peak = zgemm_peak_tflops(torch, dev)
    ctx.close()
    m = float(np.mean(ms))
    line = {"metric": "uneven batched RGF energy-pts/s (one persistent launch, graph replay)",
            "value": ntask / (m * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": m, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "rgf_uneven_64dev", "devices": ndev, "nx": [int(v) for v in nxs],
                       "nb": [int(v) for v in nbs], "energies_per_device_per_step": nen, "eta_eV": ETA,
                       "outputs": ["G^R_ll", "G^<_ll", "T", "tr", "tre"], "tasks_per_step": ntask,
                       "full_configuration_s": 2048 * ndev / (ntask / (m * 1e-3)),
                       "autotuned": {str(k): [v["variant"], v["ctas_per_sm"]] for k, v in tuned.items()},
                       "l2": "flushed between timed steps (256 MiB write)", "seed": 2},
            "status_nonzero": int(np.count_nonzero(info["status"])),
            "roofline": {"bound": "tensor", "achieved": alg / (m * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": alg / (m * 1e-3) / 1e12 / peak, "traffic": None,
                         "peak_source": "cuBLAS ZGEMM 4096^3 measured live",
                         "algorithmic_flops_per_launch": alg},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def run_band_edge(args):
    """Band-edge workload: nb = 256, Nx = 64, eta = 1e-6 in device and
    leads, energies from a 4096-point grid of [-3, 3] eV with 10 % of them
    within 1e-3 eV of a lead subband edge; one step solves --nen of them (a
    seeded sample that keeps the 10 %), outputs G^R_ll, G^<_ll, T, tr, tre.
    Plain FP64 (the split-integer form is built for nb = 128)."""
    import torch
    from liteqt_b200 import rgf, synthetic as S
    nb, nx, eta = 256, 64, 1e-6
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    d = S.make_device(nb, nx, seed=3)
    edges = S.lead_band_edges(d.Hii, d.H1i, 0, 128)
    grid = S.band_edge_energy_grid(4096, edges, -3.0, 3.0, 0.1, 1e-3, seed=5)
    near = np.min(np.abs(grid[:, None] - edges[None, :]), axis=1) <= 1e-3
    nen = args.nen
    pick = np.sort(np.random.default_rng(7).choice(len(grid), nen, replace=False))
    E = np.ascontiguousarray(grid[pick])
    temp = (S.temperature_for_kT(KT),) * 2
    ctx = rgf.Context(rgf.Options(eta_dev=eta, eta_lead=eta))
    Hii, H1i = torch.from_numpy(d.Hii).to(dev), torch.from_numpy(d.H1i).to(dev)
    o = {k: torch.empty((nen, nx, nb, nb), dtype=torch.complex128, device=dev) for k in ("ldos", "ndens")}
    for k in ("tr", "tre", "T"):
        o[k] = torch.empty(nen, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    ms = _timed_steps(torch, lambda: ctx.solve_energies(Hii, H1i, E, MU, temp, stream=stream.cuda_stream, **o),
                      args.steps, max(3, args.warmup), flush, stream)
    clk = clocks.stop()
    info = np.zeros(nen, rgf.INFO_DTYPE)
    ctx.solve_energies(Hii, H1i, E, MU, temp, info=info, stream=stream.cuda_stream, **o)
    torch.cuda.synchronize()
    peak = zgemm_peak_tflops(torch, dev)
    ctx.close()
    nsum = info["sancho_iters_left"].astype(np.float64) + info["sancho_iters_right"]
    alg = float(np.sum(8.0 * nb ** 3 * ((28 * nx - 18 + 6 * nsum) + (nx + 4 + nsum))))
    m = float(np.mean(ms))
    line = {"metric": "band-edge RGF energy-pts/s (nb 256, eta 1e-6)", "value": nen / (m * 1e-3), "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": m,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "rgf_band_edge_nb256_nx64", "nb": nb, "nx": nx, "eta_eV": eta,
                       "grid_points": len(grid), "near_edge_in_grid": int(near.sum()),
                       "energies_per_step": nen, "near_edge_in_step": int(near[pick].sum()),
                       "outputs": ["G^R_ll", "G^<_ll", "T", "tr", "tre"],
                       "full_grid_s": len(grid) / (nen / (m * 1e-3)),
                       "l2": "flushed between timed steps (256 MiB write)", "seed": 3},
            "sancho_iters": {"mean": float(np.mean(nsum) / 2), "max": int(max(info["sancho_iters_left"].max(),
                                                                             info["sancho_iters_right"].max()))},
            "status_nonzero": int(np.count_nonzero(info["status"])),
            "roofline": {"bound": "tensor", "achieved": alg / (m * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": alg / (m * 1e-3) / 1e12 / peak, "traffic": None,
                         "peak_source": "cuBLAS ZGEMM 4096^3 measured live",
                         "algorithmic_flops_per_launch": alg},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def run_aux(args):
    """The HBM-bound routines around the solve on arrays of the benchmark's
    output size (G (nen, nx, nb, nb) complex(8), seeded): the GW loop's
    energy -> (i,j) transpose (rgf_permute_c16, energies_to_ijs_2's second
    RESHAPE as an 8-rank run has it), calc_n_electron, calc_block_current
    (4 sub-blocks of nb/4) and the writers' GPU sums (write_spectrum's
    diagonal traces, write_dos_summed_over_k).  Each routine is timed with
    CUDA events through its public entry point (host outputs included), the
    L2 flushed before each call.  Algorithmic bytes: the transpose reads and
    writes the array once; the integrals and traces read the elements they
    sum (16 B each; the diagonal gathers touch one 32-byte sector per
    element)."""
    import torch
    from liteqt_b200 import rgf, writers as Wr
    nen, nx, nm = args.nen, args.nx, args.nb
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = torch.Generator(device=dev).manual_seed(5)
    shape = (1, nen, nx, nm, nm)

    def rnd():
        return torch.complex(torch.randn(shape, generator=g, device=dev, dtype=torch.float64),
                             torch.randn(shape, generator=g, device=dev, dtype=torch.float64))
    Gl, Gg = rnd(), rnd()
    H = torch.complex(torch.randn((nx, nm, nm), generator=g, device=dev, dtype=torch.float64),
                      torch.randn((nx, nm, nm), generator=g, device=dev, dtype=torch.float64))
    dst = torch.empty_like(Gl)
    E = np.linspace(-3.0, 3.0, nen)
    midgap = np.zeros(nx)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ranks = 8
    nij = nm * nm // ranks
    src_shape, order = (nij, nx, nen, 1, ranks), (5, 4, 1, 3, 2)
    ns = 4
    sub = nm // ns
    tmp = tempfile.mkdtemp()
    ctx = rgf.Context(rgf.Options())
    arr = 16 * Gl.numel()
    calls = {
        "permute_c16": (lambda: ctx.permute(Gl, dst, src_shape, order), 2.0 * arr),
        "calc_n_electron": (lambda: ctx.calc_n_electron(Gl, Gg, E, midgap), 16.0 * nen * nx * nm),
        "calc_block_current": (lambda: ctx.calc_block_current(H, Gl[0], E, 2.0, sub, ns),
                               2 * 16.0 * nen * nx * (ns - 1) * sub * sub),
        "write_spectrum": (lambda: Wr.write_spectrum(ctx, os.path.join(tmp, "ldos"), 1, Gl, E, nx, sub, ns,
                                                     1.0, (1.0, 1.0)), 16.0 * nen * nx * nm),
        "write_dos": (lambda: Wr.write_dos_summed_over_k(ctx, os.path.join(tmp, "dos"), 1, Gl, E, 1, nx, sub,
                                                          ns, 1.0), 16.0 * nen * nx * nm),
    }
    peak = None
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        peak = float(json.load(open(path)).get("hbm_gbs"))
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    out = {}
    for name, (fn, nbytes) in calls.items():
        ms = []
        for it in range(args.warmup + args.steps):
            flush.fill_(1.0)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            e.synchronize()
            if it >= args.warmup:
                ms.append(s.elapsed_time(e))
        m = float(np.mean(ms))
        out[name] = {"ms": m, "alg_bytes": nbytes, "GB/s": nbytes / (m * 1e-3) / 1e9,
                     "frac": nbytes / (m * 1e-3) / 1e9 / peak}
    ctx.close()
    for f in os.listdir(tmp):
        os.unlink(os.path.join(tmp, f))
    os.rmdir(tmp)
    top = out["permute_c16"]
    line = {"metric": "redistribution transpose GB/s (energies_to_ijs_2)", "value": top["GB/s"], "unit": "GB/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": top["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c16", "data": "synthetic",
            "config": {"workload": f"aux_nb{nm}_nx{nx}_nen{nen}", "array_bytes": arr, "ranks_in_layout": ranks,
                       "sub_blocks": ns, "l2": "flushed before each call (256 MiB write)"},
            "routines": out,
            "roofline": {"bound": "hbm", "achieved": top["GB/s"], "peak": peak, "unit": "GB/s",
                         "frac": top["frac"], "traffic": None, "peak_source": peak_src}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.aux:
        run_aux(args)
    elif args.uneven:
        run_uneven(args)
    elif args.band_edge:
        run_band_edge(args)
    elif args.gw_fft:
        run_gw_fft(args)
    elif args.blocks:
        run_blocks(args)
    elif args.dropin:
        run_dropin(args)
    elif args.gw:
        run_gw(args)
    elif args.w:
        run_w(args)
    elif args.adjoint:
        run_adjoint(args)
    elif args.single:
        run_single(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
