"""Python mirror of the liteQT RGF interface over the C ABI of librgf_b200.so.

``green_RGF_RS`` and ``RGF_G`` keep the argument lists of the Fortran
subroutines they replace (src/green_rgf.f90:3950, src/rgf_mod.f90:26);
``solve_energies`` / ``solve_batch`` are the batched entry points the drivers
use instead of their ``do ie`` loops.  Every call goes through the C ABI in
include/rgf.h; there is no Python or CPU implementation of the solver here,
and importing this module fails if the CUDA library has not been built.

Arrays follow the Fortran layout: complex128, column-major (nm, nm, nx).  A
NumPy array of shape (nx, nm, nm) (C order) has exactly that memory layout,
with the last two axes being (column, row); (nen, nx, nm, nm) stacks energies.
Host arrays are staged by the library; torch CUDA tensors are used in place.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librgf_b200.so")

RGF_OK = 0
RGF_E_ARG = -1
RGF_E_CUDA = -2
RGF_E_NOMEM = -3
RGF_E_UNSUPPORTED = -4
RGF_E_STATUS = -5

RGF_ST_SINGULAR = 1
RGF_ST_SANCHO_NC = 2
RGF_ST_BAD_TASK = 4
RGF_ST_REFINE_NC = 8

RGF_PREC_FP64 = 0
RGF_PREC_MIXED = 1

BOLTZ_RGF_RS = 8.61734e-05       # green_rgf.f90:3968
BOLTZ_RGF_G = 8.617333262e-05    # parameters.f90:38

EXPORTS = (
    "rgf_opts_default", "rgf_ctx_create", "rgf_ctx_destroy", "rgf_ctx_set_opts",
    "rgf_solve_batch", "rgf_green_rgf_rs", "rgf_rgf_g", "rgf_solve_energies",
    "rgf_terminal_current", "rgf_calc_n_electron", "rgf_last_error", "rgf_version",
    "rgf_ctx_get_stats", "rgf_adjoint_energies", "rgf_solve_energies_noalloc",
    "rgf_noalloc_last_error", "rgf_calc_block_current", "rgf_plan_create", "rgf_plan_execute",
    "rgf_plan_destroy", "rgf_autotune", "rgf_variant_name", "rgf_green_rgf_cms",
    "rgf_w_solve_batch", "rgf_w_solve_energies", "rgf_green_rgf_calc_w",
    "rgf_gw_polarization", "rgf_gw_self_energy", "rgf_gw_last_error", "rgf_permute_c16",
    "rgf_permute_last_error", "rgf_write_spectrum", "rgf_write_dos", "rgf_write_current_spectrum",
    "rgf_write_current_summed_over_k", "rgf_write_transmission_spectrum", "rgf_write_id_iteration",
    "rgf_io_last_error", "rgf_read_ham_dat", "rgf_gw_polarization_fft", "rgf_gw_self_energy_fft",
    "rgf_gw_fft_last_error", "rgf_ctx_synchronize",
)

# kernel variant ids (rgf_variant_name)
VARIANTS = ("staged32", "staged64", "staged128", "staged256", "generic1x1", "generic1x2", "generic2x2")


class RgfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rgf error {code}: {msg}")
        self.code = code


class c_opts(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32), ("device", ctypes.c_int32),
        ("eta_dev", ctypes.c_double), ("eta_lead", ctypes.c_double),
        ("boltz", ctypes.c_double), ("sancho_tol", ctypes.c_double),
        ("sancho_nmax", ctypes.c_int32), ("consistent", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("want_T", ctypes.c_int32),
        ("verbose", ctypes.c_int32), ("zero_copy", ctypes.c_int32), ("pipelined", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 5),
    ]


class c_device(ctypes.Structure):
    _fields_ = [
        ("nm", ctypes.c_int64), ("nx", ctypes.c_int64),
        ("Hii", ctypes.c_void_p), ("H1i", ctypes.c_void_p),
        ("mu", ctypes.c_double * 2), ("temp", ctypes.c_double * 2),
        ("Sii", ctypes.c_void_p),
    ]


class c_task(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32), ("reserved", ctypes.c_int32), ("E", ctypes.c_double),
        ("sigma_lesser", ctypes.c_void_p), ("sigma_r", ctypes.c_void_p),
        ("ldos", ctypes.c_void_p), ("ndens", ctypes.c_void_p), ("pdens", ctypes.c_void_p),
        ("GRi1", ctypes.c_void_p), ("GLi1", ctypes.c_void_p), ("GGi1", ctypes.c_void_p),
        ("cur", ctypes.c_void_p), ("tr", ctypes.c_void_p), ("tre", ctypes.c_void_p),
        ("T", ctypes.c_void_p),
    ]


class c_w_device(ctypes.Structure):
    _fields_ = [("nm", ctypes.c_int64), ("nx", ctypes.c_int64), ("Vii", ctypes.c_void_p),
                ("V1i", ctypes.c_void_p)]


class c_w_task(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("reserved", ctypes.c_int32), ("PL", ctypes.c_void_p),
                ("PG", ctypes.c_void_p), ("PR", ctypes.c_void_p), ("WL", ctypes.c_void_p),
                ("WG", ctypes.c_void_p), ("WR", ctypes.c_void_p), ("WRi1", ctypes.c_void_p)]


class c_ham_info(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("nvb", "spin_deg", "nb", "nx", "ny", "xmin", "xmax", "ymin", "ymax",
                                               "n_entries")] + \
               [("cell", ctypes.c_double * 9), ("Lx", ctypes.c_double), ("Ly", ctypes.c_double),
                ("Lz", ctypes.c_double), ("b1", ctypes.c_double * 3), ("b2", ctypes.c_double * 3)]


class c_stats(ctypes.Structure):
    _fields_ = [("last_kernel_ms", ctypes.c_double), ("last_flops", ctypes.c_double),
                ("last_tasks", ctypes.c_int64), ("launches", ctypes.c_int64),
                ("last_int8_ops", ctypes.c_double), ("reserved", ctypes.c_int64 * 3)]


INFO_DTYPE = np.dtype([("status", "<i4"), ("sancho_iters_left", "<i4"),
                       ("sancho_iters_right", "<i4"), ("n_gemm", "<i4"), ("n_inv", "<i4"),
                       ("mixed_pairs", "<i4")])



class c_tune_result(ctypes.Structure):
    _fields_ = [("nb", ctypes.c_int32), ("variant", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("n_candidates", ctypes.c_int32), ("cand_variant", ctypes.c_int32 * 16),
                ("cand_ctas_per_sm", ctypes.c_int32 * 16), ("cand_us_per_energy", ctypes.c_double * 16)]


_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m liteqt_b200.build` "
                           "(the RGF solver has no CPU fallback)")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    L.rgf_opts_default.argtypes = [ctypes.POINTER(c_opts)]
    L.rgf_opts_default.restype = None
    L.rgf_ctx_create.argtypes = [ctypes.POINTER(c_opts), ctypes.POINTER(ctypes.c_void_p)]
    L.rgf_ctx_destroy.argtypes = [P]
    L.rgf_ctx_set_opts.argtypes = [P, ctypes.POINTER(c_opts)]
    L.rgf_solve_batch.argtypes = [P, ctypes.POINTER(c_device), ctypes.c_int32,
                                  ctypes.POINTER(c_task), ctypes.c_int64, P, P]
    L.rgf_green_rgf_rs.argtypes = [P] * 20
    L.rgf_rgf_g.argtypes = [P] * 20
    L.rgf_green_rgf_cms.argtypes = [P] * 21
    L.rgf_green_rgf_cms.restype = ctypes.c_int
    L.rgf_w_solve_batch.argtypes = [P, ctypes.POINTER(c_w_device), ctypes.c_int32,
                                    ctypes.POINTER(c_w_task), ctypes.c_int64, P, P]
    L.rgf_w_solve_energies.argtypes = [P, ctypes.POINTER(c_w_device), ctypes.c_int64] + [P] * 9
    L.rgf_green_rgf_calc_w.argtypes = [P] * 18
    for name in ("rgf_w_solve_batch", "rgf_w_solve_energies", "rgf_green_rgf_calc_w"):
        getattr(L, name).restype = ctypes.c_int
    I64, D = ctypes.c_int64, ctypes.c_double
    L.rgf_gw_polarization.argtypes = [P] + [I64] * 6 + [D, D, ctypes.c_int32] + [P] * 7
    L.rgf_gw_self_energy.argtypes = [P] + [I64] * 6 + [D, D, ctypes.c_int32] + [P] * 10
    L.rgf_gw_polarization.restype = ctypes.c_int
    L.rgf_gw_self_energy.restype = ctypes.c_int
    L.rgf_gw_last_error.restype = ctypes.c_char_p
    L.rgf_gw_polarization_fft.argtypes = [P] + [I64] * 8 + [D, D] + [P] * 9
    L.rgf_gw_self_energy_fft.argtypes = [P] + [I64] * 8 + [D] + [P] * 10
    L.rgf_gw_polarization_fft.restype = ctypes.c_int
    L.rgf_gw_self_energy_fft.restype = ctypes.c_int
    L.rgf_gw_fft_last_error.restype = ctypes.c_char_p
    L.rgf_permute_c16.argtypes = [P, P, P, ctypes.c_int32, P, P, P]
    L.rgf_permute_c16.restype = ctypes.c_int
    L.rgf_permute_last_error.restype = ctypes.c_char_p
    S, I32 = ctypes.c_char_p, ctypes.c_int32
    L.rgf_write_spectrum.argtypes = [P, S, I32, P, I64, P, I64, I64, I64, I64, D, P, I32, I32]
    L.rgf_write_dos.argtypes = [P, S, I32, P, I64, P, I64, I64, I64, I64, D, I32]
    L.rgf_write_current_spectrum.argtypes = [P, S, I32, P, I64, P, I64, I64, I64, D, I32, I32]
    L.rgf_write_current_summed_over_k.argtypes = [P, S, I32, P, I64, I64, D, I64]
    L.rgf_write_transmission_spectrum.argtypes = [S, I32, P, I64, P, I64, I32]
    L.rgf_write_id_iteration.argtypes = [S, I32, D, D]
    for name in ("rgf_write_spectrum", "rgf_write_dos", "rgf_write_current_spectrum",
                 "rgf_write_current_summed_over_k", "rgf_write_transmission_spectrum", "rgf_write_id_iteration"):
        getattr(L, name).restype = ctypes.c_int
    L.rgf_io_last_error.restype = ctypes.c_char_p
    L.rgf_read_ham_dat.argtypes = [S, P, P, P]
    L.rgf_read_ham_dat.restype = ctypes.c_int
    L.rgf_solve_energies.argtypes = [P, ctypes.POINTER(c_device), ctypes.c_int64] + [P] * 13
    L.rgf_terminal_current.argtypes = [P, P, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int64, P]
    L.rgf_calc_n_electron.argtypes = [P, P, P, ctypes.c_int64, P, ctypes.c_int64, ctypes.c_int64,
                                      ctypes.c_int64, P, P, P]
    L.rgf_ctx_get_stats.argtypes = [P, ctypes.POINTER(c_stats)]
    L.rgf_ctx_synchronize.argtypes = [P]
    L.rgf_ctx_synchronize.restype = ctypes.c_int
    L.rgf_calc_block_current.argtypes = [P, P, P, ctypes.c_int64, P, ctypes.c_double, ctypes.c_int64,
                                         ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, P, P, P]
    L.rgf_calc_block_current.restype = ctypes.c_int
    L.rgf_adjoint_energies.argtypes = [P, ctypes.POINTER(c_device), ctypes.c_int64, P, P, P, P,
                                       ctypes.c_double, P, P, P, P]
    L.rgf_plan_create.argtypes = [P, ctypes.POINTER(c_device), ctypes.c_int32, ctypes.POINTER(c_task),
                                  ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p)]
    L.rgf_plan_execute.argtypes = [P, P, P]
    L.rgf_plan_destroy.argtypes = [P]
    L.rgf_autotune.argtypes = [P, ctypes.POINTER(c_device), ctypes.POINTER(c_tune_result)]
    L.rgf_variant_name.argtypes = [ctypes.c_int32]
    L.rgf_variant_name.restype = ctypes.c_char_p
    for name in ("rgf_plan_create", "rgf_plan_execute", "rgf_plan_destroy", "rgf_autotune"):
        getattr(L, name).restype = ctypes.c_int
    L.rgf_block_product.argtypes = [P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, P, ctypes.c_int32, P,
                                  ctypes.c_int32, P, P]
    L.rgf_block_inverse.argtypes = [P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, P, P, P, P]
    L.rgf_block_product.restype = ctypes.c_int
    L.rgf_block_inverse.restype = ctypes.c_int
    L.rgf_last_error.restype = ctypes.c_char_p
    L.rgf_version.restype = ctypes.c_char_p
    for name in ("rgf_ctx_create", "rgf_ctx_destroy", "rgf_ctx_set_opts", "rgf_solve_batch",
                 "rgf_green_rgf_rs", "rgf_rgf_g", "rgf_solve_energies", "rgf_terminal_current",
                 "rgf_calc_n_electron", "rgf_ctx_get_stats", "rgf_adjoint_energies"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def last_error() -> str:
    return load().rgf_last_error().decode()


def _check(rc, allow_status=False):
    if rc == RGF_OK or (allow_status and rc == RGF_E_STATUS):
        return rc
    raise RgfError(rc, last_error())


@dataclass
class Options:
    """rgf_opts.  Defaults reproduce green_RGF_RS (compat mode)."""
    device: int = 0
    eta_dev: float = 0.0
    eta_lead: float = 1e-3
    boltz: float = BOLTZ_RGF_RS
    sancho_tol: float = 1e-100
    sancho_nmax: int = 100
    consistent: bool = False
    precision: int = RGF_PREC_FP64
    want_T: bool = True
    verbose: bool = False
    zero_copy: bool = True
    pipelined: bool = False

    def c(self) -> c_opts:
        o = c_opts()
        load().rgf_opts_default(ctypes.byref(o))
        o.device = self.device
        o.eta_dev = self.eta_dev
        o.eta_lead = self.eta_lead
        o.boltz = self.boltz
        o.sancho_tol = self.sancho_tol
        o.sancho_nmax = int(self.sancho_nmax)
        o.consistent = int(self.consistent)
        o.precision = int(self.precision)
        o.want_T = int(self.want_T)
        o.verbose = int(self.verbose)
        o.zero_copy = int(self.zero_copy)
        o.pipelined = int(self.pipelined)
        return o


def _ptr(a):
    """Address of a NumPy array or torch tensor (host or CUDA), or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous (Fortran block layout)")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


class Plan:
    """An rgf_plan: replay with execute(); release with close()."""

    def __init__(self, h, n_tasks):
        self.h = h
        self.n_tasks = n_tasks

    def execute(self, info=None, stream=None, allow_status=True):
        return _check(load().rgf_plan_execute(self.h, _ptr(info), stream), allow_status)

    def close(self):
        if self.h:
            load().rgf_plan_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Context:
    """An rgf_ctx: device workspace and stream.  Use one per host thread."""

    def __init__(self, opts: Options | None = None):
        self.opts = opts or Options()
        L = load()
        h = ctypes.c_void_p()
        o = self.opts.c()
        _check(L.rgf_ctx_create(ctypes.byref(o), ctypes.byref(h)))
        self.h = h

    def stats(self) -> dict:
        s = c_stats()
        _check(load().rgf_ctx_get_stats(self.h, ctypes.byref(s)))
        return dict(last_kernel_ms=s.last_kernel_ms, last_flops=s.last_flops,
                    last_tasks=s.last_tasks, launches=s.launches, last_int8_ops=s.last_int8_ops)

    # ------------------------------------------------------------------ blocks
    def block_product(self, A, B, C, conj_a=False, conj_b=False, precision=None, stream=None):
        """rgf_block_product on device tensors of shape (count, nb, nb) (Fortran
        block layout: the last two axes are (column, row))."""
        prec = self.opts.precision if precision is None else precision
        count, nb = int(A.shape[0]), int(A.shape[-1])
        _check(load().rgf_block_product(self.h, int(prec), nb, count, _ptr(A), int(bool(conj_a)), _ptr(B),
                                      int(bool(conj_b)), _ptr(C), stream))

    def block_inverse(self, X, Xinv, status=None, precision=None, stream=None, allow_status=True):
        """rgf_block_inverse on device tensors of shape (count, nb, nb); status:
        host int32 array (count,) or None."""
        prec = self.opts.precision if precision is None else precision
        count, nb = int(X.shape[0]), int(X.shape[-1])
        return _check(load().rgf_block_inverse(self.h, int(prec), nb, count, _ptr(X), _ptr(Xinv), _ptr(status),
                                            stream), allow_status)

    def set_opts(self, opts: Options):
        o = opts.c()
        _check(load().rgf_ctx_set_opts(self.h, ctypes.byref(o)))
        self.opts = opts

    def synchronize(self):
        """rgf_ctx_synchronize: wait for queued (pipelined) solves and copies."""
        _check(load().rgf_ctx_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None):
            load().rgf_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------ batch
    def solve_energies(self, Hii, H1i, E, mu, temp, *, sigma_lesser=None, sigma_r=None,
                       ldos=None, ndens=None, pdens=None, GRi1=None, cur=None, tr=None, tre=None,
                       T=None, info=None, stream=None, allow_status=True, Sii=None):
        """Solve all energies of one device (rgf_solve_energies).

        Hii, H1i (and the overlap Sii of green_RGF_CMS, or None): (nx, nm, nm)
        complex128.  Per-energy arrays: (nen, nx, nm, nm); tr, tre, T: (nen,)
        float64.  Outputs are written in place.  Returns the rc (RGF_OK or
        RGF_E_STATUS)."""
        nx, nm = int(Hii.shape[0]), int(Hii.shape[1])
        d = c_device()
        d.nm, d.nx = nm, nx
        d.Hii, d.H1i = _ptr(Hii), _ptr(H1i)
        d.Sii = _ptr(Sii)
        d.mu[0], d.mu[1] = float(mu[0]), float(mu[1])
        d.temp[0], d.temp[1] = float(temp[0]), float(temp[1])
        nen = int(E.shape[0])
        rc = load().rgf_solve_energies(
            self.h, ctypes.byref(d), nen, _ptr(E), _ptr(sigma_lesser), _ptr(sigma_r), _ptr(ldos),
            _ptr(ndens), _ptr(pdens), _ptr(GRi1), _ptr(cur), _ptr(tr), _ptr(tre), _ptr(T),
            _ptr(info), stream)
        return _check(rc, allow_status)

    def adjoint_energies(self, Hii, H1i, E, mu, temp, *, T=None, dTdV=None, dTds=None,
                         spindeg=1.0, want_current=True, info=None, stream=None, allow_status=True):
        """rgf_adjoint_energies: T(E), dT/dV_l, dT/ds per energy and the current's
        derivatives.  Returns (dIdV, dIds) (NumPy) when want_current."""
        nx, nm = int(Hii.shape[0]), int(Hii.shape[1])
        d = c_device()
        d.nm, d.nx = nm, nx
        d.Hii, d.H1i = _ptr(Hii), _ptr(H1i)
        d.mu[0], d.mu[1] = float(mu[0]), float(mu[1])
        d.temp[0], d.temp[1] = float(temp[0]), float(temp[1])
        E = np.ascontiguousarray(E, np.float64)
        dIdV = np.zeros(nx) if want_current else None
        dIds = np.zeros(1) if want_current else None
        rc = load().rgf_adjoint_energies(self.h, ctypes.byref(d), int(E.shape[0]), _ptr(E), _ptr(T),
                                         _ptr(dTdV), _ptr(dTds), float(spindeg), _ptr(dIdV),
                                         _ptr(dIds), _ptr(info), stream)
        _check(rc, allow_status)
        return (dIdV, float(dIds[0])) if want_current else None

    def plan(self, devices, tasks):
        """rgf_plan_create: a CUDA-graph-captured batched solve over ctypes
        c_device / c_task arrays whose pointers are all device memory."""
        nd, nt = len(devices), len(tasks)
        DA = (c_device * nd)(*devices)
        TA = (c_task * nt)(*tasks)
        h = ctypes.c_void_p()
        _check(load().rgf_plan_create(self.h, DA, nd, TA, nt, ctypes.byref(h)))
        return Plan(h, nt)

    def autotune(self, Hii, H1i, mu, temp) -> dict:
        """rgf_autotune for the block size of this device; returns the choice
        and every candidate's time per energy."""
        nx, nm = int(Hii.shape[0]), int(Hii.shape[1])
        d = c_device()
        d.nm, d.nx = nm, nx
        d.Hii, d.H1i = _ptr(Hii), _ptr(H1i)
        d.mu[0], d.mu[1] = float(mu[0]), float(mu[1])
        d.temp[0], d.temp[1] = float(temp[0]), float(temp[1])
        r = c_tune_result()
        _check(load().rgf_autotune(self.h, ctypes.byref(d), ctypes.byref(r)))
        cands = [(VARIANTS[r.cand_variant[i]], r.cand_ctas_per_sm[i], r.cand_us_per_energy[i])
                 for i in range(r.n_candidates)]
        return {"nb": r.nb, "variant": VARIANTS[r.variant], "ctas_per_sm": r.ctas_per_sm,
                "candidates": cands}

    def w_solve_energies(self, Vii, V1i, PL, PG, PR, *, WL, WG, WR, WRi1=None, info=None,
                         stream=None, allow_status=True):
        """rgf_w_solve_energies: W^<, W^>, W^R (and W^R_{l,l+1}) of every
        energy of one q-point; arrays (nen, nx, nm, nm), host or device."""
        nx, nm = int(Vii.shape[0]), int(Vii.shape[1])
        d = c_w_device()
        d.nm, d.nx = nm, nx
        d.Vii, d.V1i = _ptr(Vii), _ptr(V1i)
        nen = int(PL.shape[0])
        rc = load().rgf_w_solve_energies(self.h, ctypes.byref(d), nen, _ptr(PL), _ptr(PG), _ptr(PR),
                                         _ptr(WL), _ptr(WG), _ptr(WR), _ptr(WRi1), _ptr(info), stream)
        return _check(rc, allow_status)

    def gw_polarization(self, GL, GG, GR, *, PL, PG, PR, nky, nkz, ndiag, dE, spindeg, imag_only=True,
                        stream=None):
        """rgf_gw_polarization; arrays (nk, nen, nx, nm, nm) (the Fortran
        (nm,nm,nx,nen,nk) layout), host or device."""
        nk, nen, nx, nm = (int(v) for v in GL.shape[:4])
        rc = load().rgf_gw_polarization(self.h, nm, nx, nen, int(nky), int(nkz), int(ndiag), float(dE),
                                        float(spindeg), int(imag_only), _ptr(GL), _ptr(GG), _ptr(GR),
                                        _ptr(PL), _ptr(PG), _ptr(PR), stream)
        if rc != RGF_OK:
            raise RgfError(rc, load().rgf_gw_last_error().decode())

    def gw_self_energy(self, GL, GG, GR, WL, WG, WR, *, SL, SG, SR, nky, nkz, ndiag, dE, alpha_mix,
                       imag_only=True, stream=None):
        """rgf_gw_self_energy; SL / SG / SR (the running self-energies) are
        updated in place."""
        nk, nen, nx, nm = (int(v) for v in GL.shape[:4])
        rc = load().rgf_gw_self_energy(self.h, nm, nx, nen, int(nky), int(nkz), int(ndiag), float(dE),
                                       float(alpha_mix), int(imag_only), _ptr(GL), _ptr(GG), _ptr(GR),
                                       _ptr(WL), _ptr(WG), _ptr(WR), _ptr(SL), _ptr(SG), _ptr(SR), stream)
        if rc != RGF_OK:
            raise RgfError(rc, load().rgf_gw_last_error().decode())

    def gw_polarization_fft(self, GL, GG, GR, GLt, GGt, *, PL, PG, PR, nky, nkz, nm, ndiag, first_ij, dEn,
                            spindeg, stream=None):
        """rgf_gw_polarization_fft on device arrays in the *_by_blocks layout,
        NumPy view (nij, nx, nk, nen) of the Fortran (nen, nk, nx, nij)."""
        nij, nx, nk, nen = (int(v) for v in GL.shape)
        rc = load().rgf_gw_polarization_fft(self.h, int(nm), nx, nen, int(nky), int(nkz), int(ndiag), nij,
                                            int(first_ij), float(dEn), float(spindeg), _ptr(GL), _ptr(GG),
                                            _ptr(GR), _ptr(GLt), _ptr(GGt), _ptr(PL), _ptr(PG), _ptr(PR), stream)
        if rc != RGF_OK:
            raise RgfError(rc, load().rgf_gw_fft_last_error().decode())

    def gw_self_energy_fft(self, GL, GG, GR, WL, WG, WR, *, SL, SG, SR, nky, nkz, nm, ndiag, first_ij, dEn,
                           stream=None):
        """rgf_gw_self_energy_fft (same layout as gw_polarization_fft)."""
        nij, nx, nk, nen = (int(v) for v in GL.shape)
        rc = load().rgf_gw_self_energy_fft(self.h, int(nm), nx, nen, int(nky), int(nkz), int(ndiag), nij,
                                           int(first_ij), float(dEn), _ptr(GL), _ptr(GG), _ptr(GR), _ptr(WL),
                                           _ptr(WG), _ptr(WR), _ptr(SL), _ptr(SG), _ptr(SR), stream)
        if rc != RGF_OK:
            raise RgfError(rc, load().rgf_gw_fft_last_error().decode())

    def permute(self, src, dst, src_shape, order, stream=None):
        """rgf_permute_c16: dst = RESHAPE(src, ORDER=order) (Fortran meaning,
        1-based order) of flat complex128 device tensors."""
        shp = (ctypes.c_int64 * len(src_shape))(*[int(v) for v in src_shape])
        odr = (ctypes.c_int32 * len(order))(*[int(v) for v in order])
        rc = load().rgf_permute_c16(self.h, _ptr(src), _ptr(dst), len(src_shape), ctypes.addressof(shp),
                                    ctypes.addressof(odr), stream)
        if rc != RGF_OK:
            raise RgfError(rc, load().rgf_permute_last_error().decode())

    def solve_batch(self, devices, tasks, info=None, stream=None, allow_status=True):
        """rgf_solve_batch with ctypes c_device / c_task arrays."""
        nd, nt = len(devices), len(tasks)
        DA = (c_device * nd)(*devices)
        TA = (c_task * nt)(*tasks)
        rc = load().rgf_solve_batch(self.h, DA, nd, TA, nt, _ptr(info), stream)
        return _check(rc, allow_status)

    def terminal_current(self, tr, dE, spindeg=1.0, nk=1):
        out = ctypes.c_double()
        _check(load().rgf_terminal_current(self.h, _ptr(tr), int(tr.shape[0]), float(dE),
                                           float(spindeg), int(nk), ctypes.addressof(out)))
        return out.value

    def calc_block_current(self, H, G_lesser, E, spindeg, nb, ns, jdens=False):
        """calc_block_current (green_rgf.f90:4602-4640).  H (nx, nm, nm), G_lesser
        (nen, nx, nm, nm) Fortran block layouts.  Returns tot_cur, tot_ecur
        (nx*ns, nb, nb) and jdens (nen, nx*ns, nb, nb) or None."""
        nx, nm = int(H.shape[0]), int(H.shape[1])
        nen = int(G_lesser.shape[0])
        E = np.ascontiguousarray(E, np.float64)
        tc = np.zeros((nx * ns, nb, nb))
        te = np.zeros((nx * ns, nb, nb))
        jd = np.zeros((nen, nx * ns, nb, nb)) if jdens else None
        _check(load().rgf_calc_block_current(self.h, _ptr(H), _ptr(G_lesser), nen, _ptr(E), float(spindeg),
                                             int(nb), int(ns), nm, nx, _ptr(tc), _ptr(te), _ptr(jd)))
        return tc, te, jd

    def calc_n_electron(self, G_lesser, G_greater, E, midgap):
        """G arrays (nk, nen, nx, nm, nm): the Fortran (nm,nm,nx,nen,nk) layout."""
        nk, nen, nx, nm = (int(s) for s in G_lesser.shape[:4])
        ne = np.zeros(nx)
        pe = np.zeros(nx)
        _check(load().rgf_calc_n_electron(self.h, _ptr(G_lesser), _ptr(G_greater), nen, _ptr(E),
                                          nm, nk, nx, _ptr(ne), _ptr(pe), _ptr(midgap)))
        return ne, pe


# ---------------------------------------------------------------------- drop-ins
def _scalar_slot(x):
    a = np.zeros(1, np.float64) if x is None or np.isscalar(x) else x
    return a


def green_RGF_RS(TEMP, nm, nx, E, mu, Hii, H1i, sigma_lesser_ph, sigma_greater_ph, sigma_r_ph,
                 ndens, pdens, ldos, tr, tre, cur, GRi1=None, GLi1=None, GGi1=None, ctx=None):
    """Drop-in for green_RGF_RS (src/green_rgf.f90:3950), same argument order.

    ndens, pdens, ldos, cur (and the optional GRi1, GLi1, GGi1) are written in
    place.  Fortran's inout scalars tr / tre are 1-element float64 arrays
    written in place (or None); the pair (tr, tre) is also returned."""
    return _drop_in(load().rgf_green_rgf_rs, False, TEMP, nm, nx, E, mu, Hii, H1i,
                    sigma_lesser_ph, sigma_greater_ph, sigma_r_ph, ndens, pdens, ldos, tr, tre,
                    cur, GRi1, GLi1, GGi1, ctx)


def RGF_G(temperature, nm, nx, E, mu, Hii, H1i, sigma_lesser_ph, sigma_greater_ph, sigma_r_ph,
          tr, tre, ndens, pdens, ldos, cur, GRi1=None, GLi1=None, GGi1=None, ctx=None):
    """Drop-in for RGF_G (src/rgf_mod.f90:26): its argument order and BOLTZ."""
    return _drop_in(load().rgf_rgf_g, True, temperature, nm, nx, E, mu, Hii, H1i,
                    sigma_lesser_ph, sigma_greater_ph, sigma_r_ph, ndens, pdens, ldos, tr, tre,
                    cur, GRi1, GLi1, GGi1, ctx)


def green_RGF_CMS(TEMP, nm, nx, E, mu, Sii, Hii, H1i, sigma_lesser_ph, sigma_greater_ph, sigma_r_ph,
                  ndens, pdens, ldos, tr, tre, cur, GRi1=None, GLi1=None, GGi1=None, ctx=None):
    """Drop-in for green_RGF_CMS (src/green_rgf.f90:4167): green_RGF_RS's
    arguments with the overlap blocks Sii before Hii."""
    return _drop_in(load().rgf_green_rgf_cms, False, TEMP, nm, nx, E, mu, Hii, H1i,
                    sigma_lesser_ph, sigma_greater_ph, sigma_r_ph, ndens, pdens, ldos, tr, tre,
                    cur, GRi1, GLi1, GGi1, ctx, Sii=Sii)


def green_rgf_calc_w(NBC, nm, nx, Vii, V1i, PL, PG, PR, WL, WG, WR, PL1i=None, PG1i=None, PR1i=None,
                     WLi1=None, WGi1=None, WRi1=None, ctx=None):
    """Drop-in for green_rgf_calc_w (src/green_rgf.f90:3399) / RGF_W
    (src/rgf_mod.f90:242): same argument order; WL, WG, WR (and WRi1) are
    written in place."""
    nbc = ctypes.c_int64(int(NBC))
    nm_ = ctypes.c_int64(int(nm))
    nx_ = ctypes.c_int64(int(nx))
    h = ctx.h if ctx is not None else None
    P = _ptr
    _check(load().rgf_green_rgf_calc_w(h, ctypes.addressof(nbc), ctypes.addressof(nm_),
                                       ctypes.addressof(nx_), P(Vii), P(V1i), P(PL), P(PG), P(PR),
                                       P(WL), P(WG), P(WR), P(PL1i), P(PG1i), P(PR1i), P(WLi1),
                                       P(WGi1), P(WRi1)))


def _drop_in(fn, rgf_g_order, TEMP, nm, nx, E, mu, Hii, H1i, sl, sg, sr, ndens, pdens, ldos, tr,
             tre, cur, GRi1, GLi1, GGi1, ctx, Sii=None):
    temp = np.ascontiguousarray(TEMP, np.float64)
    muv = np.ascontiguousarray(mu, np.float64)
    nm_ = ctypes.c_int64(int(nm))
    nx_ = ctypes.c_int64(int(nx))
    E_ = ctypes.c_double(float(E))
    trs = _scalar_slot(tr)
    tres = _scalar_slot(tre)
    P = _ptr
    h = ctx.h if ctx is not None else None
    base = [h, P(temp), ctypes.addressof(nm_), ctypes.addressof(nx_), ctypes.addressof(E_), P(muv)]
    if Sii is not None:
        base.append(P(Sii))
    base += [P(Hii), P(H1i), P(sl), P(sg), P(sr)]
    if rgf_g_order:
        args = base + [P(trs), P(tres), P(ndens), P(pdens), P(ldos), P(cur), P(GRi1), P(GLi1),
                       P(GGi1)]
    else:
        args = base + [P(ndens), P(pdens), P(ldos), P(trs), P(tres), P(cur), P(GRi1), P(GLi1),
                       P(GGi1)]
    _check(fn(*args))
    return float(trs[0]), float(tres[0])
