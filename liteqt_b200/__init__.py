"""liteqt_b200: B200-native (sm_100a) recursive Green's function (RGF) library.

The CUDA library (librgf_b200.so, C ABI in include/rgf.h) replaces the RGF hot
path of liteQT / eXcitonQT: green_RGF_RS (src/green_rgf.f90:3950-4164) and
RGF_G (src/rgf_mod.f90:26-237) with their Sancho-Rubio leads, plus batched
launches over all (device, k, E) points.  ``liteqt_b200.rgf`` mirrors the
reference interface from Python through that ABI.
"""
from .rgf import (Context, Options, RGF_G, RgfError, green_RGF_RS, load,  # noqa: F401
                  RGF_PREC_FP64, RGF_PREC_MIXED, BOLTZ_RGF_G, BOLTZ_RGF_RS)

__all__ = ["Context", "Options", "RGF_G", "RgfError", "green_RGF_RS", "load",
           "RGF_PREC_FP64", "RGF_PREC_MIXED", "BOLTZ_RGF_G", "BOLTZ_RGF_RS"]
