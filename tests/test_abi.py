"""CPU tests of the drop-in boundary: the CUDA library builds, loads, exports
every entry point include/rgf.h declares, its struct layouts agree between C
and the Python mirror, and error paths work without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rgf.h")


@pytest.fixture(scope="session")
def libpath():
    from liteqt_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def harness(libpath, tmp_path_factory):
    out = tmp_path_factory.mktemp("abi") / "abi_harness"
    subprocess.check_call(["gcc", "-O1", "-Wall", "-o", str(out), os.path.join(ROOT, "tests", "abi_harness.c"),
                           "-I", os.path.join(ROOT, "include"), libpath,
                           "-Wl,-rpath," + os.path.dirname(libpath)])
    return str(out)


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"RGF_API\s+[\w\s\*]*?\b(rgf_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("rgf_solve_batch", "rgf_green_rgf_rs", "rgf_rgf_g", "rgf_ctx_create", "rgf_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    from liteqt_b200 import rgf
    assert set(rgf.EXPORTS) <= set(declared_functions())


def test_library_is_built_for_sm100a_and_has_no_cpu_solver(libpath):
    from liteqt_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)
    syms = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True).stdout
    assert "zgemm" not in syms and "oracle" not in syms


def test_struct_layouts_match_python_mirror(harness):
    from liteqt_b200 import rgf
    out = subprocess.check_output([harness, "layout"], text=True).split("\n")
    vals = {l.split()[0]: [int(x) for x in l.split()[1:]] for l in out if l.strip()}
    o = vals["opts"]
    assert o[0] == ctypes.sizeof(rgf.c_opts)
    assert o[1:] == [rgf.c_opts.eta_dev.offset, rgf.c_opts.eta_lead.offset, rgf.c_opts.boltz.offset,
                     rgf.c_opts.sancho_tol.offset, rgf.c_opts.sancho_nmax.offset,
                     rgf.c_opts.consistent.offset, rgf.c_opts.precision.offset,
                     rgf.c_opts.want_T.offset, rgf.c_opts.verbose.offset, rgf.c_opts.reserved.offset]
    d = vals["device"]
    assert d == [ctypes.sizeof(rgf.c_device), rgf.c_device.Hii.offset, rgf.c_device.mu.offset,
                 rgf.c_device.temp.offset, rgf.c_device.Sii.offset]
    t = vals["task"]
    assert t == [ctypes.sizeof(rgf.c_task), rgf.c_task.E.offset, rgf.c_task.sigma_lesser.offset,
                 rgf.c_task.cur.offset, rgf.c_task.T.offset]
    assert vals["info"] == [rgf.INFO_DTYPE.itemsize]
    assert vals["c16"] == [16]


def test_defaults_reproduce_reference_constants(libpath):
    from liteqt_b200 import rgf
    o = rgf.c_opts()
    rgf.load().rgf_opts_default(ctypes.byref(o))
    assert o.struct_size == ctypes.sizeof(rgf.c_opts)
    assert o.eta_dev == 0.0 and o.eta_lead == 1e-3          # green_rgf.f90:3974, :4474
    assert o.boltz == 8.61734e-05                           # green_rgf.f90:3968
    assert o.sancho_tol == 1e-100 and o.sancho_nmax == 100  # green_rgf.f90:4457, :4473
    assert o.consistent == 0 and o.precision == 0


def test_context_without_gpu_fails_cleanly(harness):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    out = subprocess.check_output([harness, "nogpu"], text=True).strip()
    rc, msg = out.split(" ", 1)
    assert int(rc) == -2  # RGF_E_CUDA
    assert "cudaSetDevice" in msg or "cuda" in msg.lower()


def test_fortran_interface_file_binds_every_drop_in():
    src = open(os.path.join(ROOT, "fortran", "rgf_iface.f90")).read()
    for name in ("rgf_green_rgf_rs", "rgf_rgf_g", "rgf_green_rgf_cms", "rgf_solve_energies",
                 "rgf_ctx_create"):
        assert f'bind(C, name="{name}")' in src
    assert "subroutine green_RGF_RS" in src and "subroutine RGF_G" in src
    assert "subroutine green_RGF_CMS" in src
