"""CPU tests of the writers' oracle: Fortran Ew.d / Iw formatting against
values worked out from the edit descriptors' definition, and the
reference's file-name rule."""
import pytest

from oracle.writers import STRING, fE, fI, id_iteration_line


@pytest.mark.parametrize("v,w,d,want", [
    (1.5, 18, 4, "        0.1500E+01"),
    (-0.000123456, 18, 4, "       -0.1235E-03"),
    (0.0, 18, 4, "        0.0000E+00"),
    (-0.0, 18, 4, "       -0.0000E+00"),
    (123456.0, 18, 4, "        0.1235E+06"),
    (1e-120, 18, 4, "        0.1000-119"),
    (9.99996, 18, 4, "        0.1000E+02"),
    (2.5e100, 18, 4, "        0.2500+101"),
    (3.0, 16, 6, "    0.300000E+01"),
])
def test_fortran_e_edit(v, w, d, want):
    assert len(want) == w and fE(v, w, d) == want


def test_fortran_i_and_names():
    assert fI(7, 4) == "   7" and fI(12345, 4) == "****"
    assert STRING(3) == "0003" and STRING(42) == "0042"
    assert id_iteration_line(2, 1.5e-6, -2.0e-7) == "   2    0.150000E-05   -0.200000E-06\n"
