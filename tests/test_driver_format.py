"""CPU checks of the drop-in driver's Fortran number formatting
('SP,Ew.d' of the reference's output files, src/main.f90:400-411, 2614)."""
import pytest

from nrqcd_b200.driver import CORRELATOR_HEADER, NORM_HEADER, _line, _nint, fortran_e


@pytest.mark.parametrize("x,w,d,out", [
    (1.0, 16, 9, "+0.100000000E+01"),
    (0.0, 16, 9, "+0.000000000E+00"),
    (-0.5, 16, 9, "-0.500000000E+00"),
    (1.23456789012e-5, 16, 9, "+0.123456789E-04"),
    (9.9999999996, 16, 9, "+0.100000000E+02"),
    (-123.456, 16, 9, "-0.123456000E+03"),
    (1e-120, 16, 9, "+0.100000000-119"),
    (0.05, 13, 6, "+0.500000E-01"),
    (1732.0603896, 13, 6, "+0.173206E+04"),
    (float("nan"), 16, 9, "             NaN"),
])
def test_fortran_e(x, w, d, out):
    assert fortran_e(x, w, d) == out
    assert len(fortran_e(x, w, d)) == w


def test_line_layout_and_headers():
    assert _line((0.05, 1.0, -1.0), 16, 9) == "+0.500000000E-01 +0.100000000E+01 -0.100000000E+01 "
    assert NORM_HEADER == "s Quark Antiq"
    assert CORRELATOR_HEADER.split()[0] == "s" and len(CORRELATOR_HEADER.split()) == 9


def test_nint_rounds_half_away_from_zero():
    assert _nint(2.5) == 3 and _nint(-2.5) == -3 and _nint(4.9999999) == 5 and _nint(0.49) == 0
