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
    assert _line((0.05, 1.0, -1.0), 16, 9) == "+0.500000000E-01 +0.100000000E+01 -0.100000000E+01"
    assert NORM_HEADER == "s Quark Antiq"
    assert CORRELATOR_HEADER.split()[0] == "s" and len(CORRELATOR_HEADER.split()) == 9


def test_nint_rounds_half_away_from_zero():
    assert _nint(2.5) == 3 and _nint(-2.5) == -3 and _nint(4.9999999) == 5 and _nint(0.49) == 0


# ---------------------------------------------------------------- mode 3
from nrqcd_b200.driver import fortran_f, ts_grid_bounds, ts_grid_schedule, write_ts_grid  # noqa: E402


@pytest.mark.parametrize("x,w,d,out", [
    (0.0, 3, 1, "0.0"),
    (0.1, 3, 1, "0.1"),
    (-0.5, 3, 1, "-.5"),
    (5.0, 4, 1, " 5.0"),
    (35.0, 5, 1, " 35.0"),
    (12.5, 3, 1, "***"),
    (5.0, 2, 0, "5."),
    (0.25, 4, 2, "0.25"),
    (1.05, 4, 2, "1.05"),
])
def test_fortran_f(x, w, d, out):
    assert fortran_f(x, w, d) == out


def _schedule_by_integers(tmin_q, tmax_q, smax_q):
    """The same loops in integer units of a0/2 (t = (it1+it2)/2 a0 exactly):
    a point is on the ds = 2 a0 grid iff it2-it1 is even and it1+it2 is a
    multiple of 4.  Arguments are tmin, tmax, smax in units of a0."""
    t1min_2 = 2 * tmin_q - smax_q  # 2 t1min / a0
    assert t1min_2 % 2 == 0
    rows = []
    for it1 in range(t1min_2 // 2, tmax_q + 1):
        steps = []
        for it2 in range(it1 + 1, it1 + smax_q + 1):
            t_2 = it1 + it2  # 2 t / a0
            on = (it2 - it1) % 2 == 0 and t_2 % 4 == 0
            if 2 * tmin_q <= t_2 <= 2 * tmax_q and on:
                steps.append((it2, ((it2 - it1) // 2, t_2 // 4)))
            else:
                steps.append((it2, None))
                if t_2 > 2 * tmax_q:
                    break
        rows.append((it1, steps))
    return rows


@pytest.mark.parametrize("tmin,tmax,smax", [(0.0, 0.2, 0.2), (0.0, 0.1, 0.2), (0.2, 0.4, 0.2), (0.1, 0.5, 0.4),
                                           (0.0, 0.0, 0.1)])
def test_ts_grid_schedule_matches_integer_loops(tmin, tmax, smax):
    a0, ds = 0.05, 0.1
    sign, n_pre, rows = ts_grid_schedule(a0, ds, tmin, tmax, smax)
    q = lambda v: int(round(v / a0))  # noqa: E731
    assert rows == _schedule_by_integers(q(tmin), q(tmax), q(smax))
    t1min = tmin - smax / 2
    assert n_pre == abs(q(t1min)) and sign == (1.0 if t1min >= 0 else -1.0)
    ismin, ismax, itmin, itmax = ts_grid_bounds(ds, tmin, tmax, smax)
    for _, steps in rows:
        for _, pt in steps:
            if pt is not None:
                assert ismin <= pt[0] <= ismax and itmin <= pt[1] <= itmax


def test_ts_grid_schedule_example():
    """tmin 0, tmax 0.1, smax 0.2, a0 0.05: two backward leapfrog steps,
    then rows t1 = -0.1 .. 0.1 filling every s > 0 point of the 3 x 2 grid."""
    sign, n_pre, rows = ts_grid_schedule(0.05, 0.1, 0.0, 0.1, 0.2)
    assert (sign, n_pre) == (-1.0, 2)
    pts = {pt: (it1, it2) for it1, steps in rows for it2, pt in steps if pt is not None}
    assert pts == {(2, 0): (-2, 2), (1, 0): (-1, 1), (2, 1): (0, 4), (1, 1): (1, 3)}
    assert [len(steps) for _, steps in rows] == [4, 4, 4, 3, 1]


def test_write_ts_grid_layout(tmp_path):
    nan = float("nan")
    corr = [[1j, 1j], [complex(0.5, -0.25), complex(nan, nan)], [complex(-1.0, 2.0), complex(0.125, 0.0)]]
    qn = [[1.0, 1.0], [0.99, nan], [0.98, 0.97]]
    an = [[1.0, 1.0], [0.96, nan], [0.95, 0.94]]
    fc, fn = tmp_path / "c.txt", tmp_path / "n.txt"
    write_ts_grid(str(fc), str(fn), 0.1, 0, corr, qn, an)
    c = fc.read_text().splitlines()
    n = fn.read_text().splitlines()
    assert c[0] == "s Re0.0 Im0.0 Re0.1 Im0.1" and n[0] == "s Q0.0 A0.0 Q0.1 A0.1"
    assert c[1] == "+0.000000000E+00 +0.000000000E+00 +0.100000000E+01 +0.000000000E+00 +0.100000000E+01"
    assert c[2] == ("+0.100000000E+00 +0.500000000E+00 -0.250000000E+00 "
                    "             NaN              NaN")
    assert n[3] == "+0.200000000E+00 +0.980000000E+00 +0.950000000E+00 +0.970000000E+00 +0.940000000E+00"
    assert len(c) == 4 and len(n) == 4
    # ds = 1: d = 0; t = 3 has p = nint(0.48) = 0 (F2.0), t = 4 and 5 have p = 1 (F3.0)
    write_ts_grid(str(fc), str(fn), 1.0, 3, [[1j, 1j, 1j]], [[1.0] * 3], [[1.0] * 3])
    assert fc.read_text().splitlines()[0] == "s Re3. Im3. Re 4. Im 4. Re 5. Im 5."
