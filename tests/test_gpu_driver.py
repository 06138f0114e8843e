"""GPU runs of the drop-in driver (modes 2, 3, 31 and 32 of the reference's
`program simulation`), checked line by line against the FP64 oracle and the
reference's output formats."""
import re

import numpy as np
import pytest

from nrqcd_b200 import driver

pytestmark = pytest.mark.gpu

E16 = r"[+-]0\.\d{9}E[+-]\d\d"
E13 = r"[+-]0\.\d{6}E[+-]\d\d"


def rec(pat, n):
    """n values of one Fortran record, one blank apart, none trailing."""
    return f"{pat}(?: {pat}){{{n - 1}}}"


def test_mode32_free_correlators_match_oracle(oracle, tmp_path):
    n, a, M = (6, 6, 6), (0.05, 1.0, 1.0, 1.0), 1.0
    fc, fn = tmp_path / "mesoncorrelators.txt", tmp_path / "norm.txt"
    args = ["32", "6", "6", "6", "0.05", "1.0", "1.0", "1.0", "0.25", "1", "1e-12", "1.0",
            "1.0", "0.0", "1.0", "0.0", "1.0", "0.0", "1.0", "0.0", str(fc), str(fn)]
    driver.main(args)
    corr = fc.read_text().splitlines()
    norm = fn.read_text().splitlines()
    assert corr[0] == driver.CORRELATOR_HEADER and norm[0] == driver.NORM_HEADER
    assert len(corr) == 7 and len(norm) == 7  # s = 0 and 5 steps
    for ln in corr[1:]:
        assert re.fullmatch(rec(E16, 9), ln), ln
    for ln in norm[1:]:
        assert re.fullmatch(rec(E16, 3), ln), ln
    links, ef = oracle.cold(n, a)
    q, an = oracle.single_point(n, 1), oracle.single_point(n, 1)
    for step in range(6):
        if step > 0:
            oracle.cn_update(n, a, links, ef, M, [1, 1, 1, 1], 1.0, q, an, tol=1e-14)
            oracle.gauge_update(n, a, links, ef, 1.0)
        ref = oracle.meson_correlators(n, q, an)
        vals = [float(v) for v in corr[1 + step].split()]
        assert abs(vals[0] - 0.05 * step) < 1e-9
        got = [complex(vals[1 + 2 * k], vals[2 + 2 * k]) for k in range(4)]
        for g_, key in zip(got, ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1")):
            assert abs(g_ - ref[key]) <= 1e-8 * max(1.0, abs(ref[key]))
        nv = [float(v) for v in norm[1 + step].split()]
        assert abs(nv[1] - oracle.heavy_norm(n, q)) < 1e-8 and abs(nv[2] - oracle.heavy_norm(n, an)) < 1e-8


def test_mode2_energy_gauss_matches_oracle(oracle, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    n, a = (6, 6, 6), (0.05, 1.0, 1.0, 1.0)
    driver.main(["2", "6", "6", "6", "0.05", "1.0", "1.0", "1.0", "0.0", "0.25", "3", "0.8", "1.0", "0.0"])
    lines = (tmp_path / "energy_gauss.txt").read_text().splitlines()
    assert len(lines) == 6
    links, ef = oracle.transverse_box(n, a, 0.8, 1.0, 0.0, 3, identity_links=False)
    for step, ln in enumerate(lines):
        assert re.fullmatch(rec(E13, 3), ln), ln
        t, en, gauss = (float(v) for v in ln.split())
        e_ref = oracle.energy(n, a, links, ef)
        assert abs(t - 0.05 * step) < 1e-9
        assert abs(en - e_ref) <= 1e-6 * abs(e_ref)
        assert abs(gauss - oracle.gauss_ref(n, a, links, ef)) <= 1e-6 * max(1.0, abs(e_ref))
        oracle.gauge_update(n, a, links, ef, 1.0)


def test_mode3_ts_grid_matches_oracle(oracle, tmp_path):
    """(t,s)-grid correlator on a 6^3 transverse box: two backward leapfrog
    steps to t1 = -0.1, then copies of the configuration and of the point
    source evolved to every t2; every recorded point against the oracle run
    through the same loops."""
    n, ds, M, c = (6, 6, 6), 0.1, 1.0, [1, 1, 1, 1]
    a = (ds / 2, 1.0, 1.0, 1.0)
    tmin, tmax, smax, seed, qs, amp, coupling = 0.0, 0.1, 0.2, 3, 0.8, 1.0, 0.5
    fc, fn = tmp_path / "mesoncorrelators.txt", tmp_path / "norm.txt"
    args = ["3", "6", "6", "6", str(ds), "1.0", "1.0", "1.0", str(tmin), str(tmax), str(smax), str(seed),
            str(qs), str(amp), str(coupling), "1e-12", str(M),
            "1.0", "0.0", "1.0", "0.0", "1.0", "0.0", "1.0", "0.0", str(fc), str(fn)]
    driver.main(args)
    corr = fc.read_text().splitlines()
    norm = fn.read_text().splitlines()
    assert corr[0] == "s Re0.0 Im0.0 Re0.1 Im0.1" and norm[0] == "s Q0.0 A0.0 Q0.1 A0.1"
    assert len(corr) == 4 and len(norm) == 4  # s = 0, 0.1, 0.2
    for ln in corr[1:] + norm[1:]:
        assert re.fullmatch(rec(E16, 5), ln), ln
    got_c = [[float(v) for v in ln.split()] for ln in corr[1:]]
    got_n = [[float(v) for v in ln.split()] for ln in norm[1:]]
    assert got_c[0][1:] == [0.0, 1.0, 0.0, 1.0] and got_n[0][1:] == [1.0] * 4  # preset s = 0 row

    links, ef = oracle.transverse_box(n, a, qs, amp, coupling, seed, identity_links=False)
    sign, n_pre, rows = driver.ts_grid_schedule(a[0], ds, tmin, tmax, smax)
    for _ in range(n_pre):
        oracle.gauge_update(n, a, links, ef, sign)
    seen = 0
    for _, steps in rows:
        l2, e2 = links.copy(), ef.copy()
        q, an = oracle.single_point(n, 1), oracle.single_point(n, 1)
        for _, pt in steps:
            oracle.cn_update(n, a, l2, e2, M, c, 1.0, q, an, tol=1e-14)
            oracle.gauge_update(n, a, l2, e2, 1.0)
            if pt is None:
                continue
            is_, it_ = pt
            ref = oracle.meson_correlators(n, q, an)["o1_3s1"]
            g = complex(got_c[is_][1 + 2 * it_], got_c[is_][2 + 2 * it_])
            assert abs(g - ref) <= 1e-8 * max(1.0, abs(ref)), (pt, g, ref)
            assert abs(got_n[is_][1 + 2 * it_] - oracle.heavy_norm(n, q)) < 1e-8
            assert abs(got_n[is_][2 + 2 * it_] - oracle.heavy_norm(n, an)) < 1e-8
            seen += 1
        oracle.gauge_update(n, a, links, ef, 1.0)
    assert seen == 4


def test_mode31_one_t_correlators_match_oracle(oracle, tmp_path):
    """Mode 31 on 6^3: the configuration evolved to t = 0.1, then for
    it1 = 1, 2 a copy of it evolved forward 2 it1 steps (s = 2 it1 a0) and
    the configuration stepped back once; all three files against the
    oracle."""
    n, a, M, c = (6, 6, 6), (0.05, 1.0, 1.0, 1.0), 1.0, [1, 1, 1, 1]
    tcom, smax, seed, qs, amp, coupling = 0.1, 0.2, 5, 0.8, 1.0, 0.5
    fc, fn, fg = tmp_path / "c.txt", tmp_path / "n.txt", tmp_path / "g.txt"
    args = ["31", "6", "6", "6", "0.05", "1.0", "1.0", "1.0", str(tcom), str(smax), str(seed), str(qs), str(amp),
            str(coupling), "1e-12", str(M), "1.0", "0.0", "1.0", "0.0", "1.0", "0.0", "1.0", "0.0",
            str(fc), str(fn), str(fg)]
    driver.main(args)
    corr, norm, gcj = (f.read_text().splitlines() for f in (fc, fn, fg))
    assert corr[0] == driver.CORRELATOR_HEADER == gcj[0] and norm[0] == driver.NORM_HEADER
    assert len(corr) == len(norm) == len(gcj) == 4  # s = 0, 0.1, 0.2
    links, ef = oracle.transverse_box(n, a, qs, amp, coupling, seed, identity_links=False)
    oracle.gauge_update(n, a, links, ef, 1.0)
    oracle.gauge_update(n, a, links, ef, 1.0)
    q0, a0 = oracle.single_point(n, 1), oracle.single_point(n, 1)
    keys = ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1")

    def check(row, s, q, an):
        assert abs(float(corr[row].split()[0]) - s) < 1e-9
        for lines, ref in ((corr, oracle.meson_correlators(n, q, an)),
                           (gcj, oracle.meson_correlators_gconjg(n, q, an))):
            vals = [float(v) for v in lines[row].split()]
            for k, key in enumerate(keys):
                g_ = complex(vals[1 + 2 * k], vals[2 + 2 * k])
                assert abs(g_ - ref[key]) <= 1e-8 * max(1.0, abs(ref[key])), (row, key)
        nv = [float(v) for v in norm[row].split()]
        assert abs(nv[1] - oracle.heavy_norm(n, q)) < 1e-8 and abs(nv[2] - oracle.heavy_norm(n, an)) < 1e-8
    check(1, 0.0, q0, a0)
    for it1 in (1, 2):  # the copy first, the backward step at the end of the row (main.f90:601-617)
        l2, e2 = links.copy(), ef.copy()
        q, an = q0.copy(), a0.copy()
        for _ in range(2 * it1):
            oracle.cn_update(n, a, l2, e2, M, c, 1.0, q, an, tol=1e-14)
            oracle.gauge_update(n, a, l2, e2, 1.0)
        check(1 + it1, 0.05 * 2 * it1, q, an)
        oracle.gauge_update(n, a, links, ef, -1.0)
