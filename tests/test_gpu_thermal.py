"""GPU parity of the thermal initial condition (EquilibriumInit,
src/gaugeconfiguration_su3.f90:380-814) and of driver mode 33 against the
oracle, through the C ABI.

The projection is a contractive fixed-point iteration, so FP64 rounding
differences between the device and the oracle (fused multiply-adds, the
order of the 3x3 products) stay at the 1e-15 level of the field; the sweep
counts must agree exactly (the deviation lands on the tolerance from above
with a margin far beyond that level in these seeded cases)."""
import re

import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, driver
from nrqcd_b200._capi import NrqcdError
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)


def gauss_violating(oracle, n, seed=4):
    """Non-trivial links from the transverse box, and an electric field with
    a seeded random part that breaks the Gauss law."""
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, seed, identity_links=False)
    rng = np.random.default_rng(seed)
    ef = ef + 0.02 * rng.standard_normal(ef.shape)
    return links, ef


@pytest.mark.parametrize("n", [(4, 4, 4), (6, 5, 4)])
def test_gauss_projection_matches_oracle(oracle, n):
    links, ef = gauss_violating(oracle, n)
    dev0 = oracle.gauss_maxnorm(n, A, links, ef)
    assert dev0 > 1e-2
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        sw, dev = g.GaussProjection(1e-3)
        lg, eg = g.download()
    sw_ref = oracle.gauss_project(n, A, links, ef, tol=1e-3, max_sweeps=1_000_000)
    assert sw == sw_ref and sw > 10
    assert dev <= 1e-3 and abs(dev - oracle.gauss_maxnorm(n, A, links, ef)) < 1e-12
    assert np.array_equal(lg, links)
    assert np.abs(eg - ef).max() < 1e-12 * np.abs(ef).max()


def test_gauss_projection_bound_and_noop(oracle):
    n = (4, 4, 4)
    links, ef = gauss_violating(oracle, n)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        with pytest.raises(NrqcdError):
            g.GaussProjection(1e-3, max_sweeps=5)
        # the five sweeps were taken, as the oracle's bounded loop takes them
        _, e5 = g.download()
        l5, r5 = links.copy(), ef.copy()
        assert oracle.gauss_project(n, A, l5, r5, tol=1e-3, max_sweeps=5) == 5
        assert np.abs(e5 - r5).max() < 1e-13 * np.abs(r5).max()
        # a field that already satisfies the tolerance takes no sweep
        sw, dev = g.GaussProjection(10.0)
        assert sw == 0 and dev <= 10.0
        _, e6 = g.download()
        assert np.array_equal(e5, e6)


@pytest.mark.parametrize("n,beta,nef,neq,seed", [((4, 4, 4), 10.0, 2, 3, 7), ((6, 6, 6), 6.0, 1, 2, 3)])
def test_equilibrium_init_matches_oracle(oracle, n, beta, nef, neq, seed):
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        sw, en, dev = g.EquilibriumInit(beta, nef, neq, RandomSeed=seed, verbose=False)
        lg, eg = g.download()
    links, ef, sw_ref, en_ref, dev_ref = oracle.equilibrium_init(n, A, beta, nef, neq, 1e-3, seed)
    assert list(sw) == list(sw_ref)
    assert np.allclose(en, en_ref, rtol=1e-10, atol=0)
    assert np.all(dev <= 1e-3 * 1.01) and np.allclose(dev, dev_ref, rtol=1e-6, atol=1e-12)
    assert np.abs(lg - links).max() < 1e-11
    assert np.abs(eg - ef).max() < 1e-11 * np.abs(ef).max()


def test_equilibrium_init_energy_file(tmp_path, capsys):
    n = (4, 4, 4)
    f = tmp_path / "energy.txt"
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        sw, en, dev = g.EquilibriumInit(10.0, 2, 1, MeasureEnergy=True, filename=str(f), RandomSeed=2)
    lines = f.read_text().splitlines()
    assert len(lines) == 2
    for r, ln in enumerate(lines):
        assert re.fullmatch(r" {11}\d {3}\d+\.\d+ {5}", ln), repr(ln)
        k, e = ln.split()
        assert int(k) == r + 1 and abs(float(e) - en[r]) <= 1e-15 * en[r]
    out = capsys.readouterr().out
    assert out.count("G[U,E]=") == 2


def test_mode33_thermal_correlators_match_oracle(oracle, tmp_path):
    """Mode 33 on 6^3: EquilibriumInit (beta 10, one round, two leapfrog
    steps), then two coupled steps; every record against the oracle."""
    n, M, c = (6, 6, 6), 1.0, [1, 1, 1, 1]
    fc, fn, fe = tmp_path / "mesoncorrelators.txt", tmp_path / "norm.txt", tmp_path / "energy.txt"
    args = ["33", "6", "6", "6", "0.05", "1.0", "1.0", "1.0", "0.1", "9", "10.0", "1", "2", "1e-12", "1.0",
            "1.0", "0.0", "1.0", "0.0", "1.0", "0.0", "1.0", "0.0", str(fc), str(fn), "1", str(fe)]
    driver.main(args)
    corr = fc.read_text().splitlines()
    norm = fn.read_text().splitlines()
    assert corr[0] == driver.CORRELATOR_HEADER and norm[0] == driver.NORM_HEADER
    assert len(corr) == 4 and len(norm) == 4
    assert len(fe.read_text().splitlines()) == 1
    links, ef, _, _, _ = oracle.equilibrium_init(n, A, 10.0, 1, 2, 1e-3, 9)
    q, an = oracle.single_point(n, 1), oracle.single_point(n, 1)
    for step in range(3):
        if step > 0:
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
            oracle.gauge_update(n, A, links, ef, 1.0)
        ref = oracle.meson_correlators(n, q, an)
        vals = [float(v) for v in corr[1 + step].split()]
        assert abs(vals[0] - 0.05 * step) < 1e-9
        got = [complex(vals[1 + 2 * k], vals[2 + 2 * k]) for k in range(4)]
        for g_, key in zip(got, ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1")):
            assert abs(g_ - ref[key]) <= 1e-8 * max(1.0, abs(ref[key]))
        nv = [float(v) for v in norm[1 + step].split()]
        assert abs(nv[1] - oracle.heavy_norm(n, q)) < 1e-8 and abs(nv[2] - oracle.heavy_norm(n, an)) < 1e-8
