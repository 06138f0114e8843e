"""GPU parity of the gluon-distribution observables against the oracle,
through the C ABI: Coulomb gauge fixing (src/gaugeconfiguration_su3.f90:
2269-2478), the transverse AA/EE correlators (:1825-1972) and driver mode 1
(src/main.f90:3020-3296).

The device exponential of the gauge transformation is Cayley-Hamilton based
and the oracle's is the reference's Jacobi EigenH; the device ArgLogU uses
the same Jacobi EigenC as the oracle.  Both are accurate to ~1e-15, and the
gauge fixing contracts, so the loop counters agree exactly and the links to
1e-11 after the iterations."""
import re

import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, driver
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)


def evolved_box(oracle, n, a=A, steps=10, seed=3):
    links, ef = oracle.transverse_box(n, a, 1.0, 1.0, 0.5, seed, identity_links=False)
    for _ in range(steps):
        oracle.gauge_update(n, a, links, ef, 1.0)
    return links, ef


@pytest.mark.parametrize("n,a", [((8, 8, 8), A), ((6, 5, 4), (0.05, 1.0, 1.2, 0.9))])
def test_coulomb_gaugefix_matches_oracle(oracle, n, a):
    links, ef = evolved_box(oracle, n, a)
    with lattice_ctx(n, a):
        g = GaugeConfiguration()
        g.upload(links, ef)
        it, dev = g.CoulombGaugefixing(1e-8, 0.08, 100, verbose=False)
        lg, eg = g.download()
    it_ref, dev_ref = oracle.coulomb_gaugefix(n, a, links, tol=1e-8, alpha=0.08, max_iterations=100)
    assert it == it_ref and 3 < it <= 100
    assert np.allclose(dev, dev_ref, rtol=1e-9, atol=1e-15)
    assert dev[-1] <= 1e-8 < dev[-2]
    assert np.abs(lg - links).max() < 1e-11
    assert np.array_equal(eg, ef)  # the electric field is not transformed


def test_coulomb_gaugefix_iteration_bound(oracle):
    n = (6, 6, 6)
    links, ef = evolved_box(oracle, n)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        it, dev = g.CoulombGaugefixing(1e-14, 0.08, 3, verbose=False)
        lg, _ = g.download()
    it_ref, dev_ref = oracle.coulomb_gaugefix(n, A, links, tol=1e-14, alpha=0.08, max_iterations=3)
    assert it == it_ref == 4 and len(dev) == 3  # the reference's counter after a full loop
    assert np.allclose(dev, dev_ref, rtol=1e-10)
    assert np.abs(lg - links).max() < 1e-12


@pytest.mark.parametrize("n,a", [((8, 8, 8), A), ((6, 5, 4), (0.05, 1.0, 1.2, 0.9))])
def test_transverse_correlators_match_oracle(oracle, n, a):
    links, ef = evolved_box(oracle, n, a)
    oracle.coulomb_gaugefix(n, a, links)
    with lattice_ctx(n, a):
        g = GaugeConfiguration()
        g.upload(links, ef)
        aa, ee, mom = g.GetTransverseCorrelators()
        aa2 = g.GetTransverseAACorrelator()
    raa, ree, rmom = oracle.transverse_correlators(n, a, links, ef)
    assert np.array_equal(aa, aa2)
    assert np.abs(mom - rmom).max() < 1e-13
    assert np.abs(aa - raa).max() < 1e-11 * np.abs(raa).max()
    assert np.abs(ee - ree).max() < 1e-11 * np.abs(ree).max()
    assert aa[0] == 0.0 and ee[0] == 0.0 and np.all(aa >= -1e-15) and np.all(ee >= -1e-15)


def test_mode1_gluon_distribution_matches_oracle(oracle, tmp_path, capsys):
    n, a = (6, 6, 6), A
    f = tmp_path / "gluondist.txt"
    driver.main(["1", "6", "6", "6", "0.05", "1.0", "1.0", "1.0", "0.25", "3", "1.0", "1.0", "0.5",
                 "100", "1e-8", "0.08", str(f)])
    lines = f.read_text().splitlines()
    assert len(lines) == 216
    e13 = r"[+-]0\.\d{6}E[+-]\d\d"
    for ln in lines:
        assert re.fullmatch(f"{e13} {e13}", ln), ln
    out = capsys.readouterr().out
    assert "iterations in Coulomb gauge fixing performed" in out
    links, ef = oracle.transverse_box(n, a, 1.0, 1.0, 0.5, 3, identity_links=False)
    for _ in range(5):  # ceiling(0.25 / 0.05)
        oracle.gauge_update(n, a, links, ef, 1.0)
    oracle.coulomb_gaugefix(n, a, links, tol=1e-8, alpha=0.08, max_iterations=100)
    aa, ee, mom = oracle.transverse_correlators(n, a, links, ef)
    got = np.array([[float(v) for v in ln.split()] for ln in lines])
    # E13.6 keeps six significant digits: relative rounding up to 5e-6
    assert np.allclose(got[:, 0], mom, rtol=6e-6, atol=1e-12)
    assert np.allclose(got[:, 1], np.sqrt(aa * ee), rtol=6e-6, atol=1e-12)
