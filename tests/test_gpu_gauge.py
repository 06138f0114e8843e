"""GPU parity of the gauge hot path against the oracle (through the C ABI).

Tolerances: FP64 kernels against the FP64 oracle.  The device exponential is
the Cayley-Hamilton/Taylor form, the oracle's the reference's Jacobi form;
both are accurate to ~1e-16 relative, so one step agrees to 1e-14 absolute
on unit-norm links, and short horizons to 1e-12.
"""
import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)


def hot_fields(oracle, n, seed=5, Q=3.0):
    return oracle.transverse_box(n, A, Q, 1.0, 0.0, seed, identity_links=False)


def test_upload_download_roundtrip(oracle):
    n = (6, 5, 4)
    links, ef = hot_fields(oracle, n)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        l2, e2 = g.download()
        assert np.array_equal(l2, links) and np.array_equal(e2, ef)


@pytest.mark.parametrize("n", [(4, 4, 4), (5, 6, 7), (8, 8, 8)])
@pytest.mark.parametrize("dt", [1.0, -1.0])
def test_leapfrog_one_step(oracle, n, dt):
    links, ef = hot_fields(oracle, n)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        g.Update(dt)
        lg, eg = g.download()
    oracle.gauge_update(n, A, links, ef, dt)
    assert np.abs(lg - links).max() < 1e-14
    assert np.abs(eg - ef).max() < 1e-14


def test_leapfrog_50_steps_and_observables(oracle):
    n = (8, 8, 8)
    links, ef = hot_fields(oracle, n, seed=2, Q=2.0)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        e_gpu = g.GetEnergy()
        gr, gm = g.GetDeviationFromGaussLaw(), g.GetGdeviation()
        assert abs(e_gpu - oracle.energy(n, A, links, ef)) < 1e-12 * abs(e_gpu)
        assert abs(gr - oracle.gauss_ref(n, A, links, ef)) < 1e-12
        assert abs(gm - oracle.gauss_maxnorm(n, A, links, ef)) < 1e-12 * max(1.0, gm)
        for _ in range(50):
            g.Update(1.0)
            oracle.gauge_update(n, A, links, ef, 1.0)
        lg, eg = g.download()
        assert np.abs(lg - links).max() < 1e-12
        assert np.abs(eg - ef).max() < 1e-12
        assert abs(g.GetEnergy() - oracle.energy(n, A, links, ef)) < 1e-11 * abs(e_gpu)


def test_reversibility_on_device(oracle):
    n = (8, 8, 8)
    links, ef = hot_fields(oracle, n, seed=9, Q=2.0)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        for _ in range(20):
            g.Update(1.0)
        for _ in range(20):
            g.Update(-1.0)
        lg, eg = g.download()
    assert np.abs(lg - links).max() < 1e-13 and np.abs(eg - ef).max() < 1e-14


@pytest.mark.parametrize("identity_links", [True, False])
def test_initial_condition_matches_oracle(oracle, identity_links):
    n = (16, 16, 16)
    # |p| of some 16^3 modes equals 2 exactly; a saturation scale on such a
    # mode makes its occupation depend on the last ulp of sin(), so both
    # scales are kept away from every |p| of the lattice (>= 8e-3)
    Q = 0.5 if identity_links else 1.7
    lo, eo = oracle.transverse_box(n, A, Q, 1.0, 0.0, 1, identity_links=identity_links)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.TransversePolarisedOccupiedInit_Box(Q, 1.0, 0.0, RandomSeed=1, identity_links=identity_links)
        lg, eg = g.download()
        if identity_links:
            assert g.GetGdeviation() < 1e-12
    assert np.abs(eg - eo).max() < 1e-13 * max(1.0, np.abs(eo).max())
    assert np.abs(lg - lo).max() < 1e-13


@pytest.mark.parametrize("n,Q", [((6, 6, 6), 1.0), ((16, 16, 16), 2.0), ((12, 6, 8), 1.0)])
def test_initial_condition_box_edge_on_a_lattice_momentum(oracle, n, Q):
    """A saturation scale equal to lattice momenta (2 sin(pi/6) = 1 on 6 and
    12 sites, 2 sin(pi/2) = 2 on 16): the device takes the momentum
    components and moduli from a host table in the reference's arithmetic,
    so the box edge |p| < Q falls as on the host."""
    lo, eo = oracle.transverse_box(n, A, Q, 1.0, 0.5, 3, identity_links=False)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.TransversePolarisedOccupiedInit_Box(Q, 1.0, 0.5, RandomSeed=3, identity_links=False)
        lg, eg = g.download()
    assert np.abs(eg - eo).max() < 1e-13 * max(1.0, np.abs(eo).max())
    assert np.abs(lg - lo).max() < 1e-13


def test_cold_init():
    n = (4, 4, 4)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.ColdInit()
        l, e = g.download()
        assert g.GetEnergy() == 0.0
    assert np.all(e == 0) and np.allclose(l[:, :, 0, 0], 1) and np.allclose(l[:, :, 1, 0], 0)
