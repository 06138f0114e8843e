"""Parity at the workload's own configurations, against the oracle.

The reference's driver loop (src/main.f90:344-355) does, per timestep, the
Crank-Nicolson step of quark and antiquark and then a leapfrog step.  These
tests run that loop on the GPU through the Python mirror of the reference's
modules and run the oracle beside it from the same seeded fields:

* 16^3 (plain FP64): the transverse-box initial condition (n0 = 1, aQ = 0.5,
  coupling 0, ranlxd seed 1, links = 1), 200 leapfrog steps, then 100
  coupled steps at residual 1e-12 (aM = 1.0); fields compared site by site
  at steps 1, 10, 100 and 200 of the leapfrog and 1, 10 and 100 of the
  coupled loop; energy drift, both Gauss-law measures, the propagator norms,
  and the return of 100 backward coupled steps to the start.
* 32^3 (plain FP64): the same initial condition, 1000 leapfrog steps, then
  10 coupled steps at aM = 1.0 and at aM = 2.0 (residual 1e-12).
* 64^3: one application of A and of A^H by every FP64 stencil, and one
  coupled step, against the oracle.

Tolerances.  The leapfrog's long horizons are compared against the
divergence envelope of the oracle itself: the same evolution from the
initial field with every colour-electric component raised by one ulp.  At
these amplitudes the envelope grows slowly (16^3: 1.6e-14 in the links after
200 steps; 32^3: 3.4e-14 after 1000), so the link tolerance is 50 times the
envelope at the same step, and never below 1e-13.  The solves run to a
relative residual of 1e-12 on the GPU and 1e-14 in the oracle; each CN step
then differs by at most about 1e-12 per propagator entry (amplitude <= 1/sqrt 6),
and the differences of k steps add up to at most k times that: the
propagator tolerance after k coupled steps is 2e-12 k, and the norms
likewise agree to 2e-12 k.  Energies after long evolutions are compared
within 50 times the oracle's own one-ulp envelope of the energy (never below
1e-12 relative): a sum over every plaquette, it magnifies the fields'
rounding-level differences (16^3 after 200 leapfrog steps: 4e-11 absolute,
1.8e-12 relative)."""
import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField, nrqcd
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
C = [1.0, 1.0, 1.0, 1.0]
TOL = 1e-12


def initial_condition(oracle, n):
    return oracle.transverse_box(n, A, 0.5, 1.0, 0.0, 1, identity_links=True)


def leapfrog_with_envelope(oracle, n, links, ef, marks):
    """The oracle's leapfrog from (links, ef) and from the same field with
    every E component one ulp higher: {step: (links, ef, envelope_links,
    envelope_efield, envelope_energy)} at the given steps."""
    l1, e1 = links.copy(), ef.copy()
    l2, e2 = links.copy(), np.nextafter(ef, np.inf)
    out = {}
    for s in range(1, max(marks) + 1):
        oracle.gauge_update(n, A, l1, e1, 1.0)
        oracle.gauge_update(n, A, l2, e2, 1.0)
        if s in marks:
            de = abs(oracle.energy(n, A, l1, e1) - oracle.energy(n, A, l2, e2))
            out[s] = (l1.copy(), e1.copy(), float(np.abs(l1 - l2).max()), float(np.abs(e1 - e2).max()), de)
    return out


def energy_tol(e, envelope):
    """An energy after a long evolution: 50 times the oracle's own one-ulp
    envelope of it, and never below 1e-12 relative."""
    return max(1e-12 * abs(e), 50 * envelope)


def assert_leapfrog_parity(g, ref, step):
    gl, ge = g.download()
    lref, eref, env_l, env_e, _ = ref[step]
    dl, de = float(np.abs(gl - lref).max()), float(np.abs(ge - eref).max())
    assert dl <= max(1e-13, 50 * env_l), (step, dl, env_l)
    assert de <= max(1e-14, 50 * env_e), (step, de, env_e)
    return dl, de


def test_c1_16cubed_leapfrog_then_coupled_steps(oracle):
    n = (16, 16, 16)
    M = 1.0
    links, ef = initial_condition(oracle, n)
    marks = (1, 10, 100, 200)
    ref = leapfrog_with_envelope(oracle, n, links, ef, set(marks))
    with lattice_ctx(n, A, cn=(M, C, 1.0, TOL)):
        g = GaugeConfiguration()
        g.TransversePolarisedOccupiedInit_Box(0.5, 1.0, 0.0, RandomSeed=1, identity_links=True)
        gl, ge = g.download()
        assert np.abs(gl - links).max() < 1e-13 and np.abs(ge - ef).max() < 1e-13
        # links = 1 makes the field transverse: the Gauss law holds already
        assert g.GetGdeviation() <= 1e-12 and abs(g.GetDeviationFromGaussLaw()) <= 1e-12
        e_start = g.GetEnergy()
        assert abs(e_start - oracle.energy(n, A, links, ef)) <= 1e-12 * abs(e_start)
        for s in range(1, 201):
            g.Update(1.0)
            if s in marks:
                assert_leapfrog_parity(g, ref, s)
        lf_links, lf_ef, env_energy = ref[200][0], ref[200][1], ref[200][4]
        e_lf = g.GetEnergy()
        assert abs(e_lf - oracle.energy(n, A, lf_links, lf_ef)) <= energy_tol(e_lf, env_energy)

        # 100 coupled steps, the driver's order: CN step, then leapfrog step
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        q0, a0 = h.download()
        ol, oe = lf_links.copy(), lf_ef.copy()
        oq, oa = q0.copy(), a0.copy()
        for s in range(1, 101):
            st = h.Update(g, M, C, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= TOL
            g.Update(1.0)
            oracle.cn_update(n, A, ol, oe, M, C, 1.0, oq, oa, tol=1e-14)
            oracle.gauge_update(n, A, ol, oe, 1.0)
            if s in (1, 10, 100):
                gq, ga = h.download()
                assert np.abs(gq - oq).max() <= 2e-12 * s and np.abs(ga - oa).max() <= 2e-12 * s, s
                gl, ge = g.download()
                assert np.abs(gl - ol).max() <= 1e-13 and np.abs(ge - oe).max() <= 1e-14, s
        # observables after the coupled loop, against the oracle's
        e_end = g.GetEnergy()
        assert abs(e_end - oracle.energy(n, A, ol, oe)) <= energy_tol(e_end, env_energy)
        drift_gpu = abs(e_end - e_start) / abs(e_start)
        drift_oracle = abs(oracle.energy(n, A, ol, oe) - e_start) / abs(e_start)
        assert abs(drift_gpu - drift_oracle) <= energy_tol(e_end, env_energy) / abs(e_start)
        assert g.GetGdeviation() <= 1e-12 and abs(g.GetDeviationFromGaussLaw()) <= 1e-12
        assert abs(oracle.gauss_maxnorm(n, A, ol, oe) - g.GetGdeviation()) <= 1e-13
        nq, na = h.GetNorm_Quark(), h.GetNorm_AntiQ()
        assert abs(nq - oracle.heavy_norm(n, oq)) <= 2 * 100 * TOL
        assert abs(na - oracle.heavy_norm(n, oa)) <= 2 * 100 * TOL
        assert abs(nq - 1.0) <= 100 * TOL and abs(na - 1.0) <= 100 * TOL

        # forward then backward: leapfrog(-1) then CN(-1) undoes a coupled step
        for _ in range(100):
            g.Update(-1.0)
            st = h.Update(g, M, C, -1.0)
            assert st["converged"] == 1
        gl, ge = g.download()
        assert np.abs(gl - lf_links).max() <= 1e-12 and np.abs(ge - lf_ef).max() <= 1e-13
        gq, ga = h.download()
        assert np.abs(gq - q0).max() <= 200 * TOL and np.abs(ga - a0).max() <= 200 * TOL


@pytest.fixture(scope="module")
def c2_fields(oracle):
    """32^3: the initial condition and the oracle's 1000 leapfrog steps (with
    the one-ulp envelope) at steps 1, 10, 100 and 1000."""
    n = (32, 32, 32)
    links, ef = initial_condition(oracle, n)
    return n, links, ef, leapfrog_with_envelope(oracle, n, links, ef, {1, 10, 100, 1000})


@pytest.mark.parametrize("mass", [1.0, 2.0])
def test_c2_32cubed_thousand_leapfrog_steps_then_cn(oracle, c2_fields, mass):
    n, links, ef, ref = c2_fields
    with lattice_ctx(n, A, cn=(mass, C, 1.0, TOL)):
        g = GaugeConfiguration()
        g.TransversePolarisedOccupiedInit_Box(0.5, 1.0, 0.0, RandomSeed=1, identity_links=True)
        gl, ge = g.download()
        assert np.abs(gl - links).max() < 1e-13 and np.abs(ge - ef).max() < 1e-13
        for s in range(1, 1001):
            g.Update(1.0)
            if s in ref:
                assert_leapfrog_parity(g, ref, s)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        ol, oe = ref[1000][0].copy(), ref[1000][1].copy()
        oq, oa = h.download()
        for s in range(1, 11):
            st = h.Update(g, mass, C, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= TOL
            g.Update(1.0)
            oracle.cn_update(n, A, ol, oe, mass, C, 1.0, oq, oa, tol=1e-14)
            oracle.gauge_update(n, A, ol, oe, 1.0)
            if s in (1, 10):
                gq, ga = h.download()
                assert np.abs(gq - oq).max() <= 2e-12 * s and np.abs(ga - oa).max() <= 2e-12 * s, s
        # each of the 10 solves may move the norm by about its residual
        assert abs(h.GetNorm_Quark() - oracle.heavy_norm(n, oq)) <= 2 * 10 * TOL
        assert abs(h.GetNorm_AntiQ() - oracle.heavy_norm(n, oa)) <= 2 * 10 * TOL
        corr = h.GetMesoncorrelators()
        want = oracle.meson_correlators(n, oq, oa)
        for k, v in want.items():
            assert abs(corr[k] - v) <= 1e-11 * max(1.0, abs(v)), k


@pytest.fixture(scope="module")
def c64(oracle):
    n = (64, 64, 64)
    links, ef = initial_condition(oracle, n)
    for _ in range(3):  # a few steps: links no longer the identity
        oracle.gauge_update(n, A, links, ef, 1.0)
    return n, links, ef


@pytest.mark.parametrize("stencil", [nrqcd.STENCIL_REGISTER, nrqcd.STENCIL_TMA, nrqcd.STENCIL_TENSOR, nrqcd.STENCIL_FMA])
def test_64cubed_operator_every_stencil(oracle, c64, stencil):
    """One A and one A^H application at the headline size: the tensor-core
    stencil runs here with many units per CTA, a regime smaller lattices do
    not reach."""
    n, links, ef = c64
    V = int(np.prod(n))
    rng = np.random.default_rng(11)
    q = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    an = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    M = 1.0
    with lattice_ctx(n, A, cn=(M, C, 1.0, TOL)):
        nrqcd.SetStencil(stencil)
        g = GaugeConfiguration()
        g.upload(links, ef)
        fin, fout = NRQCDField(), NRQCDField()
        fin.upload(q, an)
        for herm in (False, True):
            nrqcd.apply_operator(g, M, C, 1.0, herm, fin, fout)
            oq, oa = fout.download()
            eq = oracle.cn_apply(n, A, links, ef, M, C, 1.0, int(herm), q)
            ea = oracle.cn_apply(n, A, links, ef, -M, C, 1.0, int(herm), an)
            scale = np.abs(q).max()
            assert np.abs(oq - eq).max() < 1e-13 * scale, herm
            assert np.abs(oa - ea).max() < 1e-13 * scale, herm


def test_64cubed_coupled_step(oracle, c64):
    n, links, ef = c64
    M = 1.0
    q, an = oracle.single_point(n, 1), oracle.single_point(n, 1)
    with lattice_ctx(n, A, cn=(M, C, 1.0, 1e-13)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        st = h.Update(g, M, C, 1.0)
        assert st["converged"] == 1
        g.Update(1.0)
        gq, ga = h.download()
        gl, ge = g.download()
    ol, oe = links.copy(), ef.copy()
    oracle.cn_update(n, A, ol, oe, M, C, 1.0, q, an, tol=1e-14)
    oracle.gauge_update(n, A, ol, oe, 1.0)
    assert np.abs(gq - q).max() < 5e-13 and np.abs(ga - an).max() < 5e-13
    assert np.abs(gl - ol).max() < 1e-13 and np.abs(ge - oe).max() < 1e-14
