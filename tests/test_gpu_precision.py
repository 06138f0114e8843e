"""GPU checks of the precision form of the Crank-Nicolson solve (FP32
Chebyshev inner iterations, FP64 iterative refinement) against the FP64
oracle.  The form is specified at an outer residual <= 1e-10; the tests use
the tolerances written below."""
import os

import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
GOLD = os.path.join(os.path.dirname(__file__), "golden")
FORM_PRECISION = 1


@pytest.mark.parametrize("name", ["free_kat_8x8x8_M1", "free_kat_6x4x10_M2"])
def test_precision_form_free_known_answer(name):
    g0 = np.load(os.path.join(GOLD, name + ".npz"))
    n, a, M = tuple(int(v) for v in g0["n"]), tuple(float(v) for v in g0["a"]), float(g0["mass"])
    with lattice_ctx(n, a, cn=(M, [1, 1, 1, 1], 1.0, 1e-11, 10000, FORM_PRECISION)):
        g = GaugeConfiguration()
        g.ColdInit()
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        for s in range(int(g0["nsteps"])):
            st = h.Update(g, M, [1, 1, 1, 1], 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-11
            q, an = h.download()
            eye = np.eye(6)
            assert np.abs(q - g0["amp_q"][s][:, None, None] * eye).max() < 1e-11
            assert np.abs(an - g0["amp_a"][s][:, None, None] * eye).max() < 1e-11


@pytest.mark.parametrize("n", [(6, 6, 6), (8, 8, 8), (5, 5, 5)])
def test_precision_form_matches_fp64_oracle(oracle, n):
    links, ef = oracle.transverse_box(n, A, 3.0 if n[0] == 6 else 2.0, 1.0, 0.0, 5, identity_links=False)
    M, c = 1.0, [1, 1, 1, 1]
    q = oracle.single_point(n, 1)
    an = oracle.single_point(n, 1)
    with lattice_ctx(n, A, cn=(M, c, 1.0, 1e-10, 10000, FORM_PRECISION)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        for _ in range(3):
            st = h.Update(g, M, c, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
        gq, ga = h.download()
        nq, na = h.GetNorm_Quark(), h.GetNorm_AntiQ()
    # residual 1e-10 per step on a unit-norm field: propagators agree to ~1e-10
    assert np.abs(gq - q).max() < 3e-10 and np.abs(ga - an).max() < 3e-10
    assert abs(nq - 1) < 1e-9 and abs(na - 1) < 1e-9


def test_precision_form_reversible(oracle):
    n = (8, 8, 8)
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 4, identity_links=False)
    with lattice_ctx(n, A, cn=(1.0, [1, 1, 1, 1], 1.0, 1e-11, 10000, FORM_PRECISION)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        q0, a0 = h.download()
        for _ in range(3):
            h.Update(g, 1.0, [1, 1, 1, 1], 1.0)
        for _ in range(3):
            h.Update(g, 1.0, [1, 1, 1, 1], -1.0)
        q, an = h.download()
    assert np.abs(q - q0).max() < 1e-10 and np.abs(an - a0).max() < 1e-10


def test_fp32_leapfrog_tracks_fp64_and_reunitarises(oracle):
    """Precision form of the leapfrog (FP32 links, FP64 reunitarisation
    every 10 steps) against the FP64 oracle on a hot 10^3 field."""
    n = (10, 10, 10)
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 6, identity_links=False)
    l0, e0 = links.copy(), ef.copy()
    e_ref0 = oracle.energy(n, A, links, ef)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        g.SetPrecision(1, 10)
        dev = []
        for step in range(1, 26):
            g.Update(1.0)
            oracle.gauge_update(n, A, links, ef, 1.0)
            if step in (20, 25):
                dev.append(g.GetUnitarityDeviation())
        gl, ge = g.download()
        en = g.GetEnergy()
        gref, gmax = g._gauss()
        g.SetPrecision(0)
    # 25 steps: the FP32 rounding of the links propagates at ~1e-7 per step
    assert np.abs(gl - links).max() < 2e-5 and np.abs(ge - ef).max() < 2e-5
    e_ref = oracle.energy(n, A, links, ef)
    assert abs(en - e_ref) <= 1e-5 * abs(e_ref)
    assert abs(e_ref - e_ref0) <= 1e-3 * abs(e_ref0)  # the FP64 leapfrog's own drift, for scale
    assert abs(gmax - oracle.gauss_maxnorm(n, A, links, ef)) < 1e-4
    # right after the reunitarisation (step 20) the links are unitary to FP64
    # rounding; five FP32 steps later to FP32 rounding
    assert dev[0][0] < 1e-13 and dev[0][1] < 1e-13
    assert dev[1][0] < 1e-5 and dev[1][1] < 1e-5
    del l0, e0


@pytest.mark.parametrize("n0", [0.5, 1.0, 2.0])
def test_precision_form_drift_against_fp64_oracle(oracle, n0):
    """Coupled steps of the whole precision form (FP32-link leapfrog, FP32
    Chebyshev CN with FP64 refinement at 1e-10) against the FP64 oracle (GMRES
    to 1e-14, FP64 leapfrog): the drift of every observable stays small."""
    n = (8, 8, 8)
    M, c = 1.0, [1, 1, 1, 1]
    links, ef = oracle.transverse_box(n, A, 0.5, n0, 0.0, 2, identity_links=True)
    q = oracle.single_point(n, 1)
    an = oracle.single_point(n, 1)
    with lattice_ctx(n, A, cn=(M, c, 1.0, 1e-10, 10000, FORM_PRECISION)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        g.SetPrecision(1, 10)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        for _ in range(12):
            st = h.Update(g, M, c, 1.0)
            assert st["converged"] == 1
            g.Update(1.0)
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
            oracle.gauge_update(n, A, links, ef, 1.0)
        gq, ga = h.download()
        en = g.GetEnergy()
        nq, na = h.GetNorm_Quark(), h.GetNorm_AntiQ()
    e_ref = oracle.energy(n, A, links, ef)
    assert abs(en - e_ref) <= 1e-5 * max(abs(e_ref), 1e-12)
    assert np.abs(gq - q).max() < 1e-6 and np.abs(ga - an).max() < 1e-6
    assert abs(nq - 1) < 1e-9 and abs(na - 1) < 1e-9


@pytest.mark.parametrize("n", [(6, 6, 6), (36, 4, 4), (40, 6, 4), (64, 4, 4), (16, 16, 16)])
@pytest.mark.parametrize("cheb", ["register", "blocks"])
def test_precision_form_chebyshev_steps(oracle, n, cheb):
    """Both FP32 Chebyshev steps (operator assembled per launch; FP32 blocks
    staged by TMA) against the FP64 oracle at outer residual 1e-10.  The
    lattices cover rows shorter than a tile, rows long enough for the x-wrap
    columns (36), units spanning rows (40 x 6) and several units per row."""
    from nrqcd_b200 import nrqcd
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 7, identity_links=False)
    M, c = 1.0, [1, 1, 1, 1]
    q = oracle.single_point(n, 3)
    an = oracle.single_point(n, 3)
    want = nrqcd.CHEB_BLOCKS if cheb == "blocks" else nrqcd.CHEB_REGISTER
    with lattice_ctx(n, A, cn=(M, c, 1.0, 1e-10, 10000, FORM_PRECISION)):
        nrqcd.SetChebStencil(want)
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(3, 3)
        for _ in range(3):
            st = h.Update(g, M, c, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
        assert nrqcd.ChebInfo() == want
        gq, ga = h.download()
    assert np.abs(gq - q).max() < 3e-10 and np.abs(ga - an).max() < 3e-10


def test_chebyshev_blocks_need_even_rows():
    """nx odd: the default runs the per-launch step, forcing the block step
    is refused."""
    from nrqcd_b200 import NrqcdError, nrqcd
    with lattice_ctx((5, 4, 4), A, cn=(1.0, [1, 1, 1, 1], 1.0, 1e-10, 10000, FORM_PRECISION)):
        with pytest.raises(NrqcdError):
            nrqcd.SetChebStencil(nrqcd.CHEB_BLOCKS)
        g = GaugeConfiguration()
        g.ColdInit()
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        assert h.Update(g, 1.0, [1, 1, 1, 1], 1.0)["converged"] == 1
        assert nrqcd.ChebInfo() == nrqcd.CHEB_REGISTER


def test_chebyshev_step_timed_choice():
    """By default the first update times both FP32 steps and runs the faster."""
    from nrqcd_b200 import nrqcd
    n = (16, 16, 16)
    with lattice_ctx(n, A, cn=(1.0, [1, 1, 1, 1], 1.0, 1e-10, 10000, FORM_PRECISION)):
        g = GaugeConfiguration()
        g.ColdInit()
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        assert h.Update(g, 1.0, [1, 1, 1, 1], 1.0)["converged"] == 1
        last, ms = nrqcd.ChebInfo(with_times=True)
    assert (ms > 0).all() and last == int(np.argmin(ms))


@pytest.mark.parametrize("tol", [1e-10, 1e-12])
def test_precision_form_prediction_acceptance(oracle, tol):
    """The precision form ends an update on the Chebyshev prediction of its
    last pass (previous residual over the pass's guaranteed gain, scaled by
    the true-to-predicted ratio its confirmed passes measured) where that
    meets the tolerance: the true residual of every update, recomputed by the
    oracle from the downloaded fields, is within the tolerance, some updates
    end on the prediction, and the always-confirm mode agrees with it."""
    from nrqcd_b200 import nrqcd
    from tests.test_gpu_cn import _true_rel_residuals
    n = (16, 16, 16)
    M, c = 1.0, np.array([1, 1, 1, 1], dtype=complex)
    runs = {}
    for always in (False, True):
        with lattice_ctx(n, A, cn=(M, list(c), 1.0, tol, 10000, FORM_PRECISION)):
            nrqcd.SetTrueResidual(always)
            links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 4, identity_links=False)
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(1, 1)
            predicted, mv = 0, 0
            for _ in range(6):
                old = h.download()
                gl, ge = g.download()
                st = h.Update(g, M, list(c), 1.0)
                assert st["converged"] == 1 and st["max_rel_residual"] <= tol
                if not nrqcd.LastResidualIsTrue():
                    predicted += 1
                assert _true_rel_residuals(oracle, n, gl, ge, M, c, old, h.download()) <= tol
                mv += st["matvecs"]
                g.Update(1.0)
            q, a = h.download()
            del g, h
        runs[always] = (q, a, predicted, mv)
    assert runs[True][2] == 0
    assert runs[False][2] > 0 and runs[False][3] < runs[True][3]
    assert np.abs(runs[True][0] - runs[False][0]).max() < 50 * tol
    assert np.abs(runs[True][1] - runs[False][1]).max() < 50 * tol
