"""GPU parity of the Crank-Nicolson hot path against the oracle (through the C ABI).

Tolerances: the matvec is FP64 against the FP64 oracle (1e-13 relative).
Solves run to kspTol = 1e-13 on both sides; the propagators then agree to a
few 1e-13 absolute (point-source amplitude 1/sqrt 6)."""
import os

import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField, NrqcdError, nrqcd
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def hot(oracle, n, seed=5, Q=3.0):
    return oracle.transverse_box(n, A, Q, 1.0, 0.0, seed, identity_links=False)


@pytest.mark.parametrize("herm", [False, True])
@pytest.mark.parametrize("n", [(4, 4, 4), (6, 5, 7)])
def test_operator_matches_oracle(oracle, herm, n):
    links, ef = hot(oracle, n)
    V = int(np.prod(n))
    rng = np.random.default_rng(3)
    q = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    an = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    M, c, dt = 1.3, [1.0, 0.9 + 0.1j, 1.1, 0.8 - 0.2j], 1.0
    with lattice_ctx(n, A, cn=(M, c, dt, 1e-12)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        fin, fout = NRQCDField(), NRQCDField()
        fin.upload(q, an)
        nrqcd.apply_operator(g, M, c, dt, herm, fin, fout)
        oq, oa = fout.download()
    eq = oracle.cn_apply(n, A, links, ef, M, c, dt, int(herm), q)
    ea = oracle.cn_apply(n, A, links, ef, -M, np.conj(c), dt, int(herm), an)
    scale = np.abs(q).max()
    assert np.abs(oq - eq).max() < 1e-13 * scale
    assert np.abs(oa - ea).max() < 1e-13 * scale


@pytest.mark.parametrize("name", ["free_kat_8x8x8_M1", "free_kat_6x4x10_M2"])
def test_free_known_answer_on_gpu(name):
    g0 = np.load(os.path.join(GOLD, name + ".npz"))
    n, a, M = tuple(int(v) for v in g0["n"]), tuple(float(v) for v in g0["a"]), float(g0["mass"])
    with lattice_ctx(n, a, cn=(M, [1, 1, 1, 1], 1.0, 1e-14)):
        g = GaugeConfiguration()
        g.ColdInit()
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        for s in range(int(g0["nsteps"])):
            st = h.Update(g, M, [1, 1, 1, 1], 1.0)
            assert st["converged"] == 1
            q, an = h.download()
            eye = np.eye(6)
            assert np.abs(q - g0["amp_q"][s][:, None, None] * eye).max() < 1e-13
            assert np.abs(an - g0["amp_a"][s][:, None, None] * eye).max() < 1e-13
            assert abs(h.GetMesoncorrelator_O1_1S0_ZeroMomentum() - g0["o1_1s0"][s]) < 1e-13
            assert abs(h.GetNorm_Quark() - 1) < 1e-13 and abs(h.GetNorm_AntiQ() - 1) < 1e-13


@pytest.mark.parametrize("n", [(6, 6, 6), (8, 4, 6)])
def test_cn_step_matches_oracle(oracle, n):
    links, ef = hot(oracle, n)
    M, c = 1.0, [1, 1, 1, 1]
    q = oracle.single_point(n, 1)
    an = oracle.single_point(n, 1)
    with lattice_ctx(n, A, cn=(M, c, 1.0, 1e-13)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        for _ in range(3):
            st = h.Update(g, M, c, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] < 1e-13
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
        gq, ga = h.download()
        nq, na = h.GetNorm_Quark(), h.GetNorm_AntiQ()
        corr = h.GetMesoncorrelators()
    assert np.abs(gq - q).max() < 5e-13 and np.abs(ga - an).max() < 5e-13
    assert abs(nq - 1) < 1e-12 and abs(na - 1) < 1e-12
    oc = oracle.meson_correlators(n, q, an)
    for k in oc:
        assert abs(corr[k] - oc[k]) < 1e-12, k


def test_correlators_random_fields(oracle):
    n = (4, 4, 4)
    V = 64
    rng = np.random.default_rng(8)
    q = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    an = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    with lattice_ctx(n, A):
        h = NRQCDField()
        h.upload(q, an)
        corr = h.GetMesoncorrelators()
        nq = h.GetNorm_Quark()
    oc = oracle.meson_correlators(n, q, an)
    for k in oc:
        assert abs(corr[k] - oc[k]) < 1e-11 * max(1, abs(oc[k])), k
    assert abs(nq - oracle.heavy_norm(n, q)) < 1e-12 * nq


def test_gconjg_correlators_random_fields(oracle):
    """The _gconjg correlators (src/nrqcd.f90:1728-1905) on random
    propagators: conj(A) instead of A^+ in every product, so they differ
    from the plain ones on non-symmetric A."""
    n = (5, 4, 3)
    V = 60
    rng = np.random.default_rng(9)
    q = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    an = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    with lattice_ctx(n, A):
        h = NRQCDField()
        h.upload(q, an)
        corr = h.GetMesoncorrelators_gconjg()
        one = h.GetMesoncorrelator_O8_3S1_ZeroMomentum_gconjg()
        plain = h.GetMesoncorrelators()
    oc = oracle.meson_correlators_gconjg(n, q, an)
    for k in oc:
        assert abs(corr[k] - oc[k]) < 1e-11 * max(1, abs(oc[k])), k
        assert abs(corr[k] - plain[k]) > 1e-3 * max(1, abs(oc[k])), k
    assert one == corr["o8_3s1"]


def test_forward_backward_returns_initial_propagator(oracle):
    n = (8, 8, 8)
    links, ef = hot(oracle, n, seed=4, Q=2.0)
    with lattice_ctx(n, A, cn=(1.0, [1, 1, 1, 1], 1.0, 1e-14)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        q0, a0 = h.download()
        for _ in range(4):
            h.Update(g, 1.0, [1, 1, 1, 1], 1.0)
        for _ in range(4):
            h.Update(g, 1.0, [1, 1, 1, 1], -1.0)
        q, an = h.download()
    assert np.abs(q - q0).max() < 1e-12 and np.abs(an - a0).max() < 1e-12


def test_coupled_step_matches_oracle(oracle):
    """Driver order of src/main.f90:344-348: CN step, then leapfrog."""
    n = (8, 8, 8)
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 1, identity_links=True)
    M, c = 1.0, [1, 1, 1, 1]
    q = oracle.single_point(n, 1)
    an = oracle.single_point(n, 1)
    with lattice_ctx(n, A, cn=(M, c, 1.0, 1e-13)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        for _ in range(5):
            h.Update(g, M, c)
            g.Update()
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
            oracle.gauge_update(n, A, links, ef, 1.0)
        gq, ga = h.download()
        lg, eg = g.download()
    assert np.abs(lg - links).max() < 1e-13 and np.abs(eg - ef).max() < 1e-13
    assert np.abs(gq - q).max() < 5e-13 and np.abs(ga - an).max() < 5e-13


def test_errors_fail_loudly():
    from nrqcd_b200 import NrqcdError
    n = (4, 4, 4)
    with lattice_ctx(n, A, cn=(1.0, [1, 1, 1, 1], 1.0, 1e-12)):
        h = NRQCDField()
        with pytest.raises(NrqcdError):
            h.InitSinglePoint(0, 1)
        with pytest.raises(NrqcdError):
            nrqcd.InitModule(1.0, [1, 1, 1, 1], 1.0, 1e-12)


@pytest.mark.parametrize("tol", [1e-10, 1e-12])
def test_history_start_and_half_step_exit(oracle, tol):
    """The plain solve's start extrapolated from the field's last
    corrections (the default, up to four) and the half-step exit: over coupled steps on
    an evolving 16^3 field it starts at a smaller residual and needs fewer
    stencil launches than the start 2b - psi alone, ends at the same
    tolerance, and both evolutions agree to the tolerance's level (both
    confirm every solve with the true residual, so that the launch counts
    differ by the start alone)."""
    from nrqcd_b200 import nrqcd
    n = (16, 16, 16)
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 4, identity_links=False)
    M, c = 1.0, [1, 1, 1, 1]
    runs = {}
    for hist in (True, False):
        with lattice_ctx(n, A, cn=(M, c, 1.0, tol)):
            nrqcd.SetHistoryGuess(hist)
            nrqcd.SetTrueResidual(True)
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(1, 1)
            stats = []
            for _ in range(6):
                stats.append(h.Update(g, M, c, 1.0))
                g.Update(1.0)
            q, a = h.download()
            del g, h
        for st in stats:
            assert st["converged"] == 1 and st["max_rel_residual"] <= tol
        runs[hist] = (q, a, stats)
    late_h, late_p = runs[True][2][3:], runs[False][2][3:]
    assert all(x["initial_rel_residual"] < 0.2 * y["initial_rel_residual"] for x, y in zip(late_h, late_p))
    assert sum(x["matvecs"] for x in late_h) < sum(y["matvecs"] for y in late_p)
    assert np.abs(runs[True][0] - runs[False][0]).max() < 50 * tol
    assert np.abs(runs[True][1] - runs[False][1]).max() < 50 * tol


def _true_rel_residuals(oracle, n, links, ef, M, c, old, new):
    """max over the 12 columns of ||A psi_old - A^H psi_new|| / ||A psi_old||,
    quark (M, c) and antiquark (-M, conj c), from the oracle's operator; a
    column is the site-major slice [:, col, :] (src/nrqcd.f90:1106-1124)."""
    out = []
    for k, (m, cc) in enumerate(((M, c), (-M, np.conj(c)))):
        rhs = oracle.cn_apply(n, A, links, ef, m, cc, 1.0, 0, old[k])
        lhs = oracle.cn_apply(n, A, links, ef, m, cc, 1.0, 1, new[k])
        for col in range(6):
            out.append(np.linalg.norm(rhs[:, col] - lhs[:, col]) / np.linalg.norm(rhs[:, col]))
    return max(out)


@pytest.mark.parametrize("tol", [1e-10, 1e-12])
def test_recursive_residual_acceptance(oracle, tol):
    """The plain solve accepts BiCGStab's recursive residual where it meets
    the tolerance with a margin measured on its confirmed solves: the true
    residual of each accepted update, recomputed by the oracle from the
    downloaded fields, is still within the tolerance; the always-confirm
    mode agrees with it, and the recursive acceptance saves stencil
    launches."""
    n = (16, 16, 16)
    M, c = 1.0, np.array([1, 1, 1, 1], dtype=complex)
    runs = {}
    for always in (False, True):
        with lattice_ctx(n, A, cn=(M, list(c), 1.0, tol)):
            nrqcd.SetTrueResidual(always)
            links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 4, identity_links=False)
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(1, 1)
            mv, recursive = 0, 0
            for _ in range(6):
                old = h.download()
                gl, ge = g.download()
                st = h.Update(g, M, list(c), 1.0)
                assert st["converged"] == 1 and st["max_rel_residual"] <= tol
                true_res = nrqcd.LastResidualIsTrue()
                if always:
                    assert true_res
                if not true_res:
                    recursive += 1
                new = h.download()
                assert _true_rel_residuals(oracle, n, gl, ge, M, c, old, new) <= tol
                mv += st["matvecs"]
                g.Update(1.0)
            q, a = h.download()
            del g, h
        runs[always] = (q, a, mv, recursive)
    assert runs[True][3] == 0
    assert runs[False][3] > 0
    assert runs[False][2] < runs[True][2]
    assert np.abs(runs[True][0] - runs[False][0]).max() < 50 * tol
    assert np.abs(runs[True][1] - runs[False][1]).max() < 50 * tol


@pytest.mark.parametrize("n", [(16, 16, 16), (12, 10, 8)])
def test_merged_update_matches_two_pass(oracle, n):
    """The FMA stencil's merged BiCGStab update (beta from the rh.t that the
    t = A^H s launch reduces; x, r and p in one pass) against the two-pass
    update (rho_new = rh.r reduced after r is formed): over coupled steps of
    an evolving field both converge (confirmed by the true residual) in the
    same number of iterations within one, and the evolutions agree to the
    tolerance's level."""
    tol = 1e-12
    M, c = 1.0, [1, 1, 1, 1]
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 4, identity_links=False)
    runs = {}
    for merged in (True, False):
        with lattice_ctx(n, A, cn=(M, c, 1.0, tol)):
            nrqcd.SetStencil(nrqcd.STENCIL_FMA)
            nrqcd.SetMergedUpdate(merged)
            nrqcd.SetTrueResidual(True)
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(1, 1)
            its = []
            for _ in range(5):
                st = h.Update(g, M, c, 1.0)
                assert st["converged"] == 1 and st["max_rel_residual"] <= tol
                its.append(st["iterations"])
                g.Update(1.0)
            assert nrqcd.StencilInfo()[0] == nrqcd.STENCIL_FMA
            q, a = h.download()
            del g, h
        runs[merged] = (q, a, its)
    assert all(abs(x - y) <= 1 for x, y in zip(runs[True][2], runs[False][2]))
    assert np.abs(runs[True][0] - runs[False][0]).max() < 50 * tol
    assert np.abs(runs[True][1] - runs[False][1]).max() < 50 * tol


def test_history_depth_lowers_the_start(oracle):
    """The extrapolated start of degree depth - 1: over coupled steps on an
    evolving 16^3 field, once the history is full each deeper extrapolation
    starts lower (the field's t vary smoothly from step to step), every
    update converges, and the evolutions agree to the tolerance's level."""
    n = (16, 16, 16)
    tol = 1e-12
    M, c = 1.0, [1, 1, 1, 1]
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 4, identity_links=False)
    runs = {}
    for depth in (2, 3, 4):
        with lattice_ctx(n, A, cn=(M, c, 1.0, tol)):
            nrqcd.SetHistoryDepth(depth)
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(1, 1)
            init = []
            for _ in range(8):
                st = h.Update(g, M, c, 1.0)
                assert st["converged"] == 1 and st["max_rel_residual"] <= tol
                init.append(st["initial_rel_residual"])
                g.Update(1.0)
            q, a = h.download()
            del g, h
        runs[depth] = (q, a, init)
    for lo, hi in ((3, 2), (4, 3)):
        assert all(x < 0.6 * y for x, y in zip(runs[lo][2][5:], runs[hi][2][5:]))
    for d in (3, 4):
        assert np.abs(runs[d][0] - runs[2][0]).max() < 50 * tol
        assert np.abs(runs[d][1] - runs[2][1]).max() < 50 * tol
    with lattice_ctx(n, A, cn=(M, c, 1.0, tol)):
        for bad in (0, 5):
            with pytest.raises(NrqcdError):
                nrqcd.SetHistoryDepth(bad)
