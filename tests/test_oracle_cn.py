"""Oracle checks of the Crank-Nicolson step (src/nrqcd.f90:1053-1387)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["free_kat_8x8x8_M1", "free_kat_6x4x10_M2"])
def test_free_propagation_known_answer(oracle, name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    n, a, M = tuple(g["n"]), tuple(g["a"]), float(g["mass"])
    links, ef = oracle.cold(n, a)
    q = oracle.single_point(n, 1)
    an = oracle.single_point(n, 1)
    for s in range(int(g["nsteps"])):
        st = oracle.cn_update(n, a, links, ef, M, [1, 1, 1, 1], 1.0, q, an, tol=1e-14)
        assert st.converged
        eye = np.eye(6)
        assert np.abs(q - g["amp_q"][s][:, None, None] * eye).max() < 1e-13
        assert np.abs(an - g["amp_a"][s][:, None, None] * eye).max() < 1e-13
        corr = oracle.meson_correlators(n, q, an)
        assert abs(corr["o1_1s0"] - g["o1_1s0"][s]) < 1e-13
        assert abs(oracle.heavy_norm(n, q) - 1) < 1e-13


@pytest.fixture(scope="module")
def hot(oracle):
    n, a = (6, 6, 6), (0.05, 1.0, 1.0, 1.0)
    links, ef = oracle.transverse_box(n, a, 3.0, 1.0, 0.0, 5, identity_links=False)
    return n, a, links, ef


def test_operator_adjoint_and_hermitian_parts(oracle, hot):
    n, a, links, ef = hot
    V = int(np.prod(n))
    rng = np.random.default_rng(1)
    u = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    v = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    c = [1, 1, 1, 1]
    Av = oracle.cn_apply(n, a, links, ef, 1.0, c, 1.0, 0, v)
    AHu = oracle.cn_apply(n, a, links, ef, 1.0, c, 1.0, 1, u)
    assert abs(np.vdot(u, Av) - np.vdot(AHu, v)) < 1e-12 * np.abs(np.vdot(u, Av))
    # real Wilson coefficients: A = 1 - i tau H, A^H = 1 + i tau H with H hermitian
    AHv = oracle.cn_apply(n, a, links, ef, 1.0, c, 1.0, 1, v)
    assert np.abs(Av + AHv - 2 * v).max() < 1e-14
    # the block transposition of the PETSc assembly changes the operator
    Av_src = oracle.cn_apply(n, a, links, ef, 1.0, c, 1.0, 0, v, transpose_blocks=False)
    assert np.abs(Av - Av_src).max() > 1e-3


def test_cn_unitary_and_reversible(oracle, hot):
    n, a, links, ef = hot
    q = oracle.single_point(n, 1)
    an = oracle.single_point(n, 1)
    q0, a0 = q.copy(), an.copy()
    for _ in range(3):
        st = oracle.cn_update(n, a, links, ef, 1.0, [1, 1, 1, 1], 1.0, q, an, tol=1e-14)
        assert st.converged and max(st.rel_residual) < 1e-14
    assert abs(oracle.heavy_norm(n, q) - 1) < 1e-13 and abs(oracle.heavy_norm(n, an) - 1) < 1e-13
    for _ in range(3):
        oracle.cn_update(n, a, links, ef, 1.0, [1, 1, 1, 1], -1.0, q, an, tol=1e-14)
    assert np.abs(q - q0).max() < 1e-13 and np.abs(an - a0).max() < 1e-13
