"""Oracle checks of the SU(3) layer (src/su3.f90, src/matrixoperations.f90)."""
import numpy as np
import pytest
import scipy.linalg as sl


def test_generators_are_the_reference_arrays(oracle):
    T = [oracle.generator(a) for a in range(1, 9)]
    G = np.array([[np.trace(Ta @ Tb) for Tb in T] for Ta in T])
    assert np.allclose(G, 0.5 * np.eye(8), atol=1e-15)
    for t in T:
        assert np.allclose(t, t.conj().T) and abs(np.trace(t)) < 1e-15
    # column-major reshape in su3.f90:97-131 puts -i/2 at (2,1): T2 = -lambda2/2
    assert T[1][1, 0] == -0.5j and T[1][0, 1] == 0.5j
    assert T[4][2, 0] == -0.5j and T[6][2, 1] == -0.5j


@pytest.mark.parametrize("scale", [0.01, 0.3, 2.5])
def test_group_exp_matches_expm(oracle, scale):
    rng = np.random.default_rng(int(scale * 100))
    T = [oracle.generator(a) for a in range(1, 9)]
    for _ in range(5):
        al = rng.normal(size=8) * scale
        M = sum(x * t for x, t in zip(al, T))
        G = oracle.group_exp(al)
        assert np.abs(G - sl.expm(1j * M)).max() < 2e-15 * max(1, scale * 4)
        assert np.abs(G @ G.conj().T - np.eye(3)).max() < 2e-15


def test_logu_inverts_exp(oracle):
    rng = np.random.default_rng(3)
    T = [oracle.generator(a) for a in range(1, 9)]
    for _ in range(10):
        al = rng.normal(size=8) * 0.5
        M = sum(x * t for x, t in zip(al, T))
        L = oracle.logu(oracle.group_exp(al))
        assert np.abs(L - 1j * M).max() < 5e-15


def test_eigen_solvers(oracle):
    rng = np.random.default_rng(5)
    A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    H = A + A.conj().T
    d, U = oracle.eigenh(H)
    assert np.abs(U @ H @ U.conj().T - np.diag(d)).max() < 1e-14
    Q, _ = np.linalg.qr(A)
    dc, S = oracle.eigenc(Q)
    assert np.abs(S @ Q - np.diag(dc) @ S).max() < 1e-14
    # degenerate input (identity) converges immediately
    d1, U1 = oracle.eigenh(np.eye(3, dtype=complex))
    assert np.allclose(d1, 1) and np.allclose(U1, np.eye(3))
