"""Independent numpy/scipy restatements of the oracle's gluon-distribution
and thermal-initial-condition code, one step each: a Gauss projection sweep
(src/gaugeconfiguration_su3.f90:455-500), a Coulomb gauge-fixing iteration
(:2297-2456, with scipy's expm for ExpAH and numpy's FFT for x2p/p2x) and the
transverse AA/EE correlators (:1825-1972, with scipy's logm for ArgLogU).
The oracle's C code and these restatements share nothing but the
generators."""
import numpy as np
import pytest
import scipy.linalg as sla


@pytest.fixture(scope="module")
def gens(oracle):
    return np.array([oracle.generator(a) for a in range(1, 9)])


def field(oracle, n, a, steps=3, seed=3):
    links, ef = oracle.transverse_box(n, a, 1.0, 1.0, 0.5, seed, identity_links=False)
    for _ in range(steps):
        oracle.gauge_update(n, a, links, ef, 1.0)
    return links, ef


def as_grid(x, n):
    """(V, ...) in site order x + nx (y + ny z) -> (nz, ny, nx, ...)"""
    return x.reshape((n[2], n[1], n[0]) + x.shape[1:])


def links_U(links, n):
    """U[z, y, x, dir] as 3x3 matrices (row, col); the oracle stores [site, dir, col, row]"""
    return as_grid(np.swapaxes(links, 2, 3), n)


def shift(g, d, s):
    """value at x + s e_d on the (nz, ny, nx, ...) grid, d = 0 (x), 1 (y), 2 (z)"""
    return np.roll(g, -s, axis=2 - d)


def algebra(alpha, gens):
    return np.einsum("...a,aij->...ij", alpha, gens)


def coords(M, gens):
    return 2.0 * np.real(np.einsum("aij,...ji->...a", gens, M))


def dag(M):
    return np.conj(np.swapaxes(M, -1, -2))


def gauss_G(U, E, a, gens):
    """G(x) = sum_i (E_i(x) - U_i(x-i)^+ E_i(x-i) U_i(x-i)) / a_i / a0"""
    G = 0
    for i in range(3):
        Em = algebra(E[..., i, :], gens)
        Un, En = shift(U[..., i, :, :], i, -1), shift(Em, i, -1)
        G = G + (Em - dag(Un) @ En @ Un) / a[i + 1]
    return G / a[0]


def test_projection_sweep_matches_numpy(oracle, gens):
    n, a = (4, 3, 5), (0.05, 1.0, 1.2, 0.9)
    links, ef = field(oracle, n, a)
    ef = ef + 0.01 * np.random.default_rng(2).standard_normal(ef.shape)
    U, E = links_U(links, n), as_grid(ef, n)
    G = gauss_G(U, E, a, gens)
    dev = np.max(2.0 * np.abs(np.einsum("aij,...ji->...a", gens, G)))
    assert abs(dev - oracle.gauss_maxnorm(n, a, links, ef)) < 1e-12 * dev
    kdt = 0.01 * a[0]
    En = np.empty_like(E)
    for k in range(3):
        Uk = U[..., k, :, :]
        T = kdt * (Uk @ G @ dag(Uk) @ shift(G, k, +1) - G) + algebra(E[..., k, :], gens)
        En[..., k, :] = coords(T, gens)
    l2, e2 = links.copy(), ef.copy()
    assert oracle.gauss_project(n, a, l2, e2, tol=0.0, max_sweeps=1) == 1
    assert np.abs(as_grid(e2, n) - En).max() < 1e-13 * np.abs(En).max()


def momenta(n, a):
    """backward-derivative |p| on the (nz, ny, nx) grid and the components"""
    comps = []
    for d in range(3):
        k = np.arange(n[d])
        ph = np.pi * k / n[d]
        comps.append(2 * np.sin(ph) / a[d + 1] * np.exp(-1j * ph))
    pz, py, px = np.meshgrid(comps[2], comps[1], comps[0], indexing="ij")
    p = np.stack([px, py, pz], axis=-1)
    return np.sqrt(np.sum(np.abs(p) ** 2, axis=-1)), p


def test_gaugefix_iteration_matches_numpy(oracle, gens):
    n, a = (4, 6, 5), (0.05, 1.0, 1.0, 1.1)
    links, ef = field(oracle, n, a)
    U = links_U(links, n)
    D = 0
    for i in range(3):
        d = -U[..., i, :, :] + shift(U[..., i, :, :], i, -1)
        D = D + (d - dag(d)) / 2
    pn, _ = momenta(n, a)
    pmax = pn.max()
    f = np.where(pn > 1e-12, (pmax / np.where(pn > 1e-12, pn, 1.0)) ** 2, 1.0)
    Dp = np.fft.fftn(D, axes=(0, 1, 2)) * f[..., None, None]
    Ds = 0.08 * np.fft.ifftn(Dp, axes=(0, 1, 2))
    Gt = np.array([sla.expm(m) for m in Ds.reshape(-1, 3, 3)]).reshape(Ds.shape)
    Un = np.empty_like(U)
    for i in range(3):
        Un[..., i, :, :] = Gt @ U[..., i, :, :] @ dag(shift(Gt, i, +1))
    l2 = links.copy()
    it, dev = oracle.coulomb_gaugefix(n, a, l2, tol=0.0, alpha=0.08, max_iterations=1)
    assert it == 2 and abs(dev[0] - np.max(np.sqrt(np.sum(np.abs(D) ** 2, axis=(-1, -2))) / 9)) < 1e-14
    assert np.abs(links_U(l2, n) - Un).max() < 1e-12


def test_transverse_correlators_match_numpy(oracle, gens):
    n, a = (4, 6, 5), (0.05, 1.0, 1.0, 1.1)
    links, ef = field(oracle, n, a, steps=5)
    U, E = links_U(links, n), as_grid(ef, n)
    V = int(np.prod(n))
    fwd = a[1] * a[2] * a[3]
    vol = V * fwd
    pn, p = momenta(n, a)
    P = (np.eye(3) - np.conj(p)[..., :, None] * p[..., None, :] / np.where(pn > 1e-12, pn, 1.0)[..., None, None] ** 2) / 2
    P = np.where((pn < 1e-12)[..., None, None], 0.0, np.real(P))
    out = []
    for kind in ("A", "E"):
        acc = 0
        for aa in range(8):
            f = np.empty(tuple(reversed(n)) + (3,), dtype=complex)
            for i in range(3):
                if kind == "A":
                    H = np.array([-1j * sla.logm(u) for u in U[..., i, :, :].reshape(-1, 3, 3)]).reshape(U.shape[:3] + (3, 3))
                    val = coords(H, gens)[..., aa] / a[i + 1]
                else:
                    val = E[..., i, aa] / a[i + 1] / a[0]
                f[..., i] = np.fft.fftn(val, axes=(0, 1, 2)) * fwd
            res = np.real(np.einsum("...i,...ij,...j->...", f, P, np.conj(f)))
            acc = acc + (res / vol) / 8
        out.append(acc.reshape(-1))
    aa_ref, ee_ref, mom = oracle.transverse_correlators(n, a, links, ef)
    assert np.abs(mom - pn.reshape(-1)).max() < 1e-13
    assert np.abs(aa_ref - out[0]).max() < 1e-10 * np.abs(out[0]).max()
    assert np.abs(ee_ref - out[1]).max() < 1e-12 * np.abs(out[1]).max()
