"""CPU restatement of the plain solve's algebra on the oracle's operator (no
GPU): the merged BiCGStab update with the FP32 shadow residual follows the
classic recurrence to rounding, and the history start's coefficients are
the polynomial extrapolation they are meant to be.

The merged update takes beta from rh.t before r is formed: alpha = rho /
(rh.v) makes rh.s = 0, so rho_new = rh.(s - omega t) = -omega rh.t and
beta = (rho_new / rho)(alpha / omega) = -alpha (rh.t) / rho.  The shadow
residual rh may be any fixed vector with rh.r0 != 0; the FP32-rounded r0
serves when rho_0 is taken against the same rounded values."""
import numpy as np
import pytest

A = (0.05, 1.0, 1.0, 1.0)
C = np.array([1, 1, 1, 1], dtype=complex)


def _dot(a, b):
    return np.einsum("scr,scr->c", np.conj(a), b)


def _nrm(a):
    return np.sqrt(np.real(_dot(a, a)))


def _problem(oracle, n=(6, 6, 6), seed=3):
    links, ef = oracle.transverse_box(n, A, 3.0, 1.0, 0.0, 5, identity_links=False)
    rng = np.random.default_rng(seed)
    V = int(np.prod(n))
    psi = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    b = oracle.cn_apply(n, A, links, ef, 1.0, C, 1.0, 0, psi)  # b = A psi
    return (lambda p: oracle.cn_apply(n, A, links, ef, 1.0, C, 1.0, 1, np.ascontiguousarray(p))), b, psi


def _bicgstab(apply, b, x0, tol, merged, maxit=50):
    """Per-column BiCGStab on apply(x) = b; merged: the one-pass update with
    the FP32 shadow.  Returns x, iterations and the largest |rh.s| seen
    relative to |rh| |r0| (the recurrence for rho carries rounding of that
    size from the start on, so relative to the current |r| it grows as the
    residual falls, which costs the merged beta accuracy near the end but
    not the solution's)."""
    bn = _nrm(b)
    x = x0.copy()
    r = b - apply(x)
    if merged:
        rh = r.astype(np.complex64).astype(np.complex128)
    else:
        rh = r.copy()
    rho = _dot(rh, r)
    p = r.copy()
    scale0 = _nrm(rh) * _nrm(r)
    worst = 0.0
    for it in range(1, maxit + 1):
        v = apply(p)
        al = rho / _dot(rh, v)
        s = r - al[None, :, None] * v
        worst = max(worst, float((np.abs(_dot(rh, s)) / scale0).max()))
        t = apply(s)
        om = _dot(t, s) / np.real(_dot(t, t))
        x = x + al[None, :, None] * p + om[None, :, None] * s
        if merged:
            rht = _dot(rh, t)
            be = -al * rht / rho
            rho = -om * rht
            r = s - om[None, :, None] * t
            p = r + be[None, :, None] * (p - om[None, :, None] * v)
        else:
            r = s - om[None, :, None] * t
            rn = _dot(rh, r)
            be = (rn / rho) * (al / om)
            rho = rn
            p = r + be[None, :, None] * (p - om[None, :, None] * v)
        if np.all(_nrm(r) <= tol * bn):
            return x, it, worst
    return x, maxit, worst


@pytest.mark.parametrize("tol", [1e-10, 1e-12])
def test_merged_update_follows_classic_bicgstab(oracle, tol):
    apply, b, psi = _problem(oracle)
    x0 = 2 * b - psi
    xc, itc, _ = _bicgstab(apply, b, x0, tol, merged=False)
    xm, itm, worst = _bicgstab(apply, b, x0, tol, merged=True)
    assert abs(itm - itc) <= 1
    # rh.s vanishes to rounding of the start's scale, which the merged beta
    # relies on
    assert worst < 1e-13
    bn = _nrm(b)
    assert (_nrm(b - apply(xm)) / bn).max() <= 1.01 * tol
    scale = np.abs(xc).max()
    assert np.abs(xm - xc).max() < 20 * tol * scale


@pytest.mark.parametrize("d", [1, 2, 3, 4])
def test_history_coefficients_extrapolate_polynomials(d):
    """x0 adds sum_k c_k t_k over the last d steps' corrections (t_1 the
    newest), c = (1), (2, -1), (3, -3, 1), (4, -6, 4, -1): the value at the
    next step of the polynomial of degree d - 1 through them, exact for any
    such polynomial."""
    coef = {1: [1], 2: [2, -1], 3: [3, -3, 1], 4: [4, -6, 4, -1]}[d]
    rng = np.random.default_rng(d)
    for _ in range(5):
        poly = rng.normal(size=d)  # degree d - 1
        n = 10.0
        ts = [np.polyval(poly, n - k) for k in range(1, d + 1)]
        assert abs(sum(c * t for c, t in zip(coef, ts)) - np.polyval(poly, n)) < 1e-9 * (1 + abs(np.polyval(poly, n)))
    # one degree higher is not reproduced (the next term of the series)
    poly = np.zeros(d + 1)
    poly[0] = 1.0
    ts = [np.polyval(poly, 10.0 - k) for k in range(1, d + 1)]
    assert abs(sum(c * t for c, t in zip(coef, ts)) - np.polyval(poly, 10.0)) > 0.5


@pytest.mark.parametrize("sigma", [1.5 + 0.0j, 2.0 - 3.0j, 0.3 + 4.0j, -1.2 + 0.7j])
def test_chebyshev_gain_from_the_coefficient_recurrence(sigma):
    """The batch's guaranteed gain of m Chebyshev steps: the coefficient
    recurrence rho_0 = 1/sigma, rho_{k+1} = 1/(2 sigma - rho_k) gives
    rho_k = T_k(sigma) / T_{k+1}(sigma), so 1/|rho_0 ... rho_{m-1}| equals
    |T_m(sigma)| (T the Chebyshev polynomials, T_{k+1} = 2 sigma T_k -
    T_{k-1})."""
    rho = 1.0 / sigma
    prod = 1.0 + 0.0j
    t_prev, t_cur = 1.0 + 0.0j, sigma
    for m in range(1, 20):
        prod *= rho
        assert abs(1.0 / abs(prod) - abs(t_cur)) <= 1e-9 * abs(t_cur)
        rho = 1.0 / (2.0 * sigma - rho)
        t_prev, t_cur = t_cur, 2.0 * sigma * t_cur - t_prev
