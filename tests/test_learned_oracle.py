"""CPU checks of the learned-guess oracle: its exact FP64 gradient against
central finite differences, and the rounded (BF16 operand) gradient that
the kernels mirror against the exact one."""
import numpy as np

from oracle import learned_mlp as lm


def random_stats(n, rng, m=6):
    """Gram statistics of random complex basis vectors u, v1, v2 and targets
    t near their span (a valid, non-negative loss)."""
    cn = lambda: rng.normal(size=(n, m)) + 1j * rng.normal(size=(n, m))  # noqa: E731
    u, v1, v2 = cn(), cn(), cn()
    t = 0.3 * u + (0.8 - 0.2j) * v1 - 0.1 * v2 + 0.1 * cn()
    e = [u, v1, v2]
    G = lambda j, k: np.sum(np.conj(e[j]) * e[k], 1)  # noqa: E731
    gg = [np.sum(np.conj(e[j]) * t, 1) for j in range(3)]
    return np.stack([G(0, 0).real, G(1, 1).real, G(2, 2).real, G(0, 1).real, G(0, 1).imag, G(0, 2).real,
                     G(0, 2).imag, G(1, 2).real, G(1, 2).imag, gg[0].real, gg[0].imag, gg[1].real, gg[1].imag,
                     gg[2].real, gg[2].imag, np.sum(np.abs(t) ** 2, 1)], axis=1)


def _problem(n=96, seed=0):
    rng = np.random.default_rng(seed)
    feat = rng.normal(size=(n, lm.NIN))
    stats = random_stats(n, rng)
    p = rng.normal(size=lm.NPARAMS) * 0.2
    return p, feat, stats


def test_exact_gradient_matches_finite_differences():
    p, feat, stats = _problem()
    loss, g = lm.loss_grad_exact(p, feat, stats)
    rng = np.random.default_rng(1)
    for k in rng.choice(lm.NPARAMS, size=40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (lm.loss_grad_exact(pp, feat, stats)[0] - lm.loss_grad_exact(pm, feat, stats)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])
    assert loss >= 0


def test_loss_is_the_guess_error():
    """The Gram-statistics loss equals |w0 u + w1 v1 + w2 v2 - t|^2 computed
    directly from the (V, 6, 6) fields the statistics come from."""
    rng = np.random.default_rng(3)
    c = lambda: rng.normal(size=(5, 6, 6)) + 1j * rng.normal(size=(5, 6, 6))  # noqa: E731
    psi, b, v1, v2, x = c(), c(), c(), c(), c()
    st = lm.stats(psi, b, v1, v2, x)
    Y = rng.normal(size=(5, lm.NOUT))
    loss, _ = lm.loss_and_dy(Y, st, 1)
    w = Y[:, 0::2] + 1j * Y[:, 1::2]
    t = x - (2 * b - psi)
    guess = w[:, 0, None, None] * (b - psi) + w[:, 1, None, None] * v1 + w[:, 2, None, None] * v2
    direct = np.sum(np.abs(guess - t) ** 2)
    assert abs(loss - direct) <= 1e-9 * direct


def test_rounded_gradient_close_to_exact():
    p, feat, stats = _problem(seed=5)
    l0, g0 = lm.loss_grad_exact(p, feat, stats)
    l1, g1 = lm.loss_grad(p, feat, stats)
    assert abs(l1 - l0) <= 0.05 * l0
    assert np.linalg.norm(g1 - g0) <= 0.05 * np.linalg.norm(g0)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.140625], dtype=np.float32)
    r = lm.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5 and r[4] == 3.140625


def test_adam_matches_the_update_rule():
    p = np.array([1.0, -2.0])
    g = np.array([0.5, -0.25])
    p1, m, v = lm.adam(p, g, np.zeros(2), np.zeros(2), 1, 0.1)
    # the first bias-corrected Adam step moves every parameter by lr * sign(g)
    assert np.allclose(p1, p - 0.1 * np.sign(g), atol=1e-6)
