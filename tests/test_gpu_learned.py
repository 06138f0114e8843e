"""GPU checks of the learned initial guess (form 2): the tensor-core forward
and backward kernels against the CPU oracle (oracle/learned_mlp.py, which
mirrors their BF16 rounding points), the recorded training samples against
features and statistics recomputed on the CPU, and the trained network's
gain over the plain precision form at the same FP64 residual."""
import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField, nrqcd
from nrqcd_b200.learned import LearnedGuess
from oracle import learned_mlp as lm
from tests.gpu_util import lattice_ctx
from tests.test_learned_oracle import random_stats

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
C = [1, 1, 1, 1]


def _random_problem(n, seed):
    rng = np.random.default_rng(seed)
    feat = rng.normal(size=(n, lm.NIN)).astype(np.float32)
    st = random_stats(n, rng)
    p = (rng.normal(size=lm.NPARAMS) * 0.2).astype(np.float32)
    return p, feat, st.astype(np.float32)


@pytest.mark.parametrize("n", [128, 300])
def test_forward_matches_oracle(n):
    p, feat, _ = _random_problem(n, 1)
    with lattice_ctx((4, 4, 4), A):
        net = LearnedGuess(seed=3)
        net.params = p
        y = net.forward(feat)
        net.Destructor()
    yo, _ = lm.forward(p.astype(np.float64), feat)
    scale = np.abs(yo).max()
    # FP32 accumulation order and the rare BF16 tie of a hidden unit
    assert np.abs(y - yo).max() <= 2e-3 * scale


@pytest.mark.parametrize("n", [128, 1000])
def test_gradient_matches_oracle(n):
    p, feat, st = _random_problem(n, 2)
    with lattice_ctx((4, 4, 4), A):
        net = LearnedGuess(seed=3)
        net.params = p
        loss, g = net.loss_grad(feat, st)
        net.Destructor()
    lo, go = lm.loss_grad(p.astype(np.float64), feat, st)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    # every parameter block within 1e-3 of its own scale
    o = 0
    for name, shape in lm.SIZES:
        k = int(np.prod(shape))
        a, b = g[o:o + k], go[o:o + k]
        assert np.abs(a - b).max() <= 1e-3 * max(np.abs(b).max(), 1e-12), name
        o += k


def test_recorded_samples_match_oracle(oracle):
    n = (6, 6, 6)
    V = int(np.prod(n))
    M, tau = 1.0, 1.0 * A[0] / 2
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 9, identity_links=False)
    with lattice_ctx(n, A, cn=(M, C, 1.0, 1e-12, 10000, 1)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        net = LearnedGuess(seed=3)
        nsteps = 3
        net.reserve(nsteps * 2 * V)
        hist = []  # per step: [quark miss, antiquark miss]
        rows = []
        for step in range(nsteps):
            q0, a0 = h.download()
            net.record(h, g, M, C, 1.0)
            q1, a1 = h.download()
            cur = []
            for sp, (psi, x) in enumerate(((q0, q1), (a0, a1))):
                b = oracle.cn_apply(n, A, links, ef, M if sp == 0 else -M, C, 1.0, 0, psi)
                v1 = hist[-1][sp] if len(hist) >= 1 else None
                v2 = hist[-2][sp] if len(hist) >= 2 else None
                f = lm.features(n, links, ef, psi, b, v1, v2, M, tau, sp)
                s = lm.stats(psi, b, v1, v2, x, s0=abs(tau))
                cur.append((f, s, (x - (2 * b - psi))))
            rows.append(cur)
            hist.append([cur[0][2], cur[1][2]])
        feat, st = net.read(0, nsteps * 2 * V)
        net.Destructor()
    for step in range(nsteps):
        f_all = np.concatenate([rows[step][0][0], rows[step][1][0]])
        s_all = np.concatenate([rows[step][0][1], rows[step][1][1]])
        s_all = s_all * (2 * V / s_all[:, -1].sum())
        fg = feat[step * 2 * V:(step + 1) * 2 * V]
        sg = st[step * 2 * V:(step + 1) * 2 * V]
        assert np.abs(fg - f_all).max() <= 1e-4 * max(1.0, np.abs(f_all).max())
        assert np.abs(sg - s_all).max() <= 1e-4 * np.abs(s_all).max()


def test_trained_guess_beats_plain_extrapolation(oracle):
    """Train on 8 recorded steps of two seeded 8^3 fields; a third field then
    needs fewer inner steps with the learned start than from 2b - psi, and
    the two forms agree to the solve tolerance."""
    n = (8, 8, 8)
    V = int(np.prod(n))
    M, tol = 1.0, 1e-10
    with lattice_ctx(n, A, cn=(M, C, 1.0, tol, 10000, nrqcd.FORM_LEARNED)):
        net = LearnedGuess(seed=5)
        net.reserve(16 * 2 * V)
        for seed in (21, 22):
            links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, seed, identity_links=False)
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(1 + seed, 1 + 2 * seed)
            for _ in range(8):
                net.record(h, g, M, C, 1.0)
                g.Update(1.0)
        l0, l1 = net.train(400, batch=2048, lr=2e-3, seed=7)
        assert l1 < 0.2 * l0
        links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 23, identity_links=False)
        runs = {}
        for use in (False, True):
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(5, 9)
            if use:
                net.attach()
            else:
                net.detach()
                nrqcd.SetHistoryGuess(False)  # the start 2b - psi alone
            its, r0 = [], []
            for _ in range(5):
                st = h.Update(g, M, C, 1.0)
                assert st["converged"] == 1 and st["max_rel_residual"] <= tol
                its.append(st["iterations"])
                r0.append(st["initial_rel_residual"])
                g.Update(1.0)
            runs[use] = (its, h.download(), r0)
            nrqcd.SetHistoryGuess(True)
        net.detach()
        net.Destructor()
    its_plain, (qp, ap), r0_plain = runs[False]
    its_learned, (ql, al), r0_learned = runs[True]
    # from the third step on both history vectors exist
    assert max(r0_learned[2:]) < 0.1 * min(r0_plain[2:])
    assert sum(its_learned[2:]) < sum(its_plain[2:])
    assert np.abs(ql - qp).max() < 5e-10 and np.abs(al - ap).max() < 5e-10
