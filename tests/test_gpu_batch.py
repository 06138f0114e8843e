"""GPU checks of the batching form of the Crank-Nicolson step: a batch of
fields (sources x masses) in one gauge field per launch, and ensembles of
members of different lattice sizes stepped by one CUDA graph launch.

Every field of a batch must equal the single-field update of the same field
to within the solve tolerance (tol 1e-10 on unit-norm propagators: the
fields agree to a few 1e-10), the graph replay must equal the eager launch
sequence bit for bit, and an ensemble step must equal its members stepped
one by one."""
import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField, NrqcdError, lattice
from nrqcd_b200.batch import CNBatch, Ensemble
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
C = [1, 1, 1, 1]
FORM_PRECISION = 1


def _sources(V, k, seed):
    rng = np.random.default_rng(seed)
    return [(int(a) + 1, int(b) + 1) for a, b in rng.integers(0, V, size=(k, 2))]


def _hot_gauge(oracle, n, seed, lat=None):
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, seed, identity_links=False)
    g = GaugeConfiguration(lat=lat)
    g.upload(links, ef)
    return g, links, ef


def _fields(V, srcs, lat=None):
    out = []
    for lq, la in srcs:
        h = NRQCDField(lat=lat)
        h.InitSinglePoint(lq, la)
        out.append(h)
    return out


def test_batch_matches_single_field_updates(oracle):
    """4 sources x 2 masses at 8^3: batch (graph replays) vs one precision
    update per field, and the oracle for two of the fields."""
    n = (8, 8, 8)
    V = int(np.prod(n))
    masses = [1.0, 1.5]
    srcs = _sources(V, 4, 11)
    tol = 1e-10
    with lattice_ctx(n, A, cn=(masses[0], C, 1.0, tol, 10000, FORM_PRECISION)):
        g, links, ef = _hot_gauge(oracle, n, 7)
        hs = _fields(V, srcs) + _fields(V, srcs)
        ms = [masses[0]] * 4 + [masses[1]] * 4
        b = CNBatch(hs, ms, tol)
        singles = _fields(V, srcs) + _fields(V, srcs)
        for step in range(3):
            st = b.Update(g, C, 1.0, use_graph=True)
            assert st["converged"] == 1 and st["max_rel_residual"] <= tol
            assert (b.residuals() <= tol).all()
            for h, m in zip(singles, ms):
                s1 = h.Update(g, m, C, 1.0)
                assert s1["converged"] == 1
        info = b.info()
        assert info["fields_per_tile"] in (1, 2) and info["block_order"] in (0, 1)
        assert info["candidate_ms"]["tile1_2blocks_order0"] > 0 and info["candidate_ms"]["tile1_3blocks_order1"] > 0
        assert 1 <= len(info["schedule"]) <= 8
        for hb, hsg in zip(hs, singles):
            qb, ab = hb.download()
            qs, as_ = hsg.download()
            assert np.abs(qb - qs).max() < 5e-10 and np.abs(ab - as_).max() < 5e-10
            assert abs(hb.GetNorm_Quark() - 1) < 1e-9 and abs(hb.GetNorm_AntiQ() - 1) < 1e-9
        # the oracle (FP64 GMRES to 1e-14) for the first field of each mass
        for idx in (0, 4):
            lq, la = srcs[idx % 4]
            q = oracle.single_point(n, lq)
            an = oracle.single_point(n, la)
            for _ in range(3):
                oracle.cn_update(n, A, links, ef, ms[idx], C, 1.0, q, an, tol=1e-14)
            qb, ab = hs[idx].download()
            assert np.abs(qb - q).max() < 5e-10 and np.abs(ab - an).max() < 5e-10
        b.Destructor()


def test_batch_predicted_acceptance_true_residuals(oracle):
    """The scheduled steps accept columns on the Chebyshev prediction of the
    last pass (with the margin the measured columns calibrate): over graph
    replays on an evolving 16^3 gauge field, the true residual of every
    field, recomputed by the oracle from the downloaded fields, stays within
    the tolerance, and the margin has been measured."""
    from tests.test_gpu_cn import _true_rel_residuals
    n = (16, 16, 16)
    V = int(np.prod(n))
    masses = [1.0, 1.5]
    srcs = _sources(V, 2, 5)
    tol = 1e-10
    with lattice_ctx(n, A, cn=(masses[0], C, 1.0, tol, 10000, FORM_PRECISION)):
        g, _, _ = _hot_gauge(oracle, n, 3)
        hs = _fields(V, srcs) + _fields(V, srcs)
        ms = [masses[0]] * 2 + [masses[1]] * 2
        b = CNBatch(hs, ms, tol)
        for _ in range(6):
            olds = [h.download() for h in hs]
            gl, ge = g.download()
            st = b.Update(g, C, 1.0, use_graph=True)
            assert st["converged"] == 1 and st["max_rel_residual"] <= tol
            for h, m, old in zip(hs, ms, olds):
                assert _true_rel_residuals(oracle, n, gl, ge, m, np.array(C, dtype=complex), old, h.download()) <= tol
            g.Update(1.0)
        info = b.prediction_info()
        assert info["ratio"] >= 0.0 and info["steps"] >= 1
        b.Destructor()


def test_graph_replay_equals_eager_launches(oracle):
    """The captured step and the same launches issued one by one agree bit for bit."""
    n = (6, 6, 6)
    V = int(np.prod(n))
    srcs = _sources(V, 4, 5)
    with lattice_ctx(n, A, cn=(1.0, C, 1.0, 1e-10, 10000, FORM_PRECISION)):
        g, _, _ = _hot_gauge(oracle, n, 3)
        ha = _fields(V, srcs)
        hb = _fields(V, srcs)
        ms = [1.0, 1.0, 2.0, 2.0]
        ba = CNBatch(ha, ms, 1e-10)
        bb = CNBatch(hb, ms, 1e-10)
        for _ in range(4):
            ba.Update(g, C, 1.0, use_graph=False)
            bb.Update(g, C, 1.0, use_graph=True)
        # same tuning choice is not guaranteed (timing); equal results only when equal
        if ba.info()["variant"] == bb.info()["variant"] and \
                ba.info()["block_order"] == bb.info()["block_order"] and \
                ba.info()["schedule"] == bb.info()["schedule"]:
            for x, y in zip(ha, hb):
                qa, aa = x.download()
                qb, ab = y.download()
                assert np.array_equal(qa, qb) and np.array_equal(aa, ab)
        else:
            for x, y in zip(ha, hb):
                qa, aa = x.download()
                qb, ab = y.download()
                assert np.abs(qa - qb).max() < 5e-10 and np.abs(aa - ab).max() < 5e-10
        ba.Destructor()
        bb.Destructor()


def test_ensemble_of_uneven_members_matches_member_steps(oracle):
    """Members 2 x 6^3 + 1 x 8^3, 4 fields each (2 sources x 2 masses): one
    graph launch per step equals each member's batch update plus leapfrog."""
    sizes = [(6, 6, 6), (6, 6, 6), (8, 8, 8)]
    ms = [1.0, 1.0, 1.5, 1.5]
    lat6 = lattice.Lattice((6, 6, 6), A)
    lat8 = lattice.Lattice((8, 8, 8), A)
    lats = [lat6, lat6, lat8]
    try:
        runs = []
        for use_graph in (True, False):
            gauges, batches, fields = [], [], []
            for i, (n, lat) in enumerate(zip(sizes, lats)):
                g, _, _ = _hot_gauge(oracle, n, 20 + i, lat=lat)
                V = int(np.prod(n))
                srcs = _sources(V, 2, 30 + i)
                hs = _fields(V, srcs + srcs, lat=lat)
                gauges.append(g)
                fields.append(hs)
                batches.append(CNBatch(hs, ms, 1e-10, lat=lat))
            if use_graph:
                ens = Ensemble(batches, gauges)
                for _ in range(4):
                    st = ens.Step(C, 1.0, use_graph=True)
                    assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
                ens.Destructor()
            else:
                for _ in range(4):
                    for b, g in zip(batches, gauges):
                        b.Update(g, C, 1.0, use_graph=False)
                        g.Update(1.0)
            runs.append(([[h.download() for h in hs] for hs in fields], [g.download() for g in gauges],
                         [b.info() for b in batches]))
            for b in batches:
                b.Destructor()
            for hs in fields:
                for h in hs:
                    h.Destructor()
            for g in gauges:
                g.Deallocate()
        (fa, ga, ia), (fb, gb, ib) = runs
        for m in range(3):
            la, ea = ga[m]
            lb, eb = gb[m]
            assert np.array_equal(la, lb) and np.array_equal(ea, eb)
            same = ia[m]["variant"] == ib[m]["variant"] and \
                ia[m]["block_order"] == ib[m]["block_order"] and ia[m]["schedule"] == ib[m]["schedule"]
            for (qa, aa), (qb, ab) in zip(fa[m], fb[m]):
                if same:
                    assert np.array_equal(qa, qb) and np.array_equal(aa, ab)
                else:
                    assert np.abs(qa - qb).max() < 5e-10 and np.abs(aa - ab).max() < 5e-10
    finally:
        lat6.close()
        lat8.close()


def test_batch_rejects_bad_arguments(oracle):
    n = (4, 4, 4)
    with lattice_ctx(n, A):
        g, _, _ = _hot_gauge(oracle, n, 1)
        h1, h2 = NRQCDField(), NRQCDField()
        h1.InitSinglePoint(1, 1)
        h2.InitSinglePoint(2, 2)
        with pytest.raises(NrqcdError):
            CNBatch([h1, h1], [1.0, 1.0], 1e-10)
        with pytest.raises(NrqcdError):
            CNBatch([h1, h2], [1.0, 0.0], 1e-10)
        b = CNBatch([h1, h2], [1.0, 2.0], 1e-10)
        with pytest.raises(NrqcdError):
            b.Update(g, [1, 1j, 1, 1], 1.0)
        other = lattice.Lattice((4, 4, 4), A)
        try:
            g2 = GaugeConfiguration(lat=other)
            with pytest.raises(NrqcdError):
                b.Update(g2, C, 1.0)
            g2.Deallocate()
        finally:
            other.close()
        st = b.Update(g, C, 1.0)
        assert st["converged"] == 1
        b.Destructor()


def test_batch_with_learned_guess_matches_single_updates(oracle):
    """Forms combined: a batch whose solves start from the learned guess
    (network trained on recorded 8^3 steps) gives every field the result of
    its own precision-form update, and needs no more inner steps per step
    than the batch started from 2b - psi once the history is full."""
    from nrqcd_b200 import nrqcd
    from nrqcd_b200.learned import LearnedGuess
    n = (8, 8, 8)
    V = int(np.prod(n))
    tol = 1e-10
    with lattice_ctx(n, A, cn=(1.0, C, 1.0, tol, 10000, FORM_PRECISION)):
        net = LearnedGuess(seed=5)
        net.reserve(16 * 2 * V)
        for seed in (41, 42):
            g0, _, _ = _hot_gauge(oracle, n, seed)
            h0 = NRQCDField()
            h0.InitSinglePoint(3 + seed, 7 + seed)
            for _ in range(8):
                net.record(h0, g0, 1.0, C, 1.0)
                g0.Update(1.0)
        net.train(400, batch=2048, lr=2e-3, seed=7)
        g, _, _ = _hot_gauge(oracle, n, 43)
        srcs = _sources(V, 2, 17)
        ms = [1.0, 1.0, 1.5, 1.5]
        hl = _fields(V, srcs + srcs)
        hp = _fields(V, srcs + srcs)
        singles = _fields(V, srcs + srcs)
        bl = CNBatch(hl, ms, tol)
        bl.attach_learned(net)
        bp = CNBatch(hp, ms, tol)
        bp.set_history(False)  # the start 2b - psi the guess improves on
        inner_l, inner_p = [], []
        for step in range(6):
            sl = bl.Update(g, C, 1.0, use_graph=True)
            sp_ = bp.Update(g, C, 1.0, use_graph=True)
            assert sl["converged"] == 1 and sl["max_rel_residual"] <= tol
            inner_l.append(sl["iterations"])
            inner_p.append(sp_["iterations"])
            for h, m in zip(singles, ms):
                assert nrqcd.solver_handle() is not None
                h.Update(g, m, C, 1.0)
        assert sum(inner_l[3:]) <= sum(inner_p[3:])
        for a_, b_ in zip(hl, singles):
            qa, aa = a_.download()
            qb, ab = b_.download()
            assert np.abs(qa - qb).max() < 5e-10 and np.abs(aa - ab).max() < 5e-10
        bl.attach_learned(None)
        bl.Destructor()
        bp.Destructor()
        net.Destructor()


def test_batch_learned_guess_gate(oracle):
    """A guess attached after plain steps is gated at the calibration with
    its full history: its cost and the value of the steps it saved are
    measured, the gate is decided, and the fields keep their single-field
    results either way (once off, the batch runs the plain start)."""
    from nrqcd_b200.learned import LearnedGuess
    n = (8, 8, 8)
    V = int(np.prod(n))
    tol = 1e-10
    with lattice_ctx(n, A, cn=(1.0, C, 1.0, tol, 10000, FORM_PRECISION)):
        net = LearnedGuess(seed=3)
        net.reserve(16 * 2 * V)
        g0, _, _ = _hot_gauge(oracle, n, 51)
        h0 = NRQCDField()
        h0.InitSinglePoint(5, 9)
        for _ in range(8):
            net.record(h0, g0, 1.0, C, 1.0)
            g0.Update(1.0)
        net.train(300, batch=2048, lr=2e-3, seed=3)
        g, _, _ = _hot_gauge(oracle, n, 52)
        srcs = _sources(V, 2, 19)
        ms = [1.0, 1.0, 1.5, 1.5]
        hb = _fields(V, srcs + srcs)
        singles = _fields(V, srcs + srcs)
        b = CNBatch(hb, ms, tol)
        assert b.learned_info()["gate"] == "none"
        for step in range(7):
            if step == 2:
                b.attach_learned(net)
                assert b.learned_info()["gate"] == "undecided"
            assert b.Update(g, C, 1.0, use_graph=True)["converged"] == 1
            for h, m in zip(singles, ms):
                h.Update(g, m, C, 1.0)
        info = b.learned_info()
        assert info["gate"] in ("on", "off") and info["guess_ms"] > 0 and info["saving_ms"] >= 0
        for a_, b_ in zip(hb, singles):
            qa, aa = a_.download()
            qb, ab = b_.download()
            assert np.abs(qa - qb).max() < 5e-10 and np.abs(aa - ab).max() < 5e-10
        b.attach_learned(None)
        b.Destructor()
        net.Destructor()


@pytest.mark.parametrize("n", [(8, 8, 8), (36, 4, 4)])
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("fp64", ["register", "blocks"])
def test_batch_fp32_block_step(oracle, n, order, fp64):
    """The batch forced onto the FP32 block Chebyshev step (variant 3) with
    either FP64 stencil for the right-hand side and residuals: every field
    equals its single-field update to within the tolerance, and two fields
    the oracle.  36 x 4 x 4 has rows long enough for the x-wrap columns;
    2 masses x 3 sources use two block sets."""
    V = int(np.prod(n))
    masses = [1.0, 1.5]
    srcs = _sources(V, 3, 13)
    tol = 1e-10
    with lattice_ctx(n, A, cn=(masses[0], C, 1.0, tol, 10000, FORM_PRECISION)):
        g, links, ef = _hot_gauge(oracle, n, 9)
        hs = _fields(V, srcs) + _fields(V, srcs)
        ms = [masses[0]] * 3 + [masses[1]] * 3
        b = CNBatch(hs, ms, tol)
        b.set_variant("fp32_blocks_tma", order)
        b.set_fp64(fp64)
        singles = _fields(V, srcs) + _fields(V, srcs)
        for step in range(3):
            st = b.Update(g, C, 1.0, use_graph=step > 0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= tol
            for h, m in zip(singles, ms):
                assert h.Update(g, m, C, 1.0)["converged"] == 1
        info = b.info()
        assert info["variant"] == "fp32_blocks_tma" and info["block_order"] == order
        assert info["fp64_stencil"] == fp64
        for hb, hsg in zip(hs, singles):
            qb, ab = hb.download()
            qs, as_ = hsg.download()
            assert np.abs(qb - qs).max() < 5e-10 and np.abs(ab - as_).max() < 5e-10
        for idx in (0, 3):
            lq, la = srcs[idx % 3]
            q = oracle.single_point(n, lq)
            an = oracle.single_point(n, la)
            for _ in range(3):
                oracle.cn_update(n, A, links, ef, ms[idx], C, 1.0, q, an, tol=1e-14)
            qb, ab = hs[idx].download()
            assert np.abs(qb - q).max() < 5e-10 and np.abs(ab - an).max() < 5e-10
        b.Destructor()


def test_batch_fp32_block_step_refused_for_odd_rows():
    with lattice_ctx((5, 4, 4), A, cn=(1.0, C, 1.0, 1e-10, 10000, FORM_PRECISION)):
        hs = _fields(80, [(1, 1), (2, 2)])
        b = CNBatch(hs, [1.0, 1.0], 1e-10)
        with pytest.raises(NrqcdError):
            b.set_variant("fp32_blocks_tma", 0)
        b.Destructor()
