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
