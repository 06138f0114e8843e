"""Ragged and degenerate lattice shapes through every CN path and the
leapfrog, against the FP64 oracle: odd extents, extents 1 and 2, volumes
that are not multiples of the 32-site blocks, and a volume that takes the
TMA-staged stencil with tiles wrapping over several x-rows."""
import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField
from nrqcd_b200.batch import CNBatch
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
C = [1, 1, 1, 1]
SHAPES = [(5, 5, 5), (7, 5, 3), (9, 4, 6), (2, 3, 4), (4, 1, 5), (4, 1, 16), (16, 2, 4)]


@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("form,tol,atol", [(0, 1e-12, 5e-12), (1, 1e-10, 5e-10)])
def test_cn_and_leapfrog_on_shape(oracle, n, form, tol, atol):
    V = int(np.prod(n))
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 4, identity_links=False)
    lq, la = 1 + (V // 3), 1 + (2 * V) // 3
    q, an = oracle.single_point(n, lq), oracle.single_point(n, la)
    with lattice_ctx(n, A, cn=(1.0, C, 1.0, tol, 10000, form)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(lq, la)
        for _ in range(3):
            st = h.Update(g, 1.0, C, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= tol
            g.Update(1.0)
            oracle.cn_update(n, A, links, ef, 1.0, C, 1.0, q, an, tol=1e-14)
            oracle.gauge_update(n, A, links, ef, 1.0)
        gq, ga = h.download()
        gl, ge = g.download()
    assert np.abs(gq - q).max() < atol and np.abs(ga - an).max() < atol
    assert np.abs(gl - links).max() < 1e-12 and np.abs(ge - ef).max() < 1e-12


@pytest.mark.parametrize("n", [(7, 5, 3), (4, 1, 16)])
def test_batch_on_shape(oracle, n):
    V = int(np.prod(n))
    links, ef = oracle.transverse_box(n, A, 2.0, 1.0, 0.0, 8, identity_links=False)
    with lattice_ctx(n, A, cn=(1.0, C, 1.0, 1e-10, 10000, 1)):
        g = GaugeConfiguration()
        g.upload(links, ef)
        srcs = [(1, V), (V // 2 + 1, 2)]
        hs, singles = [], []
        for lq, la in srcs * 2:
            for lst in (hs, singles):
                h = NRQCDField()
                h.InitSinglePoint(lq, la)
                lst.append(h)
        ms = [1.0, 1.0, 2.0, 2.0]
        b = CNBatch(hs, ms, 1e-10)
        for _ in range(3):
            st = b.Update(g, C, 1.0, use_graph=True)
            assert st["converged"] == 1
            for h, m in zip(singles, ms):
                h.Update(g, m, C, 1.0)
        for x, y in zip(hs, singles):
            qa, aa = x.download()
            qb, ab = y.download()
            assert np.abs(qa - qb).max() < 5e-10 and np.abs(aa - ab).max() < 5e-10
        b.Destructor()
