"""GPU parity of each FP64 stencil of the Crank-Nicolson solver (register-
tiled, TMA-staged, FP64 tensor-core, FP64 FMA on cached blocks), forced one
at a time, against the oracle through the C ABI.

The tensor-core and FMA stencils apply per-update 6x6 blocks and derive the
backward blocks from the forward ones (-W^H), which needs real Wilson
coefficients; with complex ones the solver runs the TMA-staged stencil
instead, and the results must not change.  Lattices cover a partial last
unit (V = 216; units of 16 and 20 sites), rows shorter than a unit (4^3,
every x neighbour wraps inside the tiles), rows of exactly one 16-site unit
(16 x 4 x 4) and units spanning rows (10 x 6 x 4).

Tolerances as for the other FP64 parity tests: matvec 1e-13 relative, CN
steps to kspTol 1e-13 agree with the oracle to 5e-13 absolute."""
import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField, NrqcdError, nrqcd
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
STENCILS = [nrqcd.STENCIL_REGISTER, nrqcd.STENCIL_TMA, nrqcd.STENCIL_TENSOR, nrqcd.STENCIL_FMA]
SHAPES = [(4, 4, 4), (6, 6, 6), (16, 4, 4), (10, 6, 4)]


def hot(oracle, n, seed=5, Q=3.0):
    return oracle.transverse_box(n, A, Q, 1.0, 0.0, seed, identity_links=False)


@pytest.mark.parametrize("stencil", STENCILS)
@pytest.mark.parametrize("n", SHAPES)
@pytest.mark.parametrize("herm", [False, True])
@pytest.mark.parametrize("coeffs", ["real", "complex"])
def test_operator_matches_oracle(oracle, stencil, n, herm, coeffs):
    links, ef = hot(oracle, n)
    V = int(np.prod(n))
    rng = np.random.default_rng(11)
    q = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    an = rng.normal(size=(V, 6, 6)) + 1j * rng.normal(size=(V, 6, 6))
    M, dt = 1.3, 0.7
    c = [1.0, 0.9, 1.1, 0.8] if coeffs == "real" else [1.0, 0.9 + 0.1j, 1.1, 0.8 - 0.2j]
    with lattice_ctx(n, A, cn=(M, c, dt, 1e-12)):
        nrqcd.SetStencil(stencil)
        g = GaugeConfiguration()
        g.upload(links, ef)
        fin, fout = NRQCDField(), NRQCDField()
        fin.upload(q, an)
        nrqcd.apply_operator(g, M, c, dt, herm, fin, fout)
        oq, oa = fout.download()
        # a second application with the other operator (A vs A^H) after the first
        fout2 = NRQCDField()
        nrqcd.apply_operator(g, M, c, dt, not herm, fin, fout2)
        oq2, oa2 = fout2.download()
        assert nrqcd.StencilInfo()[0] == stencil
    scale = np.abs(q).max()
    for h_, gq, ga in ((herm, oq, oa), (not herm, oq2, oa2)):
        eq = oracle.cn_apply(n, A, links, ef, M, c, dt, int(h_), q)
        ea = oracle.cn_apply(n, A, links, ef, -M, np.conj(c), dt, int(h_), an)
        assert np.abs(gq - eq).max() < 1e-13 * scale
        assert np.abs(ga - ea).max() < 1e-13 * scale


@pytest.mark.parametrize("stencil", STENCILS)
@pytest.mark.parametrize("n", [(6, 6, 6), (10, 6, 4), (16, 16, 16)])
def test_cn_steps_match_oracle(oracle, stencil, n):
    """Plain FP64 BiCGStab steps (RHS with A, residual, v and t with A^H)."""
    links, ef = hot(oracle, n, seed=9)
    M, c = 1.0, [1.0, 1.0, 1.0, 1.0]
    q = oracle.single_point(n, 3)
    an = oracle.single_point(n, 5)
    with lattice_ctx(n, A, cn=(M, c, 1.0, 1e-13)):
        nrqcd.SetStencil(stencil)
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(3, 5)
        for _ in range(3):
            st = h.Update(g, M, c, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] < 1e-13
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
        gq, ga = h.download()
        assert nrqcd.StencilInfo()[0] == stencil
    assert np.abs(gq - q).max() < 5e-13 and np.abs(ga - an).max() < 5e-13


@pytest.mark.parametrize("stencil", [nrqcd.STENCIL_TMA, nrqcd.STENCIL_TENSOR, nrqcd.STENCIL_FMA])
def test_precision_form_residual_stencil(oracle, stencil):
    """The FP64 refinement residual (FP32 outputs) of the precision form."""
    n = (8, 8, 8)
    links, ef = hot(oracle, n, seed=4)
    M, c, tol = 1.0, [1.0, 1.0, 1.0, 1.0], 1e-10
    q = oracle.single_point(n, 7)
    an = oracle.single_point(n, 7)
    with lattice_ctx(n, A, cn=(M, c, 1.0, tol, 10000, nrqcd.FORM_PRECISION)):
        nrqcd.SetStencil(stencil)
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(7, 7)
        for _ in range(3):
            st = h.Update(g, M, c, 1.0)
            assert st["converged"] == 1 and st["max_rel_residual"] <= tol
            oracle.cn_update(n, A, links, ef, M, c, 1.0, q, an, tol=1e-14)
        gq, ga = h.download()
    assert np.abs(gq - q).max() < 5e-10 and np.abs(ga - an).max() < 5e-10


def test_stencils_agree_and_timed_choice(oracle):
    """At 16^3 the three stencils give the same step to the solve tolerance,
    and the timed choice reports a time for each applicable stencil."""
    n = (16, 16, 16)
    links, ef = hot(oracle, n, seed=2)
    M, c = 1.0, [1.0, 1.0, 1.0, 1.0]
    out = {}
    with lattice_ctx(n, A, cn=(M, c, 1.0, 1e-12)):
        for stencil in STENCILS + [None]:
            nrqcd.SetStencil(stencil)
            g = GaugeConfiguration()
            g.upload(links, ef)
            h = NRQCDField()
            h.InitSinglePoint(1, 2)
            for _ in range(2):
                assert h.Update(g, M, c, 1.0)["converged"] == 1
            out[stencil] = h.download()
        which, ms = nrqcd.StencilInfo()
    assert which in STENCILS and (ms > 0).all()
    ref_q, ref_a = out[nrqcd.STENCIL_REGISTER]
    for k, (gq, ga) in out.items():
        assert np.abs(gq - ref_q).max() < 5e-12 and np.abs(ga - ref_a).max() < 5e-12, k


def test_staged_stencils_rejected_for_odd_volume():
    with lattice_ctx((5, 5, 5), A, cn=(1.0, [1, 1, 1, 1], 1.0, 1e-12)):
        nrqcd.SetStencil(nrqcd.STENCIL_REGISTER)
        for stencil in (nrqcd.STENCIL_TMA, nrqcd.STENCIL_TENSOR, nrqcd.STENCIL_FMA):
            with pytest.raises(NrqcdError):
                nrqcd.SetStencil(stencil)
        with pytest.raises(NrqcdError):
            nrqcd.SetStencil(7)
        nrqcd.SetStencil(None)
