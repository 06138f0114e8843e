"""The Crank-Nicolson solve's failure paths on the GPU, made on the host.

The reference never checks KSP convergence (src/nrqcd.f90:803-804, 1123):
a solve that stops early or meets a non-finite value goes on silently.  The
C ABI reports both: NRQ_ERR_NOT_CONVERGED when the iteration limit ends the
solve above the tolerance (the residual it reached is in the statistics), and
NRQ_ERR_NONFINITE when a residual turns NaN or Inf.  These tests cause each
from the host (an iteration limit of one, a NaN in an uploaded field), with
every stencil and both the plain and the precision form, and check that the
context then runs a clean step that matches the oracle."""
import ctypes

import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, NRQCDField, _capi, nrqcd
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)
N = (8, 8, 8)
M, C = 1.0, [1.0, 1.0, 1.0, 1.0]
STENCILS = [nrqcd.STENCIL_REGISTER, nrqcd.STENCIL_TMA, nrqcd.STENCIL_TENSOR, nrqcd.STENCIL_FMA]


def raw_update(h, g):
    """nrq_heavy_update_cn through the C ABI: (status, statistics)."""
    st = _capi.CnStats()
    c = _capi.coeffs(C)
    rc = _capi.load().nrq_heavy_update_cn(nrqcd.solver_handle(), h.handle, g.handle, M, _capi.dptr(c), 1.0,
                                          ctypes.byref(st))
    return rc, st.as_dict()


def clean_step_matches_oracle(oracle, links, ef, tol):
    """Upload clean fields into fresh objects, run one coupled CN step and
    compare with the oracle."""
    g = GaugeConfiguration()
    g.upload(links, ef)
    h = NRQCDField()
    q, an = oracle.single_point(N, 1), oracle.single_point(N, 1)
    h.upload(q, an)
    rc, st = raw_update(h, g)
    assert rc == _capi.NRQ_OK and st["converged"] == 1, (rc, st)
    gq, ga = h.download()
    oracle.cn_update(N, A, links, ef, M, C, 1.0, q, an, tol=1e-14)
    assert np.abs(gq - q).max() < 50 * tol and np.abs(ga - an).max() < 50 * tol


@pytest.mark.parametrize("form,tol", [(nrqcd.FORM_PLAIN_FP64, 1e-12), (nrqcd.FORM_PRECISION, 1e-10)])
@pytest.mark.parametrize("stencil", STENCILS)
def test_iteration_limit_reports_not_converged(oracle, form, tol, stencil):
    links, ef = oracle.transverse_box(N, A, 3.0, 1.0, 0.0, 5, identity_links=False)
    with lattice_ctx(N, A, cn=(M, C, 1.0, tol, 1, form)):
        nrqcd.SetStencil(stencil)
        nrqcd.SetHistoryGuess(False)
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        rc, st = raw_update(h, g)
        assert rc == _capi.NRQ_ERR_NOT_CONVERGED, (rc, st)
        assert st["converged"] == 0 and st["max_rel_residual"] > tol and np.isfinite(st["max_rel_residual"])
        # the Python mirror raises, with the code, unless asked not to
        with pytest.raises(_capi.NrqcdError) as e:
            h.Update(g, M, C, 1.0)
        assert e.value.code == _capi.NRQ_ERR_NOT_CONVERGED
        assert h.Update(g, M, C, 1.0, raise_on_nonconvergence=False)["converged"] == 0
    # a solver with the default limit on a new context converges
    with lattice_ctx(N, A, cn=(M, C, 1.0, tol, 10000, form)):
        nrqcd.SetStencil(stencil)
        clean_step_matches_oracle(oracle, links, ef, tol)


@pytest.mark.parametrize("where", ["propagator", "efield"])
@pytest.mark.parametrize("form,tol", [(nrqcd.FORM_PLAIN_FP64, 1e-12), (nrqcd.FORM_PRECISION, 1e-10)])
@pytest.mark.parametrize("stencil", STENCILS)
def test_nan_in_a_field_reports_nonfinite(oracle, where, form, tol, stencil):
    links, ef = oracle.transverse_box(N, A, 3.0, 1.0, 0.0, 5, identity_links=False)
    q, an = oracle.single_point(N, 1), oracle.single_point(N, 1)
    bad_links, bad_ef, bad_q = links.copy(), ef.copy(), q.copy()
    if where == "propagator":
        bad_q[37, 2, 4] = np.nan
    else:
        bad_ef[37, 1, 5] = np.nan
    with lattice_ctx(N, A, cn=(M, C, 1.0, tol, 10000, form)):
        nrqcd.SetStencil(stencil)
        g = GaugeConfiguration()
        g.upload(bad_links, bad_ef)
        h = NRQCDField()
        h.upload(bad_q, an)
        rc, st = raw_update(h, g)
        assert rc == _capi.NRQ_ERR_NONFINITE, (rc, st)
        assert st["converged"] == 0
        # the same context, clean fields: the next step is right
        del g, h
        clean_step_matches_oracle(oracle, links, ef, tol)


@pytest.mark.parametrize("form,tol", [(nrqcd.FORM_PLAIN_FP64, 1e-12), (nrqcd.FORM_PRECISION, 1e-10)])
def test_pipeline_wait_that_runs_out_reports_timeout(oracle, form, tol):
    """The FMA stencil's loader stops before its fourth load in every CTA
    (a load that nothing will issue), with the waits bounded at about a
    millisecond: the consumers' wait for it runs out, the stencil records
    NRQ_ERR_TIMEOUT and drains the loads it did issue, the update returns
    NRQ_ERR_TIMEOUT, and the same context then runs a clean step."""
    links, ef = oracle.transverse_box(N, A, 3.0, 1.0, 0.0, 5, identity_links=False)
    with lattice_ctx(N, A, cn=(M, C, 1.0, tol, 10000, form)):
        nrqcd.SetStencil(nrqcd.STENCIL_FMA)
        g = GaugeConfiguration()
        g.upload(links, ef)
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        nrqcd.SetWaitTest(wait_cycles=2_000_000, stall_load=3)
        rc, st = raw_update(h, g)
        assert rc == _capi.NRQ_ERR_TIMEOUT, (rc, st)
        assert b"wait" in _capi.load().nrq_last_error(_capi_ctx())
        nrqcd.SetWaitTest()
        del g, h
        clean_step_matches_oracle(oracle, links, ef, tol)
        assert nrqcd.StencilInfo()[0] == nrqcd.STENCIL_FMA


def _capi_ctx():
    from nrqcd_b200 import lattice
    return lattice.context()
