"""The device draw of the initial conditions' random stream.

The ranlxd recurrence runs on the device in 48-bit integers, each thread
from a starting state the host computes by one modular multiplication
(block_states, nrqcd_b200/csrc/ranlxd_host.h), and the Box-Muller transform
of src/random.f90:238-255 follows on the device.  The uniform numbers must
equal the oracle's stream bit for bit, at any (even) starting position and
for both luxury levels.  The normals use the device's FP64 log and cos in
the host's expression; against the oracle (the host C library) they agree
to 4 ulp of the normal's magnitude, far below what the initial-condition
tests (1e-13 on the fields) resolve."""
import ctypes

import numpy as np
import pytest

from nrqcd_b200 import _capi
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)


def device_draw(level, seed, first, count, normals):
    from nrqcd_b200 import lattice
    out = np.empty(count)
    rc = _capi.load().nrq_ranlxd_draw(lattice.context(), level, seed, first, count, int(normals), _capi.dptr(out))
    assert rc == _capi.NRQ_OK, rc
    return out


@pytest.mark.parametrize("level,seed", [(2, 1), (2, 2147483647), (2, 12345), (1, 7)])
@pytest.mark.parametrize("first,count", [(0, 2), (0, 12), (2, 10), (10, 1000), (24, 50000), (123456, 30002)])
def test_device_uniforms_equal_the_stream(oracle, level, seed, first, count):
    with lattice_ctx((8, 8, 8), A):
        got = device_draw(level, seed, first, count, False)
    want = oracle.Ranlxd(level, seed).draw(first + count)[first:]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("seed,first,count", [(1, 0, 20000), (3, 48 * 512, 4097), (99, 14, 6)])
def test_device_normals_match_the_host(oracle, seed, first, count):
    with lattice_ctx((8, 8, 8), A):
        got = device_draw(2, seed, first, count, True)
    r = oracle.Ranlxd(2, seed)
    if first:
        r.draw(first)
    want = r.normal_cmplx(count).real
    ulp = np.spacing(np.abs(want))
    assert np.all(np.abs(got - want) <= 4 * ulp)


def test_device_draw_rejects_bad_arguments():
    from nrqcd_b200 import lattice
    lib = _capi.load()
    out = np.empty(4)
    with lattice_ctx((8, 8, 8), A):
        ctx = lattice.context()
        for level, seed, first, count in ((3, 1, 0, 2), (2, 0, 0, 2), (2, 2 ** 31, 0, 2), (2, 1, 1, 2), (2, 1, 0, 3)):
            assert lib.nrq_ranlxd_draw(ctx, level, seed, first, count, 0, _capi.dptr(out)) == _capi.NRQ_ERR_BAD_ARG
