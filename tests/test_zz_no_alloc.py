"""GPU test of nrq_gauge_energy_noalloc, the energy entry point for callers
that cannot allocate device memory.  An example is a driver whose fields live
in device buffers owned by another runtime, such as OpenACC or CUDA Fortran
data regions or a framework's caching allocator.

This test plays such a caller.  torch owns the input and output buffers.  The
entry point gets only those pointers and uses the library's fixed scratch
array.  Its result must equal nrq_gauge_energy's on the same field, within
the 1e-12 relative tolerance the other energy tests use, on two calls in a
row: the second call reuses the scratch the first one left behind.

The file name sorts last, so a run that stops at the first failure has run
every other test first.
"""
import ctypes

import numpy as np
import pytest

from nrqcd_b200 import GaugeConfiguration, _capi
from tests.gpu_util import lattice_ctx

pytestmark = pytest.mark.gpu

A = (0.05, 1.0, 1.0, 1.0)


def soa_planes(links, efield):
    """Fortran-layout host arrays -> device plane layout of the header."""
    V = links.shape[0]
    # links [site, dir, col, row] -> planes (dir, row, col) of V complex
    lp = np.ascontiguousarray(np.transpose(links, (1, 3, 2, 0))).reshape(27, V)
    lp_ri = np.ascontiguousarray(np.stack([lp.real, lp.imag], axis=-1))  # (27, V, 2)
    ep = np.ascontiguousarray(np.transpose(efield, (1, 2, 0))).reshape(24, V)
    return lp_ri, ep


def test_noalloc_energy_matches_handle_api(oracle):
    import torch

    n = (16, 12, 10)
    links, ef = oracle.transverse_box(n, A, 1.7, 1.0, 0.0, 3, identity_links=False)
    with lattice_ctx(n, A):
        g = GaugeConfiguration()
        g.upload(links, ef)
        e_handle = g.GetEnergy()
        del g
    assert e_handle > 0

    lib = _capi.load()
    lp, ep = soa_planes(links, ef)
    dev = torch.device("cuda:0")
    U = torch.from_numpy(lp).to(dev)
    E = torch.from_numpy(ep).to(dev)
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    ext = np.array(n, dtype=np.int64)
    sp = np.array(A, dtype=np.float64)
    stream = torch.cuda.current_stream(dev)
    free_after = []
    for _ in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.nrq_gauge_energy_noalloc(ext.ctypes.data_as(_capi._i64p), sp.ctypes.data_as(_capi._dp),
                                          ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(E.data_ptr()),
                                          ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == _capi.NRQ_OK
        torch.cuda.synchronize()
        # cudaMemGetInfo: the device's free memory, which any hidden cudaMalloc
        # (including one by a library) would lower
        free_after.append(torch.cuda.mem_get_info(dev)[0])
        e_noalloc = float(out.item())
        assert abs(e_noalloc - e_handle) <= 1e-12 * abs(e_handle), (e_noalloc, e_handle)
    # the first call may load the library's module on this device; the second
    # must leave the device's free memory exactly as it found it
    assert free_after[1] == free_after[0], free_after
    # the oracle agrees as well
    assert abs(e_noalloc - oracle.energy(n, A, links, ef)) <= 1e-12 * abs(e_handle)


def test_noalloc_rejects_lattices_beyond_capacity():
    import torch

    lib = _capi.load()
    dev = torch.device("cuda:0")
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    ext = np.array([256, 256, 128], dtype=np.int64)  # 8.4M sites > 4,194,304
    sp = np.array(A, dtype=np.float64)
    p = ctypes.c_void_p(buf.data_ptr())
    rc = lib.nrq_gauge_energy_noalloc(ext.ctypes.data_as(_capi._i64p), sp.ctypes.data_as(_capi._dp), p, p, p, None)
    assert rc == _capi.NRQ_ERR_CAPACITY
    assert b"capacity" in lib.nrq_status_string(rc)
    # extents whose product overflows 64 bits are rejected before it is formed
    for big in ([2 ** 40, 2 ** 40, 2 ** 40], [2 ** 21, 2 ** 21, 2], [1, 1, 2 ** 62]):
        ext = np.array(big, dtype=np.int64)
        rc = lib.nrq_gauge_energy_noalloc(ext.ctypes.data_as(_capi._i64p), sp.ctypes.data_as(_capi._dp),
                                          p, p, p, None)
        assert rc == _capi.NRQ_ERR_CAPACITY, big


# A caller that owns its buffers through the CUDA runtime directly, resets
# its device between two calls and allocates again.  It runs in a child
# process, since the reset would invalidate the test process's own CUDA
# state; the child reports the two energies and the oracle's.
_RESET_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import oracle as oc
from nrqcd_b200 import _capi
lib = _capi.load()
rt = ctypes.CDLL("libcudart.so.12")
n, A = (12, 10, 8), (0.05, 1.0, 1.0, 1.0)
links, ef = oc.transverse_box(n, A, 1.7, 1.0, 0.0, 5, identity_links=False)
V = links.shape[0]
lp = np.ascontiguousarray(np.transpose(links, (1, 3, 2, 0))).reshape(27, V)
lp = np.ascontiguousarray(np.stack([lp.real, lp.imag], axis=-1))
ep = np.ascontiguousarray(np.transpose(ef, (1, 2, 0))).reshape(24, V)
ext = np.array(n, dtype=np.int64)
sp = np.array(A, dtype=np.float64)
out = []
for call in range(2):
    bufs = []
    for host in (lp, ep, np.zeros(1)):
        d = ctypes.c_void_p()
        assert rt.cudaMalloc(ctypes.byref(d), ctypes.c_size_t(host.nbytes)) == 0
        assert rt.cudaMemcpy(d, host.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(host.nbytes), 1) == 0
        bufs.append(d)
    rc = lib.nrq_gauge_energy_noalloc(ext.ctypes.data_as(_capi._i64p), sp.ctypes.data_as(_capi._dp),
                                      bufs[0], bufs[1], bufs[2], None)
    assert rc == 0, rc
    e = np.zeros(1)
    assert rt.cudaMemcpy(e.ctypes.data_as(ctypes.c_void_p), bufs[2], ctypes.c_size_t(8), 2) == 0
    out.append(float(e[0]))
    for d in bufs:
        assert rt.cudaFree(d) == 0
    if call == 0:
        assert rt.cudaDeviceReset() == 0
print(json.dumps({"energies": out, "oracle": oc.energy(n, A, links, ef)}))
"""


def test_noalloc_after_device_reset(tmp_path):
    """The cached scratch address belongs to one CUDA context: after the
    caller resets the device, the next call must look it up again and still
    return the right energy."""
    import json
    import subprocess
    import sys

    from tests.conftest import ROOT
    r = subprocess.run([sys.executable, "-c", _RESET_CHILD, ROOT], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    e_ref = res["oracle"]
    for e in res["energies"]:
        assert abs(e - e_ref) <= 1e-12 * abs(e_ref), res
