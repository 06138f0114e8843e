"""C ABI: the library loads and exports every entry point the header declares;
without a GPU the product fails loudly (no CPU fallback)."""
import ctypes
import os
import re

import pytest

from tests.conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "nrqcd_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nrq_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from nrqcd_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
    return ctypes.CDLL(build.LIB)


def test_header_symbols_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s


def test_python_binding_covers_header():
    from nrqcd_b200 import _capi
    assert set(declared_symbols()) == set(_capi.SIGNATURES)


def test_status_strings(lib):
    lib.nrq_status_string.restype = ctypes.c_char_p
    assert lib.nrq_status_string(0) == b"ok"
    assert b"converge" in lib.nrq_status_string(5)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    from nrqcd_b200 import NrqcdError, lattice
    with pytest.raises(NrqcdError) as e:
        lattice.InitModule([4, 4, 4], [0.05, 1, 1, 1])
    assert e.value.code == 8  # NRQ_ERR_NO_DEVICE
    assert not lattice.IsModuleInitialised()


def test_module_guards_without_device():
    from nrqcd_b200 import NrqcdError, nrqcd
    with pytest.raises(NrqcdError):
        nrqcd.FinalizeModule()
    if not gpu_available():
        with pytest.raises(NrqcdError):
            nrqcd.InitModule(1.0, [1, 1, 1, 1], 1.0, 1e-12)


def test_objects_outliving_their_module_context_are_not_destroyed_through_a_new_one():
    """A gauge or heavy object still referenced after lattice.FinalizeModule
    belongs to the finalised context: its handle must not be passed to the
    library once another module context is open (the open check compares the
    context itself, not 'some module context is open')."""
    import numpy as np
    from nrqcd_b200 import lattice
    saved = (lattice._ctx, lattice._extents, lattice._spacings)
    try:
        lattice._ctx, lattice._extents, lattice._spacings = object(), np.array([2, 2, 2]), np.ones(4)
        ctx, V, is_open = lattice._resolve(None)
        assert ctx is lattice._ctx and V == 8 and is_open()
        lattice._ctx = object()  # finalised and replaced by a new InitModule
        assert not is_open()
        lattice._ctx = None  # finalised
        assert not is_open()
    finally:
        lattice._ctx, lattice._extents, lattice._spacings = saved


def test_header_is_plain_c_and_links(lib, tmp_path):
    """A C99 program includes the header and links the library the way the
    reference's Fortran binding would: the header is valid C (no C++ or torch
    types) and the entry points resolve at link time.  Without a GPU,
    nrq_init reports an error and no context; with one, it opens and
    finalises a context."""
    import shutil
    import subprocess
    from nrqcd_b200 import build
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text(r'''
#include <stdio.h>
#include "nrqcd_b200.h"
int main(void) {
  int64_t ext[3] = {4, 4, 4};
  double sp[4] = {0.05, 1.0, 1.0, 1.0};
  nrq_ctx *ctx = NULL;
  int rc = nrq_init(ext, sp, 0, &ctx);
  printf("%d %s\n", rc, nrq_status_string(rc));
  if (rc == NRQ_OK) return nrq_finalize(ctx) == NRQ_OK ? 0 : 5;
  return ctx == NULL ? 3 : 4;
}
''')
    exe = tmp_path / "abi"
    libdir = os.path.dirname(build.LIB)
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-L", libdir, "-lnrqcd_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == (0 if gpu_available() else 3), run.stdout + run.stderr


# every entry point of the C ABI; a declaration added to or removed from the
# header must be added to or removed from this list as well
EXPECTED_SYMBOLS = {
    "nrq_init", "nrq_finalize", "nrq_synchronize", "nrq_cuda_stream", "nrq_status_string", "nrq_last_error",
    "nrq_profile_enable", "nrq_profile_read", "nrq_ranlxd_draw",
    "nrq_gauge_create", "nrq_gauge_destroy", "nrq_gauge_upload", "nrq_gauge_download", "nrq_gauge_copy",
    "nrq_gauge_cold_init", "nrq_gauge_transverse_box_init", "nrq_gauge_update", "nrq_gauge_set_precision",
    "nrq_gauge_unitarity", "nrq_gauge_energy", "nrq_gauge_gauss", "nrq_gauge_gauss_project",
    "nrq_gauge_equilibrium_init", "nrq_gauge_coulomb_gaugefix", "nrq_gauge_transverse_correlators",
    "nrq_gauge_energy_noalloc",
    "nrq_heavy_create", "nrq_heavy_destroy", "nrq_heavy_upload", "nrq_heavy_download", "nrq_heavy_copy",
    "nrq_heavy_init_single_point", "nrq_heavy_norms", "nrq_heavy_correlators", "nrq_heavy_correlators_gconjg",
    "nrq_heavy_update_cn",
    "nrq_cn_init", "nrq_cn_finalize", "nrq_cn_apply", "nrq_cn_stencil_info", "nrq_cn_set_stencil",
    "nrq_cn_set_history_guess", "nrq_cn_attach_learned", "nrq_cn_set_wait_test",
    "nrq_cn_set_cheb_stencil", "nrq_cn_cheb_info", "nrq_cn_set_true_residual", "nrq_cn_true_residual_info",
    "nrq_cn_set_merged_update", "nrq_cn_set_history_depth",
    "nrq_cn_batch_create", "nrq_cn_batch_destroy", "nrq_cn_batch_update", "nrq_cn_batch_info",
    "nrq_cn_batch_set_variant", "nrq_cn_batch_set_fp64", "nrq_cn_batch_fp64_info", "nrq_cn_batch_learned_info",
    "nrq_cn_batch_prediction_info", "nrq_cn_batch_set_history",
    "nrq_cn_batch_residuals", "nrq_cn_batch_attach_learned",
    "nrq_ensemble_create", "nrq_ensemble_destroy", "nrq_ensemble_step",
    "nrq_learn_create", "nrq_learn_destroy", "nrq_learn_record", "nrq_learn_train", "nrq_learn_params",
    "nrq_learn_set_trained", "nrq_learn_forward", "nrq_learn_loss_grad", "nrq_learn_dataset_reserve",
    "nrq_learn_dataset_size", "nrq_learn_dataset_read",
}


def test_header_declares_exactly_the_expected_entry_points(lib):
    """The header declares the C ABI's entry points, no more and no fewer, and
    the library exports each of them."""
    assert set(declared_symbols()) == EXPECTED_SYMBOLS
    for s in EXPECTED_SYMBOLS:
        assert hasattr(lib, s), s
