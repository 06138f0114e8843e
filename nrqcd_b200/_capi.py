"""ctypes binding of the C ABI in ``include/nrqcd_b200.h``.

The shared library is built in-tree by ``nrqcd_b200/build.py``.  There is no
fallback: if the library is missing or no CUDA device is present, the calls
raise ``NrqcdError``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libnrqcd_b200.so")

NRQ_OK = 0
NRQ_ERR_NOT_INITIALISED = 1
NRQ_ERR_ALREADY_INITIALISED = 2
NRQ_ERR_BAD_ARG = 3
NRQ_ERR_CUDA = 4
NRQ_ERR_NOT_CONVERGED = 5
NRQ_ERR_TIMEOUT = 6
NRQ_ERR_NONFINITE = 7
NRQ_ERR_NO_DEVICE = 8
NRQ_ERR_OOM = 9
NRQ_ERR_CAPACITY = 10


class NrqcdError(RuntimeError):
    """Raised where the reference calls MPIStop (src/mpiinterface.f90:148-173)."""

    def __init__(self, message, code=None):
        super().__init__(message)
        self.code = code


class CnStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("matvecs", ctypes.c_int64),
                ("vector_streams", ctypes.c_int64), ("max_rel_residual", ctypes.c_double),
                ("converged", ctypes.c_int), ("initial_rel_residual", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_pp = ctypes.POINTER(ctypes.c_void_p)
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)

# name -> (restype, argtypes); every entry point of include/nrqcd_b200.h
SIGNATURES = {
    "nrq_init": (ctypes.c_int, [_i64p, _dp, ctypes.c_int, _pp]),
    "nrq_finalize": (ctypes.c_int, [_vp]),
    "nrq_last_error": (ctypes.c_char_p, [_vp]),
    "nrq_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "nrq_synchronize": (ctypes.c_int, [_vp]),
    "nrq_cuda_stream": (ctypes.c_void_p, [_vp]),
    "nrq_profile_enable": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_profile_read": (ctypes.c_int, [_vp, _i64p, _dp, _dp]),
    "nrq_ranlxd_draw": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int, _dp]),
    "nrq_gauge_create": (ctypes.c_int, [_vp, _pp]),
    "nrq_gauge_destroy": (ctypes.c_int, [_vp]),
    "nrq_gauge_upload": (ctypes.c_int, [_vp, _dp, _dp]),
    "nrq_gauge_download": (ctypes.c_int, [_vp, _dp, _dp]),
    "nrq_gauge_copy": (ctypes.c_int, [_vp, _vp]),
    "nrq_gauge_cold_init": (ctypes.c_int, [_vp]),
    "nrq_gauge_transverse_box_init": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                      ctypes.c_int64, ctypes.c_int]),
    "nrq_gauge_update": (ctypes.c_int, [_vp, ctypes.c_double]),
    "nrq_gauge_set_precision": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "nrq_gauge_unitarity": (ctypes.c_int, [_vp, _dp, _dp]),
    "nrq_gauge_energy": (ctypes.c_int, [_vp, _dp]),
    "nrq_gauge_gauss": (ctypes.c_int, [_vp, _dp, _dp]),
    "nrq_gauge_gauss_project": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int64, _i64p, _dp]),
    "nrq_gauge_coulomb_gaugefix": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int64, _i64p,
                                                  _dp]),
    "nrq_gauge_transverse_correlators": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "nrq_gauge_equilibrium_init": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int64, ctypes.c_int64,
                                                  ctypes.c_double, ctypes.c_int64, ctypes.c_int64, _i64p, _dp,
                                                  _dp]),
    "nrq_heavy_create": (ctypes.c_int, [_vp, _pp]),
    "nrq_heavy_destroy": (ctypes.c_int, [_vp]),
    "nrq_heavy_upload": (ctypes.c_int, [_vp, _dp, _dp]),
    "nrq_heavy_download": (ctypes.c_int, [_vp, _dp, _dp]),
    "nrq_heavy_copy": (ctypes.c_int, [_vp, _vp]),
    "nrq_heavy_init_single_point": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64]),
    "nrq_heavy_norms": (ctypes.c_int, [_vp, _dp, _dp]),
    "nrq_heavy_correlators": (ctypes.c_int, [_vp, _dp]),
    "nrq_heavy_correlators_gconjg": (ctypes.c_int, [_vp, _dp]),
    "nrq_cn_init": (ctypes.c_int, [_vp, ctypes.c_double, _dp, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int64, ctypes.c_int, _pp]),
    "nrq_cn_finalize": (ctypes.c_int, [_vp]),
    "nrq_cn_stencil_info": (ctypes.c_int, [_vp, _ip, _dp]),
    "nrq_cn_set_wait_test": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int]),
    "nrq_cn_set_stencil": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_cn_set_cheb_stencil": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_cn_set_true_residual": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_cn_set_history_depth": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_cn_set_merged_update": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_cn_true_residual_info": (ctypes.c_int, [_vp, _ip]),
    "nrq_cn_batch_set_variant": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "nrq_cn_batch_set_fp64": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_cn_batch_fp64_info": (ctypes.c_int, [_vp, _ip, _dp]),
    "nrq_cn_batch_learned_info": (ctypes.c_int, [_vp, _ip, _dp, _dp]),
    "nrq_cn_batch_prediction_info": (ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_int64)]),
    "nrq_cn_batch_set_history": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_cn_cheb_info": (ctypes.c_int, [_vp, _ip, _dp]),
    "nrq_cn_set_history_guess": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_heavy_update_cn": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, _dp, ctypes.c_double,
                                           ctypes.POINTER(CnStats)]),
    "nrq_cn_apply": (ctypes.c_int, [_vp, _vp, ctypes.c_double, _dp, ctypes.c_double, ctypes.c_int, _vp, _vp]),
    "nrq_cn_batch_create": (ctypes.c_int, [_vp, ctypes.c_int, _pp, _dp, ctypes.c_double, _pp]),
    "nrq_cn_batch_destroy": (ctypes.c_int, [_vp]),
    "nrq_cn_batch_update": (ctypes.c_int, [_vp, _vp, _dp, ctypes.c_double, ctypes.c_int,
                                           ctypes.POINTER(CnStats)]),
    "nrq_cn_batch_residuals": (ctypes.c_int, [_vp, _dp]),
    "nrq_cn_batch_attach_learned": (ctypes.c_int, [_vp, _vp]),
    "nrq_cn_batch_info": (ctypes.c_int, [_vp, _ip, _ip, _dp, _ip, _ip]),
    "nrq_ensemble_create": (ctypes.c_int, [ctypes.c_int, _pp, _pp, _pp]),
    "nrq_ensemble_destroy": (ctypes.c_int, [_vp]),
    "nrq_ensemble_step": (ctypes.c_int, [_vp, _dp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(CnStats)]),
    "nrq_learn_create": (ctypes.c_int, [_vp, ctypes.c_uint64, _pp]),
    "nrq_learn_destroy": (ctypes.c_int, [_vp]),
    "nrq_learn_params": (ctypes.c_int, [_vp, _fp, ctypes.c_int]),
    "nrq_learn_set_trained": (ctypes.c_int, [_vp, ctypes.c_int]),
    "nrq_learn_dataset_reserve": (ctypes.c_int, [_vp, ctypes.c_int64]),
    "nrq_learn_dataset_size": (ctypes.c_int, [_vp, _i64p]),
    "nrq_learn_dataset_read": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, _fp, _fp]),
    "nrq_learn_record": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double, _dp, ctypes.c_double,
                                        ctypes.POINTER(CnStats)]),
    "nrq_learn_train": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_uint64,
                                       _dp, _dp]),
    "nrq_learn_loss_grad": (ctypes.c_int, [_vp, _fp, _fp, ctypes.c_int64, _dp, _fp]),
    "nrq_learn_forward": (ctypes.c_int, [_vp, _fp, ctypes.c_int64, _fp]),
    "nrq_cn_attach_learned": (ctypes.c_int, [_vp, _vp]),
    "nrq_gauge_energy_noalloc": (ctypes.c_int, [_i64p, _dp, _vp, _vp, _vp, _vp]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise NrqcdError(f"CUDA extension not built: {path} missing (run python -m nrqcd_b200.build)")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(rc: int, ctx=None, what: str = ""):
    if rc != NRQ_OK:
        lib = load()
        msg = lib.nrq_status_string(rc).decode()
        detail = lib.nrq_last_error(ctx).decode() if ctx else ""
        raise NrqcdError(f"{what}: {msg}" + (f" ({detail})" if detail else ""), rc)


def dptr(a: np.ndarray):
    if not a.flags.c_contiguous:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(_dp)


def coeffs(c) -> np.ndarray:
    """Wilson coefficients (4 complex) as 8 interleaved doubles."""
    c = np.asarray(c, dtype=np.complex128).reshape(4)
    out = np.empty(8)
    out[0::2] = c.real
    out[1::2] = c.imag
    return out


PROFILE_CLASSES = ("cn_stencil", "cn_vector", "cn_scalar", "cn_prepare", "leapfrog_links", "leapfrog_efield")


def profile_enable(ctx, enable=True):
    check(load().nrq_profile_enable(ctx, int(bool(enable))), ctx, "profile_enable")


def profile_read(ctx) -> dict:
    """Per kernel class: launches, device ms (CUDA events) and algorithmic bytes."""
    n = np.zeros(6, dtype=np.int64)
    ms = np.zeros(6)
    by = np.zeros(6)
    check(load().nrq_profile_read(ctx, n.ctypes.data_as(_i64p), dptr(ms), dptr(by)), ctx, "profile_read")
    return {name: {"launches": int(n[k]), "ms": float(ms[k]), "bytes": float(by[k])}
            for k, name in enumerate(PROFILE_CLASSES)}
