"""Lattice module: host mirror of ``lattice%InitModule`` (src/lattice.f90:124-228).

On one GPU the whole periodic lattice lives in one device's memory, so the
reference's MPI domain decomposition and halo lists (src/halocomm.f90) become
periodic indexing inside the kernels.  ``InitModule`` creates the device
context every other object of this package is bound to.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi

modulename = "lattice"

_ctx = None
_extents = None
_spacings = None


def InitModule(LatticeExtensions, LatticeSpacings, device: int = 0):
    """Extents (Nx,Ny,Nz) and spacings (a0,ax,ay,az) as in the reference."""
    global _ctx, _extents, _spacings
    if _ctx is not None:
        raise _capi.NrqcdError(f"Error in init of {modulename}: already initialised.",
                               _capi.NRQ_ERR_ALREADY_INITIALISED)
    ext = np.ascontiguousarray(LatticeExtensions, dtype=np.int64).reshape(3)
    sp = np.ascontiguousarray(LatticeSpacings, dtype=np.float64).reshape(4)
    lib = _capi.load()
    h = ctypes.c_void_p()
    rc = lib.nrq_init(ext.ctypes.data_as(_capi._i64p), _capi.dptr(sp), int(device), ctypes.byref(h))
    _capi.check(rc, None, f"Error in init of {modulename}")
    _ctx, _extents, _spacings = h, ext.copy(), sp.copy()


def FinalizeModule():
    global _ctx
    if _ctx is None:
        raise _capi.NrqcdError(f"Error in finalization of {modulename}: is not initialised.",
                               _capi.NRQ_ERR_NOT_INITIALISED)
    _capi.load().nrq_finalize(_ctx)
    _ctx = None


def IsModuleInitialised() -> bool:
    return _ctx is not None


def context():
    if _ctx is None:
        raise _capi.NrqcdError(f"Error in {modulename}: is not initialised.", _capi.NRQ_ERR_NOT_INITIALISED)
    return _ctx


def GetLatticeExtension(i: int) -> int:
    return int(_extents[i - 1])


def GetLatticeSpacing(i: int) -> float:
    return float(_spacings[i])


def GetLatticeSize() -> int:
    return int(np.prod(_extents))


def GetVolume() -> float:
    return float(np.prod(_extents * _spacings[1:]))


def synchronize():
    _capi.check(_capi.load().nrq_synchronize(context()), context(), "synchronize")


class Lattice:
    """A standalone lattice context beside the module's own, for ensembles
    whose members have different extents (nrq_init per member size).  Pass
    it as ``lat=`` to GaugeConfiguration and NRQCDField."""

    def __init__(self, LatticeExtensions, LatticeSpacings, device: int = 0):
        ext = np.ascontiguousarray(LatticeExtensions, dtype=np.int64).reshape(3)
        sp = np.ascontiguousarray(LatticeSpacings, dtype=np.float64).reshape(4)
        h = ctypes.c_void_p()
        rc = _capi.load().nrq_init(ext.ctypes.data_as(_capi._i64p), _capi.dptr(sp), int(device), ctypes.byref(h))
        _capi.check(rc, None, f"Error in init of {modulename}")
        self.ctx = h
        self.extents = ext.copy()
        self.spacings = sp.copy()
        self.V = int(np.prod(ext))

    @property
    def is_open(self) -> bool:
        return bool(self.ctx)

    def close(self):
        if self.ctx:
            _capi.load().nrq_finalize(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _resolve(lat):
    """(ctx, V, is_open) of a standalone Lattice, or of the module context."""
    if lat is None:
        # the object belongs to this module context: once it is finalised (or
        # replaced by a new InitModule), the object's handle is stale
        c = context()
        return c, GetLatticeSize(), (lambda: _ctx is c)
    return lat.ctx, lat.V, lambda: lat.is_open
