"""Host mirror of ``type(GaugeConfiguration)`` (src/gaugeconfiguration_su3.f90:33-116).

The fields live on the device in structure-of-arrays planes; ``links`` and
``efield`` are host copies in the reference's Fortran layouts, synchronised
only by ``download``/``upload`` (or the properties):

* links  complex128 (V, 3, 3, 3) = Fortran links(3,3,3,V) read [site, dir, col, row]
* efield float64    (V, 3, 8)    = Fortran efield(8,3,V) read [site, dir, a]
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi, lattice

modulename = "gaugeconfiguration_su3"


class GaugeConfiguration:
    def __init__(self, lat=None):
        """lat: a lattice.Lattice (ensemble member); default the module context."""
        self._ctx, self.V, self._open = lattice._resolve(lat)
        self._h = ctypes.c_void_p()
        lib = _capi.load()
        _capi.check(lib.nrq_gauge_create(self._ctx, ctypes.byref(self._h)), self._ctx,
                    f"Error in Allocate of {modulename}")

    # --------------------------------------------------------------- lifetime
    def Deallocate(self):
        if self._h:
            _capi.load().nrq_gauge_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if self._open():
                self.Deallocate()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def _call(self, name, *args):
        _capi.check(getattr(_capi.load(), name)(self._h, *args), self._ctx, f"{modulename}:{name}")

    # --------------------------------------------------------------- data
    def upload(self, links: np.ndarray, efield: np.ndarray):
        links = np.ascontiguousarray(links, dtype=np.complex128).reshape(self.V, 3, 3, 3)
        efield = np.ascontiguousarray(efield, dtype=np.float64).reshape(self.V, 3, 8)
        self._call("nrq_gauge_upload", links.ctypes.data_as(_capi._dp), efield.ctypes.data_as(_capi._dp))

    def download(self, links: np.ndarray | None = None, efield: np.ndarray | None = None):
        if links is None:
            links = np.empty((self.V, 3, 3, 3), dtype=np.complex128)
        if efield is None:
            efield = np.empty((self.V, 3, 8), dtype=np.float64)
        self._call("nrq_gauge_download", links.ctypes.data_as(_capi._dp), efield.ctypes.data_as(_capi._dp))
        return links, efield

    @property
    def links(self):
        return self.download()[0]

    @property
    def efield(self):
        return self.download()[1]

    def assign(self, other: "GaugeConfiguration"):
        _capi.check(_capi.load().nrq_gauge_copy(self._h, other._h), self._ctx, "GaugeConfiguration copy")

    # --------------------------------------------------------------- inits
    def ColdInit(self):
        """src/gaugeconfiguration_su3.f90:363-378"""
        self._call("nrq_gauge_cold_init")

    def TransversePolarisedOccupiedInit_Box(self, SaturationScale, Amplitude, Coupling, RandomSeed=1,
                                            identity_links=False):
        """src/gaugeconfiguration_su3.f90:906-951 after random%InitModule(RandomSeed)."""
        self._call("nrq_gauge_transverse_box_init", float(SaturationScale), float(Amplitude), float(Coupling),
                   int(RandomSeed), int(bool(identity_links)))

    # --------------------------------------------------------------- evolution
    def Update(self, StepWidth_: float = 1.0):
        """Update_Leapfrog, src/gaugeconfiguration_su3.f90:2082-2111"""
        self._call("nrq_gauge_update", float(StepWidth_))

    # --------------------------------------------------------------- observables
    def SetPrecision(self, prec: int = 1, reunit_every: int = 10):
        """prec 1: FP32 links in the leapfrog with FP64 reunitarisation every
        reunit_every steps; prec 0: FP64 (the reference's precision)."""
        self._call("nrq_gauge_set_precision", int(prec), int(reunit_every))

    def GetUnitarityDeviation(self):
        """(max |U U^+ - 1|, max |det U - 1|) over all links."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._call("nrq_gauge_unitarity", ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def GetEnergy(self) -> float:
        e = ctypes.c_double()
        self._call("nrq_gauge_energy", ctypes.byref(e))
        return e.value

    def _gauss(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._call("nrq_gauge_gauss", ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def GetDeviationFromGaussLaw(self) -> float:
        """src/gaugeconfiguration_su3.f90:1480-1531 (sum of 2|Im Tr(T^a D)|)."""
        return self._gauss()[0]

    def GetGdeviation(self) -> float:
        """Max-norm Gauss residual of EquilibriumInit (src/gaugeconfiguration_su3.f90:724-768)."""
        return self._gauss()[1]
