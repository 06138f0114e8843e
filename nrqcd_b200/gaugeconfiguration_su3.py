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


def _list_real8(x: float) -> str:
    """A real(8) item of gfortran's list-directed output: 17 significant
    digits, fixed form for 0.1 <= |x| < 1e16 (five blanks where the exponent
    would be), otherwise E form with a three-digit exponent; 26 characters."""
    ax = abs(x)
    if x != x or ax in (float("inf"),):
        return ("NaN" if x != x else ("-" if x < 0 else "") + "Infinity").rjust(26)
    if ax == 0.0 or 0.1 <= ax < 1e16:
        e = 0 if ax == 0.0 else int(np.floor(np.log10(ax)))
        body = f"{x:.{max(16 - e, 0)}f}"
        if len(body.lstrip("-").split(".")[0]) > e + 1 and ax != 0.0:  # rounding carried into a new digit
            body = f"{x:.{max(15 - e, 0)}f}"
        return (body + " " * 5).rjust(26)
    m, ex = f"{x:.16E}".split("E")
    return f"{m}E{int(ex):+04d}".rjust(26)


def list_directed(items) -> str:
    """One record of gfortran list-directed output: default integers as I12,
    numpy int64 (integer(int64)) as I21, reals as _list_real8, character
    items as themselves after one blank."""
    out = []
    for v in items:
        if isinstance(v, str):
            out.append(" " + v)
        elif isinstance(v, np.int64):  # integer(int64): I21
            out.append(f"{int(v):21d}")
        elif isinstance(v, (int, np.integer)):  # default integer: I12
            out.append(f"{int(v):12d}")
        else:
            out.append(_list_real8(float(v)))
    return "".join(out)


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

    def EquilibriumInit(self, Beta, nefieldinit, nequilibrium, tolerance_Eprojection=1e-3, MeasureEnergy=False,
                        filename=None, RandomSeed=1, max_sweeps=0, verbose=True):
        """EquilibriumInit, src/gaugeconfiguration_su3.f90:380-814 (no charge
        density), after random%InitModule(RandomSeed).  With MeasureEnergy the
        energy after each round is written to `filename` as the reference's
        list-directed `iefieldinit, energy` records, and echoed to stdout;
        every round prints its Gauss deviation ('G[U,E]=').  Returns per round
        the projection sweeps, the energies and the deviations."""
        if MeasureEnergy and not filename:
            raise _capi.NrqcdError("Filename for energy output missing")
        n = int(nefieldinit)
        sweeps = np.zeros(max(n, 1), dtype=np.int64)
        en = np.zeros(max(n, 1))
        dev = np.zeros(max(n, 1))
        self._call("nrq_gauge_equilibrium_init", float(Beta), n, int(nequilibrium), float(tolerance_Eprojection),
                   int(RandomSeed), int(max_sweeps), sweeps.ctypes.data_as(_capi._i64p), _capi.dptr(en),
                   _capi.dptr(dev))
        if MeasureEnergy:
            with open(filename, "w") as f:
                for r in range(n):
                    f.write(list_directed((r + 1, float(en[r]))) + "\n")
        if verbose:
            for r in range(n):
                if MeasureEnergy:
                    print(list_directed((r + 1, float(en[r]))), flush=True)
                print(list_directed(("G[U,E]=", float(dev[r]))), flush=True)
        return sweeps[:n], en[:n], dev[:n]

    def CoulombGaugefixing(self, Tolerance_=1e-8, alpha_=0.08, MaxIterations_=100, verbose=True):
        """CoulombGaugefixing (src/gaugeconfiguration_su3.f90:2269-2456):
        Fourier-accelerated gauge fixing of the links to Coulomb gauge.
        Prints, as the reference does, the divergence checked at every
        iteration and the final loop counter.  Returns (loop counter,
        deviations)."""
        n = int(MaxIterations_)
        dev = np.full(max(n, 1), np.nan)
        it = ctypes.c_int64()
        self._call("nrq_gauge_coulomb_gaugefix", float(Tolerance_), float(alpha_), n, ctypes.byref(it),
                   _capi.dptr(dev))
        checked = dev[:min(it.value, n)]
        if verbose:
            for d in checked:
                print(list_directed((float(d),)), flush=True)
            print(list_directed((np.int64(it.value), "iterations in Coulomb gauge fixing performed")), flush=True)
        return it.value, checked

    def GetTransverseCorrelators(self):
        """(AA, EE, |p|) per momentum site in lattice order
        (src/gaugeconfiguration_su3.f90:1825-1972, src/lattice.f90:1081-1089)."""
        aa, ee, mom = np.empty(self.V), np.empty(self.V), np.empty(self.V)
        self._call("nrq_gauge_transverse_correlators", _capi.dptr(aa), _capi.dptr(ee), _capi.dptr(mom))
        return aa, ee, mom

    def GetTransverseAACorrelator(self):
        """src/gaugeconfiguration_su3.f90:1825-1859"""
        return self.GetTransverseCorrelators()[0]

    def GetTransverseEECorrelator(self):
        """src/gaugeconfiguration_su3.f90:1867-1905"""
        return self.GetTransverseCorrelators()[1]

    def GaussProjection(self, tolerance=1e-3, max_sweeps=0):
        """The Gauss projection loop of EquilibriumInit
        (src/gaugeconfiguration_su3.f90:455-500) on the current
        configuration; returns (sweeps, final deviation)."""
        sw, d = ctypes.c_int64(), ctypes.c_double()
        self._call("nrq_gauge_gauss_project", float(tolerance), int(max_sweeps), ctypes.byref(sw), ctypes.byref(d))
        return sw.value, d.value

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
