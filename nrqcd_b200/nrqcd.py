"""Host mirror of the ``nrqcd`` module (src/nrqcd.f90).

``InitModule``/``FinalizeModule`` hold the solver state the reference keeps
in module globals (src/nrqcd.f90:120-158); ``NRQCDField`` mirrors
``type(NRQCDField)`` (src/nrqcd.f90:58-117).  Propagators live on the device;
``QuarkProp``/``AntiQProp`` download host copies in the reference's layout
prop(6,6,V) read as complex128 (V, 6, 6) [site, col, row].
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi, lattice
from .gaugeconfiguration_su3 import GaugeConfiguration

modulename = "nrqcd"
nDof = 6
nWilsonCoefficients = 4

_cn = None
_settings = None

FORM_PLAIN_FP64 = 0
FORM_PRECISION = 1  # FP32 Chebyshev inner iterations in FP64 iterative refinement
FORM_LEARNED = 2    # precision form started from the learned guess (nrqcd_b200.learned)


def InitModule(Mass, WilsonCoeffs, StepWidth, kspTol, maxits=10000, form=FORM_PLAIN_FP64):
    """src/nrqcd.f90:167-192 (kspTol = relative residual of every column solve)."""
    global _cn, _settings
    if _cn is not None:
        raise _capi.NrqcdError(f"Error in init of {modulename}: already initialised.",
                               _capi.NRQ_ERR_ALREADY_INITIALISED)
    if not lattice.IsModuleInitialised():
        raise _capi.NrqcdError(f"Error in init of {modulename}: lattice is not initialised.",
                               _capi.NRQ_ERR_NOT_INITIALISED)
    ctx = lattice.context()
    c = _capi.coeffs(WilsonCoeffs)
    h = ctypes.c_void_p()
    rc = _capi.load().nrq_cn_init(ctx, float(Mass), _capi.dptr(c), float(StepWidth), float(kspTol),
                                  int(maxits), int(form), ctypes.byref(h))
    _capi.check(rc, ctx, f"Error in init of {modulename}")
    _cn = h
    _settings = dict(Mass=float(Mass), WilsonCoeffs=c, StepWidth=float(StepWidth), kspTol=float(kspTol))


def FinalizeModule():
    global _cn
    if _cn is None:
        raise _capi.NrqcdError(f"Error in finalization of {modulename}: is not initialised.",
                               _capi.NRQ_ERR_NOT_INITIALISED)
    _capi.load().nrq_cn_finalize(_cn)
    _cn = None


def IsModuleInitialised() -> bool:
    return _cn is not None


def solver_handle():
    if _cn is None:
        raise _capi.NrqcdError(f"Error in {modulename}: is not initialised.", _capi.NRQ_ERR_NOT_INITIALISED)
    return _cn


STENCIL_REGISTER = 0  # register-tiled FP64 stencil (k_cn_mv2)
STENCIL_TMA = 1       # TMA-staged FP64 stencil (k_cn_mv3)
STENCIL_TENSOR = 2    # FP64 tensor-core stencil on per-update 6x6 blocks (k_cn_mv4)
STENCIL_FMA = 3       # FP64 FMA stencil on the same per-update blocks (k_cn_mv5)
STENCIL_NAMES = {STENCIL_REGISTER: "k_cn_mv2 (register-tiled)", STENCIL_TMA: "k_cn_mv3 (TMA-staged)",
                 STENCIL_TENSOR: "k_cn_mv4 (FP64 tensor cores)", STENCIL_FMA: "k_cn_mv5 (FP64 FMA on cached blocks)"}


def SetStencil(stencil=None):
    """Force the solver's FP64 stencil (STENCIL_*); None restores the choice
    timed on the next update."""
    ctx = lattice.context()
    _capi.check(_capi.load().nrq_cn_set_stencil(solver_handle(), -1 if stencil is None else int(stencil)), ctx,
                f"Error in {modulename}: stencil")


CHEB_REGISTER, CHEB_BLOCKS = 0, 1


def SetChebStencil(which=None):
    """Precision forms: force the FP32 Chebyshev step (CHEB_REGISTER: the
    operator assembled per launch; CHEB_BLOCKS: FP32 blocks staged by TMA);
    None restores the default (blocks where the lattice allows)."""
    _capi.check(_capi.load().nrq_cn_set_cheb_stencil(solver_handle(), -1 if which is None else int(which)),
                lattice.context(), f"Error in {modulename}: Chebyshev stencil")


def ChebInfo(with_times=False):
    """The FP32 Chebyshev step the last update ran (CHEB_*; -1 before any);
    with_times: also the per-launch ms of each step timed on the first
    update (-1 where not timed)."""
    last = ctypes.c_int()
    ms = np.zeros(2)
    _capi.check(_capi.load().nrq_cn_cheb_info(solver_handle(), ctypes.byref(last), _capi.dptr(ms)),
                lattice.context(), f"Error in {modulename}: Chebyshev info")
    return (int(last.value), ms) if with_times else int(last.value)


def SetMergedUpdate(on=True):
    """Plain form on the FMA stencil: update x, r and p of an iteration in one
    pass (on=True, the default) or in two (x and r, then p)."""
    _capi.check(_capi.load().nrq_cn_set_merged_update(solver_handle(), int(bool(on))), lattice.context(),
                f"Error in {modulename}: merged update")


def SetTrueResidual(always=True):
    """Confirm every converged solve with the true residual (always=True), or
    (False, the default) accept the plain form's recursive residual, or the
    precision forms' Chebyshev prediction, where it meets the tolerance with
    a margin measured on the solver's confirmed solves."""
    _capi.check(_capi.load().nrq_cn_set_true_residual(solver_handle(), int(bool(always))), lattice.context(),
                f"Error in {modulename}: true residual")


def LastResidualIsTrue():
    """Whether the last update's max_rel_residual is the true residual."""
    v = ctypes.c_int()
    _capi.check(_capi.load().nrq_cn_true_residual_info(solver_handle(), ctypes.byref(v)), lattice.context(),
                f"Error in {modulename}: true residual info")
    return bool(v.value)


def SetHistoryDepth(depth=4):
    """Plain form: the history vectors (1-4) the extrapolated start uses."""
    _capi.check(_capi.load().nrq_cn_set_history_depth(solver_handle(), int(depth)), lattice.context(),
                f"Error in {modulename}: history depth")


def SetHistoryGuess(on=True):
    """Plain form: start each solve from the extrapolation 2b - psi plus
    2 t1 - t2 of the field's last two corrections (FP32 history; the
    default), or from 2b - psi alone (on=False)."""
    _capi.check(_capi.load().nrq_cn_set_history_guess(solver_handle(), int(bool(on))), lattice.context(),
                f"Error in {modulename}: history guess")


def SetWaitTest(wait_cycles=0, stall_load=-1):
    """Test hook of the FMA stencil's bounded pipeline waits: the bound in
    clock cycles (0: the default, about two seconds) and the load its loader
    stops before (-1: none), so that the wait for it runs out."""
    _capi.check(_capi.load().nrq_cn_set_wait_test(solver_handle(), int(wait_cycles), int(stall_load)),
                lattice.context(), f"Error in {modulename}: wait test")


def StencilInfo():
    """(stencil in use, per-launch ms of each stencil timed on the first
    update; -1 where not timed)."""
    which = ctypes.c_int()
    ms = np.zeros(4)
    _capi.check(_capi.load().nrq_cn_stencil_info(solver_handle(), ctypes.byref(which), _capi.dptr(ms)),
                lattice.context(), f"Error in {modulename}: stencil info")
    return int(which.value), ms


class NRQCDField:
    def __init__(self, lat=None):
        """lat: a lattice.Lattice (ensemble member); default the module context."""
        self._ctx, self.V, self._open = lattice._resolve(lat)
        self._h = ctypes.c_void_p()
        _capi.check(_capi.load().nrq_heavy_create(self._ctx, ctypes.byref(self._h)), self._ctx,
                    f"Error in Allocate of {modulename}")
        self.last_stats = None

    def Destructor(self):
        if self._h:
            _capi.load().nrq_heavy_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if self._open():
                self.Destructor()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def _call(self, name, *args):
        _capi.check(getattr(_capi.load(), name)(self._h, *args), self._ctx, f"{modulename}:{name}")

    # ------------------------------------------------------------ data
    def upload(self, quark: np.ndarray, antiq: np.ndarray):
        q = np.ascontiguousarray(quark, dtype=np.complex128).reshape(self.V, 6, 6)
        a = np.ascontiguousarray(antiq, dtype=np.complex128).reshape(self.V, 6, 6)
        self._call("nrq_heavy_upload", q.ctypes.data_as(_capi._dp), a.ctypes.data_as(_capi._dp))

    def download(self, quark=None, antiq=None):
        if quark is None:
            quark = np.empty((self.V, 6, 6), dtype=np.complex128)
        if antiq is None:
            antiq = np.empty((self.V, 6, 6), dtype=np.complex128)
        self._call("nrq_heavy_download", quark.ctypes.data_as(_capi._dp), antiq.ctypes.data_as(_capi._dp))
        return quark, antiq

    @property
    def QuarkProp(self):
        return self.download()[0]

    @property
    def AntiQProp(self):
        return self.download()[1]

    def Assign(self, other: "NRQCDField"):
        """assignment(=), src/nrqcd.f90:219-228"""
        _capi.check(_capi.load().nrq_heavy_copy(self._h, other._h), self._ctx, "NRQCDField assign")

    # ------------------------------------------------------------ inits
    def InitSinglePoint(self, LatticeIndex_quark: int, LatticeIndex_antiq: int):
        """src/nrqcd.f90:324-350 (1-based lattice indices)."""
        self._call("nrq_heavy_init_single_point", int(LatticeIndex_quark), int(LatticeIndex_antiq))

    # ------------------------------------------------------------ evolution
    def Update(self, GaugeConf: GaugeConfiguration, Mass, WilsonCoeffs, StepWidth: float = 1.0,
               raise_on_nonconvergence: bool = True):
        """Update_CrankNicholson, src/nrqcd.f90:1053-1168."""
        st = _capi.CnStats()
        c = _capi.coeffs(WilsonCoeffs)
        rc = _capi.load().nrq_heavy_update_cn(solver_handle(), self._h, GaugeConf.handle, float(Mass),
                                              _capi.dptr(c), float(StepWidth), ctypes.byref(st))
        self.last_stats = st.as_dict()
        if rc == _capi.NRQ_ERR_NOT_CONVERGED and not raise_on_nonconvergence:
            return self.last_stats
        _capi.check(rc, self._ctx, f"Error in Update of {modulename}")
        return self.last_stats

    # ------------------------------------------------------------ observables
    def _norms(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._call("nrq_heavy_norms", ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def GetNorm_Quark(self) -> float:
        return self._norms()[0]

    def GetNorm_AntiQ(self) -> float:
        return self._norms()[1]

    def _correlators(self):
        out = np.empty(8)
        self._call("nrq_heavy_correlators", _capi.dptr(out))
        return out[0::2] + 1j * out[1::2]

    def GetMesoncorrelator_O1_1S0_ZeroMomentum(self) -> complex:
        return complex(self._correlators()[0])

    def GetMesoncorrelator_O1_3S1_ZeroMomentum(self) -> complex:
        return complex(self._correlators()[1])

    def GetMesoncorrelator_O8_1S0_ZeroMomentum(self) -> complex:
        return complex(self._correlators()[2])

    def GetMesoncorrelator_O8_3S1_ZeroMomentum(self) -> complex:
        return complex(self._correlators()[3])

    def _correlators_gconjg(self):
        out = np.empty(8)
        self._call("nrq_heavy_correlators_gconjg", _capi.dptr(out))
        return out[0::2] + 1j * out[1::2]

    def GetMesoncorrelator_O1_1S0_ZeroMomentum_gconjg(self) -> complex:
        """src/nrqcd.f90:1728-1761"""
        return complex(self._correlators_gconjg()[0])

    def GetMesoncorrelator_O1_3S1_ZeroMomentum_gconjg(self) -> complex:
        """src/nrqcd.f90:1769-1809"""
        return complex(self._correlators_gconjg()[1])

    def GetMesoncorrelator_O8_1S0_ZeroMomentum_gconjg(self) -> complex:
        """src/nrqcd.f90:1817-1857"""
        return complex(self._correlators_gconjg()[2])

    def GetMesoncorrelator_O8_3S1_ZeroMomentum_gconjg(self) -> complex:
        """src/nrqcd.f90:1865-1905"""
        return complex(self._correlators_gconjg()[3])

    def GetMesoncorrelators_gconjg(self) -> dict:
        c = self._correlators_gconjg()
        return {"o1_1s0": complex(c[0]), "o1_3s1": complex(c[1]), "o8_1s0": complex(c[2]),
                "o8_3s1": complex(c[3])}

    def GetMesoncorrelators(self) -> dict:
        c = self._correlators()
        return {"o1_1s0": complex(c[0]), "o1_3s1": complex(c[1]), "o8_1s0": complex(c[2]),
                "o8_3s1": complex(c[3])}


def apply_operator(GaugeConf: GaugeConfiguration, Mass, WilsonCoeffs, StepWidth, herm: bool,
                   field_in: NRQCDField, field_out: NRQCDField):
    """field_out = A field_in (herm=False) or A^H field_in, quark and antiquark
    operators as assembled in BuildSystemMatrix (MatMult of src/nrqcd.f90:1112)."""
    c = _capi.coeffs(WilsonCoeffs)
    rc = _capi.load().nrq_cn_apply(solver_handle(), GaugeConf.handle, float(Mass), _capi.dptr(c),
                                   float(StepWidth), int(bool(herm)), field_in.handle, field_out.handle)
    _capi.check(rc, lattice.context(), "apply_operator")
