"""Batching form of the Crank-Nicolson step: many heavy fields in one gauge
field per launch (``CNBatch``), and ensembles of independent members of
different lattice sizes stepped by one CUDA graph launch (``Ensemble``).

The reference advances one ``NRQCDField`` per ``Update`` call
(src/nrqcd.f90:1053), field after field where the driver evolves several
(src/main.f90:983-985).  A ``CNBatch`` gives every field the result of
``NRQCDField.Update`` with the precision form (form 1) at the same
tolerance; an ``Ensemble`` step is the driver's coupled step
(src/main.f90:346-348: heavy fields, then the leapfrog) for every member.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi, lattice
from .gaugeconfiguration_su3 import GaugeConfiguration
from .nrqcd import NRQCDField


class CNBatch:
    def __init__(self, fields, masses, kspTol: float, lat=None):
        ctx, _, self._open = lattice._resolve(lat)
        self._ctx = ctx
        self.fields = list(fields)
        masses = np.ascontiguousarray(masses, dtype=np.float64).reshape(len(self.fields))
        arr = (ctypes.c_void_p * len(self.fields))(*[f.handle.value for f in self.fields])
        self._h = ctypes.c_void_p()
        rc = _capi.load().nrq_cn_batch_create(ctx, len(self.fields), ctypes.cast(arr, _capi._pp),
                                              _capi.dptr(masses), float(kspTol), ctypes.byref(self._h))
        _capi.check(rc, ctx, "nrq_cn_batch_create")
        self.masses = masses.copy()
        self.last_stats = None

    @property
    def handle(self):
        return self._h

    def Destructor(self):
        if self._h:
            _capi.load().nrq_cn_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if self._open():
                self.Destructor()
        except Exception:
            pass

    def Update(self, GaugeConf: GaugeConfiguration, WilsonCoeffs, StepWidth: float = 1.0, use_graph: bool = True,
               raise_on_nonconvergence: bool = True) -> dict:
        """One CN step of every field (each with its own mass)."""
        st = _capi.CnStats()
        c = _capi.coeffs(WilsonCoeffs)
        rc = _capi.load().nrq_cn_batch_update(self._h, GaugeConf.handle, _capi.dptr(c), float(StepWidth),
                                              int(bool(use_graph)), ctypes.byref(st))
        self.last_stats = st.as_dict()
        if rc == _capi.NRQ_ERR_NOT_CONVERGED and not raise_on_nonconvergence:
            return self.last_stats
        _capi.check(rc, self._ctx, "nrq_cn_batch_update")
        return self.last_stats

    def attach_learned(self, net):
        """Start every field's solve from the learned guess of ``net`` (a
        trained nrqcd_b200.learned.LearnedGuess of the same lattice; None
        detaches)."""
        handle = net.handle if net is not None else None
        _capi.check(_capi.load().nrq_cn_batch_attach_learned(self._h, handle), self._ctx, "attach_learned")

    def residuals(self) -> np.ndarray:
        out = np.zeros(len(self.fields))
        _capi.check(_capi.load().nrq_cn_batch_residuals(self._h, _capi.dptr(out)), self._ctx, "residuals")
        return out

    VARIANTS = ("tile1_2blocks", "tile1_3blocks", "tile2_1block", "fp32_blocks_tma")

    def set_variant(self, variant=None, order=0):
        """Force the Chebyshev kernel (a name of VARIANTS or its index) and
        block order; None restores the timed choice."""
        v = -1 if variant is None else (self.VARIANTS.index(variant) if isinstance(variant, str) else int(variant))
        _capi.check(_capi.load().nrq_cn_batch_set_variant(self._h, v, int(order)), self._ctx, "set_variant")

    def set_fp64(self, which):
        """Force the FP64 stencil of the right-hand side and residuals:
        "register" (0) or "blocks" (1)."""
        w = {"register": 0, "blocks": 1}.get(which, which)
        _capi.check(_capi.load().nrq_cn_batch_set_fp64(self._h, int(w)), self._ctx, "set_fp64")

    def info(self) -> dict:
        var, order, npass = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = np.zeros(8)
        steps = (ctypes.c_int * 16)()
        _capi.check(_capi.load().nrq_cn_batch_info(self._h, ctypes.byref(var), ctypes.byref(order), _capi.dptr(ms),
                                                   ctypes.byref(npass), steps), self._ctx, "info")
        names = self.VARIANTS
        return {"variant": names[var.value], "fields_per_tile": 2 if var.value == 2 else 1,
                "block_order": order.value,
                "candidate_ms": {f"{names[v]}_order{o}": float(ms[2 * v + o]) for v in range(4) for o in range(2)},
                "schedule": [int(steps[k]) for k in range(npass.value)], **self._fp64_info()}

    def learned_info(self) -> dict:
        """The attached learned guess's gate ("none", "undecided", "on",
        "off"), its measured cost and the value of the steps it saved (ms)."""
        gate = ctypes.c_int()
        cost, saving = ctypes.c_double(), ctypes.c_double()
        _capi.check(_capi.load().nrq_cn_batch_learned_info(self._h, ctypes.byref(gate), ctypes.byref(cost),
                                                           ctypes.byref(saving)), self._ctx, "learned info")
        names = {-2: "none", -1: "undecided", 0: "off", 1: "on"}
        return {"gate": names[gate.value], "guess_ms": cost.value, "saving_ms": saving.value}

    def set_history(self, on=True):
        """Start every field from 2b - psi plus the cubic extrapolation of its
        history (True, the default) or from 2b - psi alone (False)."""
        _capi.check(_capi.load().nrq_cn_batch_set_history(self._h, int(bool(on))), self._ctx, "set history")

    def prediction_info(self) -> dict:
        """The scheduled steps' predicted acceptance: the largest measured
        ratio of true to predicted residual (-1 before the first) and the
        scheduled steps taken."""
        ratio, steps = ctypes.c_double(), ctypes.c_int64()
        _capi.check(_capi.load().nrq_cn_batch_prediction_info(self._h, ctypes.byref(ratio), ctypes.byref(steps)),
                    self._ctx, "prediction info")
        return {"ratio": ratio.value, "steps": steps.value}

    def _fp64_info(self) -> dict:
        which = ctypes.c_int()
        ms = np.zeros(2)
        _capi.check(_capi.load().nrq_cn_batch_fp64_info(self._h, ctypes.byref(which), _capi.dptr(ms)), self._ctx,
                    "fp64 info")
        names = ("register", "blocks")
        return {"fp64_stencil": names[which.value], "fp64_candidate_ms": {n: float(ms[k]) for k, n in enumerate(names)}}


class Ensemble:
    """Members (batch, gauge) stepped together; with use_graph every step
    after the calibration is one CUDA graph launch."""

    def __init__(self, batches, gauges):
        self.batches = list(batches)
        self.gauges = list(gauges)
        n = len(self.batches)
        bh = (ctypes.c_void_p * n)(*[b.handle.value for b in self.batches])
        gh = (ctypes.c_void_p * n)(*[g.handle.value for g in self.gauges])
        self._h = ctypes.c_void_p()
        rc = _capi.load().nrq_ensemble_create(n, ctypes.cast(bh, _capi._pp), ctypes.cast(gh, _capi._pp),
                                              ctypes.byref(self._h))
        _capi.check(rc, None, "nrq_ensemble_create")
        self.last_stats = None

    def Destructor(self):
        if self._h:
            _capi.load().nrq_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Destructor()
        except Exception:
            pass

    def Step(self, WilsonCoeffs, StepWidth: float, use_graph: bool = True,
             raise_on_nonconvergence: bool = True) -> dict:
        st = _capi.CnStats()
        c = _capi.coeffs(WilsonCoeffs)
        rc = _capi.load().nrq_ensemble_step(self._h, _capi.dptr(c), float(StepWidth), int(bool(use_graph)),
                                            ctypes.byref(st))
        self.last_stats = st.as_dict()
        if rc == _capi.NRQ_ERR_NOT_CONVERGED and not raise_on_nonconvergence:
            return self.last_stats
        _capi.check(rc, self.batches[0]._ctx, "nrq_ensemble_step")
        return self.last_stats


__all__ = ["CNBatch", "Ensemble", "NRQCDField", "GaugeConfiguration"]
