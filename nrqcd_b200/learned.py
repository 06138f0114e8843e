"""Learned initial guess of the Crank-Nicolson solve (form 2).

A per-sample (site, species) MLP, 16 -> 64 -> 64 -> 6 with BF16 weights on
the tensor cores, predicts complex weights (w0, w1, w2) of the start
    x0 = 2 b - psi + w0 |tau| (b - psi) + w1 v1 + w2 v2
of the solve A^H x = b (b = A psi), v1 and v2 being what the extrapolation
2 b - psi missed in the field's previous two steps.  It is trained on the method's own
solves (``record`` then ``train``); the solve's FP64 residual check decides
convergence with or without it.  No counterpart in the reference, whose
PETSc solve starts from zero (src/nrqcd.f90:1108-1123; the solution vector
holds psi, but KSPSetInitialGuessNonzero is never called).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi, lattice, nrqcd

NPARAMS = 5668
NFEATURES = 16
NSTATS = 16
NOUT = 6
FORM_LEARNED = 2


def _fptr(a):
    if a.dtype != np.float32 or not a.flags.c_contiguous:
        raise ValueError("float32 C-contiguous array required")
    return a.ctypes.data_as(_capi._fp)


class LearnedGuess:
    def __init__(self, seed: int = 1, lat=None):
        self._ctx, _, self._open = lattice._resolve(lat)
        self._h = ctypes.c_void_p()
        _capi.check(_capi.load().nrq_learn_create(self._ctx, int(seed), ctypes.byref(self._h)), self._ctx,
                    "nrq_learn_create")

    @property
    def handle(self):
        return self._h

    def Destructor(self):
        if self._h:
            _capi.load().nrq_learn_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            if self._open():
                self.Destructor()
        except Exception:
            pass

    def _call(self, name, *args):
        _capi.check(getattr(_capi.load(), name)(self._h, *args), self._ctx, name)

    # ---------------------------------------------------------- parameters
    @property
    def params(self) -> np.ndarray:
        p = np.zeros(NPARAMS, dtype=np.float32)
        self._call("nrq_learn_params", _fptr(p), 0)
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32).reshape(NPARAMS)
        self._call("nrq_learn_params", _fptr(p), 1)

    def set_trained(self, trained: bool = True):
        self._call("nrq_learn_set_trained", int(bool(trained)))

    # ---------------------------------------------------------- data
    def reserve(self, max_samples: int):
        self._call("nrq_learn_dataset_reserve", int(max_samples))

    def size(self) -> int:
        n = ctypes.c_int64()
        self._call("nrq_learn_dataset_size", ctypes.byref(n))
        return n.value

    def read(self, first: int, count: int):
        f = np.zeros((count, NFEATURES), dtype=np.float32)
        s = np.zeros((count, NSTATS), dtype=np.float32)
        self._call("nrq_learn_dataset_read", int(first), int(count), _fptr(f), _fptr(s))
        return f, s

    def record(self, field, gauge, mass, WilsonCoeffs, StepWidth=1.0, cn=None) -> dict:
        """One CN step of ``field`` that appends its samples to the dataset."""
        st = _capi.CnStats()
        c = _capi.coeffs(WilsonCoeffs)
        cn = nrqcd.solver_handle() if cn is None else cn
        self._call("nrq_learn_record", cn, field.handle, gauge.handle, float(mass), _capi.dptr(c),
                   float(StepWidth), ctypes.byref(st))
        return st.as_dict()

    # ---------------------------------------------------------- training
    def train(self, iterations: int, batch: int = 8192, lr: float = 2e-3, seed: int = 1):
        l0, l1 = ctypes.c_double(), ctypes.c_double()
        self._call("nrq_learn_train", int(iterations), int(batch), float(lr), int(seed), ctypes.byref(l0),
                   ctypes.byref(l1))
        return l0.value, l1.value

    def loss_grad(self, features, stats):
        f = np.ascontiguousarray(features, dtype=np.float32)
        s = np.ascontiguousarray(stats, dtype=np.float32)
        loss = ctypes.c_double()
        g = np.zeros(NPARAMS, dtype=np.float32)
        self._call("nrq_learn_loss_grad", _fptr(f), _fptr(s), f.shape[0], ctypes.byref(loss), _fptr(g))
        return loss.value, g

    def forward(self, features) -> np.ndarray:
        f = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros((f.shape[0], NOUT), dtype=np.float32)
        self._call("nrq_learn_forward", _fptr(f), f.shape[0], _fptr(out))
        return out

    # ---------------------------------------------------------- use
    def attach(self, cn=None):
        """Initial guess of the nrqcd module's solver (form 2)."""
        cn = nrqcd.solver_handle() if cn is None else cn
        _capi.check(_capi.load().nrq_cn_attach_learned(cn, self._h), self._ctx, "attach")

    @staticmethod
    def detach(cn=None):
        cn = nrqcd.solver_handle() if cn is None else cn
        _capi.check(_capi.load().nrq_cn_attach_learned(cn, None), None, "detach")


def train_on_seeded_configs(extent=32, configs=(1, 2), steps=6, mass=1.0, WilsonCoeffs=(1, 1, 1, 1),
                            spacings=(0.05, 1.0, 1.0, 1.0), tol=1e-10, iterations=600, batch=8192, lr=2e-3,
                            init_seed=5, train_seed=7, device=0, Q=0.5, n0=1.0, masses=None):
    """Train the guess on the method's own solves: for every seed in
    ``configs`` and every heavy mass in ``masses`` (default: ``mass``) a
    transverse-polarised occupation field (saturation Q, amplitude n0,
    identity links) on an ``extent``^3 lattice and one point source at a
    seeded random site evolve ``steps`` coupled steps (precision form at
    ``tol``, then the leapfrog), every CN step recording 2 V samples.
    Returns (params, info); the parameters load into a LearnedGuess of any
    lattice size."""
    masses = tuple(masses) if masses is not None else (mass,)
    from .gaugeconfiguration_su3 import GaugeConfiguration
    from .nrqcd import NRQCDField
    lat = lattice.Lattice((extent, extent, extent), spacings, device=device)
    try:
        lib = _capi.load()
        cn = ctypes.c_void_p()
        c = _capi.coeffs(WilsonCoeffs)
        _capi.check(lib.nrq_cn_init(lat.ctx, float(mass), _capi.dptr(c), 1.0, float(tol), 10000, 1,
                                    ctypes.byref(cn)), lat.ctx, "nrq_cn_init")
        net = LearnedGuess(seed=init_seed, lat=lat)
        V = extent ** 3
        net.reserve(len(configs) * len(masses) * steps * 2 * V)
        for seed in configs:
            for m in masses:
                g = GaugeConfiguration(lat=lat)
                g.TransversePolarisedOccupiedInit_Box(Q, n0, 0.0, RandomSeed=int(seed), identity_links=True)
                h = NRQCDField(lat=lat)
                src = np.random.default_rng(int(seed)).integers(0, V, size=2) + 1
                h.InitSinglePoint(int(src[0]), int(src[1]))
                for _ in range(steps):
                    net.record(h, g, m, WilsonCoeffs, 1.0, cn=cn)
                    g.Update(1.0)
                h.Destructor()
                g.Deallocate()
        nsamples = net.size()
        l0, l1 = net.train(iterations, batch=batch, lr=lr, seed=train_seed)
        params = net.params
        net.Destructor()
        lib.nrq_cn_finalize(cn)
    finally:
        lat.close()
    return params, {"lattice": [extent] * 3, "configs": list(configs), "masses": list(masses),
                    "steps_per_config": steps,
                    "samples": nsamples, "iterations": iterations, "batch": batch,
                    "loss_first_batch": l0, "loss_last_batch": l1}
