"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use
this module; the product never imports it.

Array layouts follow the reference's Fortran arrays with the site index
slowest (see ``oracle.h``):

* ``links``  complex128, shape (V, 3, 3, 3) indexed [site, dir, col, row]
* ``efield`` float64,    shape (V, 3, 8)    indexed [site, dir, a]
* ``prop``   complex128, shape (V, 6, 6)    indexed [site, col, row]
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


class Lattice(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64 * 3), ("a", ctypes.c_double * 4)]


class RanlxdState(ctypes.Structure):
    _fields_ = [
        ("pr", ctypes.c_int64), ("ir", ctypes.c_int64), ("jr", ctypes.c_int64),
        ("ir_old", ctypes.c_int64), ("init", ctypes.c_int64),
        ("next", ctypes.c_int64 * 12), ("one_bit", ctypes.c_double),
        ("carry", ctypes.c_double), ("xdbl", ctypes.c_double * 12),
    ]


class CnStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64 * 12),
                ("rel_residual", ctypes.c_double * 12),
                ("converged", ctypes.c_int)]


def build():
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        sig = {
            "oc_ranlxd_init": (ctypes.c_int, [ctypes.POINTER(RanlxdState), ctypes.c_int64, ctypes.c_int64]),
            "oc_ranlxd": (None, [ctypes.POINTER(RanlxdState), _dp, ctypes.c_int64]),
            "oc_ranlxd_get": (None, [ctypes.POINTER(RanlxdState), _i64p]),
            "oc_ranlxd_reset": (ctypes.c_int, [ctypes.POINTER(RanlxdState), _i64p]),
            "oc_random_normal_cmplx": (None, [ctypes.POINTER(RanlxdState), ctypes.c_int64, _dp]),
            "oc_fft3d": (None, [_dp, _i64p, ctypes.c_int, ctypes.c_double]),
            "oc_generator": (None, [ctypes.c_int, _dp]),
            "oc_algebra_matrix": (None, [_dp, _dp]),
            "oc_eigenh3": (None, [_dp, _dp, _dp]),
            "oc_eigenc3": (None, [_dp, _dp, _dp]),
            "oc_group_exp": (None, [_dp, _dp]),
            "oc_logu3": (None, [_dp, _dp]),
            "oc_gauge_cold": (None, [ctypes.POINTER(Lattice), _dp, _dp]),
            "oc_gauge_transverse_box": (ctypes.c_int, [ctypes.POINTER(Lattice), ctypes.c_double, ctypes.c_double,
                                                       ctypes.c_double, ctypes.c_int64, ctypes.c_int, _dp, _dp]),
            "oc_gauge_update": (None, [ctypes.POINTER(Lattice), _dp, _dp, ctypes.c_double]),
            "oc_gauge_energy": (ctypes.c_double, [ctypes.POINTER(Lattice), _dp, _dp]),
            "oc_gauge_gauss_ref": (ctypes.c_double, [ctypes.POINTER(Lattice), _dp, _dp]),
            "oc_gauge_gauss_maxnorm": (ctypes.c_double, [ctypes.POINTER(Lattice), _dp, _dp]),
            "oc_field_strength": (None, [ctypes.POINTER(Lattice), _dp, _dp, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int64, _dp]),
            "oc_gauge_gauss_project": (ctypes.c_int64, [ctypes.POINTER(Lattice), _dp, _dp, ctypes.c_double,
                                                        ctypes.c_int64]),
            "oc_gauge_equilibrium_init": (ctypes.c_int, [ctypes.POINTER(Lattice), ctypes.c_double, ctypes.c_int64,
                                                         ctypes.c_int64, ctypes.c_double, ctypes.c_int64,
                                                         ctypes.c_int64, _dp, _dp, _i64p, _dp, _dp]),
            "oc_heavy_init_single_point": (None, [ctypes.POINTER(Lattice), ctypes.c_int64, _dp]),
            "oc_heavy_norm": (ctypes.c_double, [ctypes.POINTER(Lattice), _dp]),
            "oc_cn_apply": (None, [ctypes.POINTER(Lattice), _dp, _dp, ctypes.c_double, _dp, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, _dp, _dp]),
            "oc_cn_update": (ctypes.c_int, [ctypes.POINTER(Lattice), _dp, _dp, ctypes.c_double, _dp,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_int,
                                            _dp, _dp, ctypes.POINTER(CnStats)]),
            "oc_meson_o1_1s0": (None, [ctypes.POINTER(Lattice), _dp, _dp, _dp]),
            "oc_meson_o1_3s1": (None, [ctypes.POINTER(Lattice), _dp, _dp, _dp]),
            "oc_meson_o8_1s0": (None, [ctypes.POINTER(Lattice), _dp, _dp, _dp]),
            "oc_meson_o8_3s1": (None, [ctypes.POINTER(Lattice), _dp, _dp, _dp]),
            "oc_meson_gconjg": (None, [ctypes.POINTER(Lattice), _dp, _dp, _dp]),
            "oc_norm2_momentum": (ctypes.c_double, [ctypes.POINTER(Lattice), ctypes.c_int64]),
            "oc_gauge_coulomb_gaugefix": (ctypes.c_int64, [ctypes.POINTER(Lattice), _dp, ctypes.c_double,
                                                           ctypes.c_double, ctypes.c_int64, _dp]),
            "oc_gauge_transverse_correlators": (None, [ctypes.POINTER(Lattice), _dp, _dp, _dp, _dp, _dp]),
            "oc_num_threads": (ctypes.c_int, []),
            "oc_set_num_threads": (None, [ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def lattice(n, a):
    L = Lattice()
    for k in range(3):
        L.n[k] = int(n[k])
    for k in range(4):
        L.a[k] = float(a[k])
    return L


def volume(n):
    return int(n[0]) * int(n[1]) * int(n[2])


# ---------------- random numbers ----------------

class Ranlxd:
    def __init__(self, level=2, seed=1):
        self.s = RanlxdState()
        rc = lib().oc_ranlxd_init(ctypes.byref(self.s), level, seed)
        if rc != 0:
            raise ValueError(f"ranlxd_init failed ({rc})")

    def draw(self, n):
        r = np.empty(n, dtype=np.float64)
        lib().oc_ranlxd(ctypes.byref(self.s), _p(r), n)
        return r

    def normal_cmplx(self, n):
        r = np.empty(2 * n, dtype=np.float64)
        lib().oc_random_normal_cmplx(ctypes.byref(self.s), n, _p(r))
        return r[0::2] + 1j * r[1::2]

    def get_state(self):
        st = np.empty(25, dtype=np.int64)
        lib().oc_ranlxd_get(ctypes.byref(self.s), st.ctypes.data_as(_i64p))
        return st

    def reset(self, st):
        st = np.ascontiguousarray(st, dtype=np.int64)
        rc = lib().oc_ranlxd_reset(ctypes.byref(self.s), st.ctypes.data_as(_i64p))
        if rc != 0:
            raise ValueError("ranlxd_reset failed")


def fft3d(data, n, sign, scale):
    d = np.ascontiguousarray(data, dtype=np.complex128).copy()
    nn = np.array(n, dtype=np.int64)
    lib().oc_fft3d(d.ctypes.data_as(_dp), nn.ctypes.data_as(_i64p), sign, scale)
    return d


# ---------------- SU(3) ----------------

def generator(a):
    T = np.empty((3, 3), dtype=np.complex128)
    lib().oc_generator(a, _p(T))
    return T


def group_exp(alpha):
    alpha = np.ascontiguousarray(alpha, dtype=np.float64)
    G = np.empty((3, 3), dtype=np.complex128)
    lib().oc_group_exp(_p(alpha), _p(G))
    return G


def eigenh(A):
    A = np.ascontiguousarray(A, dtype=np.complex128)
    d = np.empty(3)
    U = np.empty((3, 3), dtype=np.complex128)
    lib().oc_eigenh3(_p(A), _p(d), _p(U))
    return d, U


def eigenc(A):
    A = np.ascontiguousarray(A, dtype=np.complex128)
    d = np.empty(3, dtype=np.complex128)
    U = np.empty((3, 3), dtype=np.complex128)
    lib().oc_eigenc3(_p(A), _p(d), _p(U))
    return d, U


def logu(P):
    P = np.ascontiguousarray(P, dtype=np.complex128)
    Lg = np.empty((3, 3), dtype=np.complex128)
    lib().oc_logu3(_p(P), _p(Lg))
    return Lg


# ---------------- gauge ----------------

def alloc_gauge(n):
    V = volume(n)
    return (np.zeros((V, 3, 3, 3), dtype=np.complex128), np.zeros((V, 3, 8), dtype=np.float64))


def cold(n, a):
    links, efield = alloc_gauge(n)
    L = lattice(n, a)
    lib().oc_gauge_cold(ctypes.byref(L), _p(links), _p(efield))
    return links, efield


def transverse_box(n, a, Q, n0, g, seed, identity_links=True):
    links, efield = alloc_gauge(n)
    L = lattice(n, a)
    rc = lib().oc_gauge_transverse_box(ctypes.byref(L), Q, n0, g, seed, int(identity_links),
                                        _p(links), _p(efield))
    if rc != 0:
        raise ValueError("transverse_box failed")
    return links, efield


def gauge_update(n, a, links, efield, dt=1.0):
    L = lattice(n, a)
    lib().oc_gauge_update(ctypes.byref(L), _p(links), _p(efield), dt)


def energy(n, a, links, efield):
    L = lattice(n, a)
    return lib().oc_gauge_energy(ctypes.byref(L), _p(links), _p(efield))


def gauss_ref(n, a, links, efield):
    L = lattice(n, a)
    return lib().oc_gauge_gauss_ref(ctypes.byref(L), _p(links), _p(efield))


def gauss_maxnorm(n, a, links, efield):
    L = lattice(n, a)
    return lib().oc_gauge_gauss_maxnorm(ctypes.byref(L), _p(links), _p(efield))


def gauss_project(n, a, links, efield, tol=1e-3, max_sweeps=1000):
    L = lattice(n, a)
    return lib().oc_gauge_gauss_project(ctypes.byref(L), _p(links), _p(efield), tol, max_sweeps)


def equilibrium_init(n, a, beta, nefieldinit, nequilibrium, tol=1e-3, seed=1, max_sweeps=10_000_000):
    """EquilibriumInit (gauge:380-814, no charges): returns links, efield and
    per round the projection sweeps, energy and deviation after the steps."""
    links, efield = alloc_gauge(n)
    L = lattice(n, a)
    sweeps = np.zeros(max(nefieldinit, 1), dtype=np.int64)
    en = np.zeros(max(nefieldinit, 1))
    dev = np.zeros(max(nefieldinit, 1))
    rc = lib().oc_gauge_equilibrium_init(ctypes.byref(L), beta, nefieldinit, nequilibrium, tol, seed, max_sweeps,
                                         _p(links), _p(efield), sweeps.ctypes.data_as(_i64p), _p(en), _p(dev))
    if rc != 0:
        raise ValueError(f"equilibrium_init failed ({rc})")
    return links, efield, sweeps[:nefieldinit], en[:nefieldinit], dev[:nefieldinit]


def field_strength(n, a, links, efield, i, j, site):
    L = lattice(n, a)
    F = np.empty((3, 3))
    lib().oc_field_strength(ctypes.byref(L), _p(links), _p(efield), i, j, site, _p(F))
    return F


# ---------------- heavy quarks ----------------

def single_point(n, lat_index_1based=1):
    V = volume(n)
    prop = np.zeros((V, 6, 6), dtype=np.complex128)
    L = lattice(n, [1, 1, 1, 1])
    lib().oc_heavy_init_single_point(ctypes.byref(L), lat_index_1based, _p(prop))
    return prop


def heavy_norm(n, prop):
    L = lattice(n, [1, 1, 1, 1])
    return lib().oc_heavy_norm(ctypes.byref(L), _p(prop))


def _coeffs(c):
    c = np.asarray(c, dtype=np.complex128).reshape(4)
    out = np.empty(8)
    out[0::2] = c.real
    out[1::2] = c.imag
    return out


def cn_apply(n, a, links, efield, mass, c, dt, herm, psi, transpose_blocks=True):
    L = lattice(n, a)
    out = np.empty_like(psi)
    cc = _coeffs(c)
    lib().oc_cn_apply(ctypes.byref(L), _p(links), _p(efield), mass, _p(cc), dt, int(herm),
                      int(transpose_blocks), _p(psi), _p(out))
    return out


def cn_update(n, a, links, efield, mass, c, dt, q, anti, tol=1e-13, maxits=10000,
              transpose_blocks=True):
    """One CN step of quark and antiquark in place; returns CnStats."""
    L = lattice(n, a)
    st = CnStats()
    cc = _coeffs(c)
    lib().oc_cn_update(ctypes.byref(L), _p(links), _p(efield), mass, _p(cc), dt, tol, maxits,
                       int(transpose_blocks), _p(q), _p(anti), ctypes.byref(st))
    return st


def meson_correlators(n, q, anti):
    L = lattice(n, [1, 1, 1, 1])
    out = {}
    for name in ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1"):
        r = np.empty(2)
        getattr(lib(), "oc_meson_" + name)(ctypes.byref(L), _p(q), _p(anti), _p(r))
        out[name] = complex(r[0], r[1])
    return out


def meson_correlators_gconjg(n, q, anti):
    """The _gconjg correlators (src/nrqcd.f90:1728-1905)."""
    L = lattice(n, [1, 1, 1, 1])
    r = np.empty(8)
    lib().oc_meson_gconjg(ctypes.byref(L), _p(q), _p(anti), _p(r))
    return {k: complex(r[2 * i], r[2 * i + 1]) for i, k in enumerate(("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1"))}


def coulomb_gaugefix(n, a, links, tol=1e-8, alpha=0.08, max_iterations=100):
    """CoulombGaugefixing on the links in place (gauge:2269-2456); returns the
    reference's loop counter and the deviation checked at each iteration."""
    L = lattice(n, a)
    dev = np.full(max(max_iterations, 1), np.nan)
    it = lib().oc_gauge_coulomb_gaugefix(ctypes.byref(L), _p(links), tol, alpha, max_iterations, _p(dev))
    return it, dev[:min(it, max_iterations)]


def transverse_correlators(n, a, links, efield):
    """(AA, EE, |p|) per momentum site (gauge:1825-1972, lattice:1081-1198)."""
    L = lattice(n, a)
    V = volume(n)
    aa, ee, mom = np.empty(V), np.empty(V), np.empty(V)
    lib().oc_gauge_transverse_correlators(ctypes.byref(L), _p(links), _p(efield), _p(aa), _p(ee), _p(mom))
    return aa, ee, mom


def num_threads():
    return lib().oc_num_threads()


def set_num_threads(n):
    lib().oc_set_num_threads(int(n))
