"""nrqcd_b200: B200 implementation of the per-timestep hot paths of the
NRQCD + classical-statistical SU(3) simulation (SU(3) leapfrog and the NRQCD
Crank-Nicolson propagator step), behind the C ABI of include/nrqcd_b200.h.

The modules mirror the reference's Fortran modules of the same names:
``lattice``, ``gaugeconfiguration_su3`` and ``nrqcd``; ``batch`` holds the
multi-field and ensemble forms of the Crank-Nicolson step and ``learned`` the
learned initial guess of its solve.
"""
from . import _capi, lattice  # noqa: F401
from ._capi import NrqcdError  # noqa: F401
from .gaugeconfiguration_su3 import GaugeConfiguration  # noqa: F401
from . import nrqcd  # noqa: F401
from .nrqcd import NRQCDField  # noqa: F401
from . import batch  # noqa: F401
from . import learned  # noqa: F401

__all__ = ["lattice", "nrqcd", "batch", "learned", "GaugeConfiguration", "NRQCDField", "NrqcdError"]
