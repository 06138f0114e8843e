"""Helpers of the GPU parity tests: open a lattice context on cuda:0 for a
given size and close it (with every handle bound to it) afterwards."""
import contextlib
import gc

from nrqcd_b200 import lattice, nrqcd


@contextlib.contextmanager
def lattice_ctx(n, a, cn=None):
    """cn = (Mass, WilsonCoeffs, StepWidth, kspTol[, maxits, form]) opens the nrqcd module too."""
    lattice.InitModule(list(n), list(a), device=0)
    try:
        if cn is not None:
            nrqcd.InitModule(*cn)
        yield
    finally:
        if nrqcd.IsModuleInitialised():
            nrqcd.FinalizeModule()
        gc.collect()
        lattice.FinalizeModule()
