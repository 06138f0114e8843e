"""Drop-in driver for the reference's hot-path simulation modes.

    python -m nrqcd_b200.driver <mode> <arguments in the reference's order> [--form F] [--device D]

Modes (the reference's `program simulation`, src/main.f90:3301-3340):

- **2**, MeasureEnergyAndGaussLawDeviation (src/main.f90:2572-2718).
  Arguments: Nx Ny Nz a0 ax ay az CoMTime TimeRange Seed Qs Amplitude Coupling.
  Transverse-polarised box initial condition, then TimeSteps = ceil(TimeRange/a0)
  leapfrog steps.  Writes `energy_gauss.txt`: time, energy, Gauss-law
  deviation (the reference's measure) per step, '(3(SP,E13.6,1X))'.
- **32**, MeasureHeavyQuarkoniumCorrelators_free (src/main.f90:282-522).
  Arguments: Nx Ny Nz a0 ax ay az smax Seed kspTol M Re(c1) Im(c1) ... Re(c4)
  Im(c4) FileMesonCorrelator FileNorm.  Cold links, point sources at the
  origin, nint(|smax|/a0) coupled steps (CN, then leapfrog).  Writes the
  correlator file (s, Re/Im of O1(1S0), O1(3S1), O8(1S0), O8(3S1)) and the
  norm file (s, quark, antiquark), '(n(SP,E16.9,1X))', with the reference's
  header lines.

`--form` selects the CN solver form (0 plain FP64, the reference's
precision; 1 precision form).  Progress goes to stdout as in the reference.
The modes whose initial state needs the thermal EquilibriumInit (33, 51, 52)
and the analysis modes (1, 11, 3, 4, 5) are outside the hot path.
"""
from __future__ import annotations

import math
import sys

from . import lattice, nrqcd
from .gaugeconfiguration_su3 import GaugeConfiguration
from .nrqcd import NRQCDField


def fortran_e(x: float, w: int, d: int) -> str:
    """Fortran 'SP,Ew.d' edit descriptor: sign, 0., d digits, exponent."""
    sign = "-" if (x < 0 or (x == 0 and math.copysign(1.0, x) < 0)) else "+"
    ax = abs(float(x))
    if ax == 0.0:
        body = "0." + "0" * d + "E+00"
    elif math.isnan(ax):
        return "NaN".rjust(w)
    elif math.isinf(ax):
        return (sign + "Infinity").rjust(w)
    else:
        m, e = f"{ax:.{d - 1}e}".split("e")
        digits = m.replace(".", "")
        exp = int(e) + 1
        if abs(exp) <= 99:
            body = f"0.{digits}E{exp:+03d}"
        else:  # three-digit exponent drops the letter
            body = f"0.{digits}{exp:+04d}"
    s = sign + body
    return s.rjust(w) if len(s) <= w else "*" * w


def _line(values, w: int, d: int) -> str:
    return "".join(fortran_e(v, w, d) + " " for v in values)


def _nint(x: float) -> int:
    """Fortran nint: nearest integer, halves away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def mode_energy_gauss(args, device=0, out="energy_gauss.txt"):
    ext = [int(a) for a in args[0:3]]
    sp = [float(a) for a in args[3:7]]
    comtime, trange = float(args[7]), float(args[8])  # CoMTime is read but unused (as in the reference)
    seed = int(args[9])
    qs, amp, coupling = float(args[10]), float(args[11]), float(args[12])
    steps = math.ceil(trange / sp[0])
    lattice.InitModule(ext, sp, device=device)
    try:
        g = GaugeConfiguration()
        g.TransversePolarisedOccupiedInit_Box(qs, amp, coupling, RandomSeed=seed, identity_links=False)
        with open(out, "w") as f:
            for it in range(steps + 1):
                t = it * sp[0]
                gauss = g.GetDeviationFromGaussLaw()
                energy = g.GetEnergy()
                f.write(_line((t, energy, gauss), 13, 6) + "\n")
                print(f" {t}", flush=True)
                g.Update(1.0)
        g.Deallocate()
    finally:
        lattice.FinalizeModule()
    print(" Simulation completed", flush=True)
    del comtime


CORRELATOR_HEADER = ("s Re(O1(1S0)) Im(O1(1S0)) Re(O1(3S1)) Im(O1(3S1)) Re(O8(1S0)) Im(O8(1S0)) "
                     "Re(O8(3S1)) Im(O8(3S1))")
NORM_HEADER = "s Quark Antiq"


def mode_correlators_free(args, form=0, device=0):
    ext = [int(a) for a in args[0:3]]
    sp = [float(a) for a in args[3:7]]
    smax = float(args[7])
    seed = int(args[8])  # the free mode draws no random numbers
    ksp_tol = float(args[9])
    mass = float(args[10])
    c = [complex(float(args[11 + 2 * k]), float(args[12 + 2 * k])) for k in range(4)]
    f_corr, f_norm = args[19], args[20]
    tsteps = _nint(abs(smax) / sp[0])
    lattice.InitModule(ext, sp, device=device)
    try:
        nrqcd.InitModule(mass, c, 1.0, ksp_tol, form=form)
        g = GaugeConfiguration()
        g.ColdInit()
        h = NRQCDField()
        h.InitSinglePoint(1, 1)
        with open(f_corr, "w") as fc, open(f_norm, "w") as fn:
            fc.write(CORRELATOR_HEADER + "\n")
            fn.write(NORM_HEADER + "\n")

            def observables(s):
                cor = h.GetMesoncorrelators()
                fn.write(_line((s, h.GetNorm_Quark(), h.GetNorm_AntiQ()), 16, 9) + "\n")
                vals = [s]
                for key in ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1"):
                    vals += [cor[key].real, cor[key].imag]
                fc.write(_line(vals, 16, 9) + "\n")
            observables(0.0)
            for it in range(1, tsteps + 1):
                h.Update(g, mass, c, 1.0)
                g.Update(1.0)
                observables(sp[0] * it)
                print(f"{100.0 * it / tsteps:7.3f}%", flush=True)
        h.Destructor()
        g.Deallocate()
        nrqcd.FinalizeModule()
    finally:
        lattice.FinalizeModule()
    print(" Simulation completed", flush=True)
    del seed


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    form, device = 0, 0
    if "--form" in argv:
        i = argv.index("--form")
        form = int(argv[i + 1])
        del argv[i:i + 2]
    if "--device" in argv:
        i = argv.index("--device")
        device = int(argv[i + 1])
        del argv[i:i + 2]
    if not argv:
        raise SystemExit(__doc__)
    mode = int(argv[0])
    if mode == 2:
        mode_energy_gauss(argv[1:], device=device)
    elif mode == 32:
        mode_correlators_free(argv[1:], form=form, device=device)
    else:
        raise SystemExit(f"Invalid simulation mode selected (this driver runs modes 2 and 32): {mode}")


if __name__ == "__main__":
    main()
