"""Drop-in driver for the reference's hot-path simulation modes.

    python -m nrqcd_b200.driver <mode> <arguments in the reference's order> [--form F] [--device D]

Modes (the reference's `program simulation`, src/main.f90:3301-3340):

- **1**, MeasureGluondistribution (src/main.f90:3020-3296).  Arguments: Nx Ny
  Nz a0 ax ay az CoMTime Seed Qs Amplitude Coupling GaugefixingMaxIterations
  GaugefixingTolerance GaugefixingCoefficient FileGluondist.  Box initial
  condition evolved to CoMTime, Coulomb gauge fixing of a copy, and per
  momentum site |p| and sqrt(AA EE) of the transverse correlators,
  '(2(SP,E13.6,1X))'.
- **11**, MeasureGluondistribution_Equilibrium (src/main.f90:2725-3012): the
  same output from the thermal EquilibriumInit.  Arguments: Nx Ny Nz a0 ax
  ay az TimeRange Seed Beta nefieldinit nequilibriumtimesteps
  TimeBetweenGluonMeasurements GaugefixingMaxIterations GaugefixingTolerance
  GaugefixingCoefficient FileGluondist MeasureEnergy [EnergyFilename].
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
- **3**, MeasureHeavyQuarkoniumCorrelators, the (t,s)-grid correlator
  (src/main.f90:2169-2565).  Arguments: Nx Ny Nz ds ax ay az tmin tmax smax
  Seed Qs Amplitude Coupling kspTol M Re(c1) Im(c1) ... Re(c4) Im(c4)
  FileMesonCorrelator FileNorm, with a0 = ds/2.  Transverse-polarised box
  initial condition and a point source at t = 0; the configuration is
  evolved to t1min = tmin - smax/2, and from every t1 a copy of the
  configuration and of the (never evolved) point source runs coupled steps
  to t2 = t1 + a0 .. t1 + smax.  Points with t = (t1+t2)/2 and s = t2 - t1 on
  the ds grid inside [tmin, tmax] record O1(3S1) and the norms.  Writes the
  correlator file (one row per s, Re/Im per t) and the norm file (Q/A per
  t), NaN where the grid has no sample, '(SP,E16.9,1X)' with the
  reference's F-formatted header.

- **31**, MeasureHeavyQuarkoniumCorrelators_oneT (src/main.f90:523-780).
  Arguments: Nx Ny Nz a0 ax ay az t smax Seed Qs Amplitude Coupling kspTol M
  Re(c1) Im(c1) ... Re(c4) Im(c4) FileMesonCorrelator FileNorm
  FileMesonCorrelator_gconjg.  Correlators for s = 0, 2a0, 4a0, ... from
  copies of the configuration evolved forward 2 it1 steps, the
  configuration stepping back by a0 after each; the third file holds the
  _gconjg correlators.
- **33**, MeasureHeavyQuarkoniumCorrelators_Equilibrium (src/main.f90:18-280).
  Arguments: Nx Ny Nz a0 ax ay az smax Seed Beta nefieldinit
  nequilibriumtimesteps kspTol M Re(c1) Im(c1) ... Re(c4) Im(c4)
  FileMesonCorrelator FileNorm MeasureEnergy [EnergyFilename].  As mode 32
  from the thermal EquilibriumInit (Gauss projection on the device); with
  MeasureEnergy = 1 the energy after each initialisation round goes to
  EnergyFilename.

`--form` selects the CN solver form (0 plain FP64, the reference's
precision; 1 precision form).  Progress goes to stdout as in the reference.
Records follow Fortran's rule that a trailing X edit descriptor transmits
no characters: values are separated by one blank and no record ends in one.
The Wilson-line modes (5, 51, 52) and the spectrum analysis (mode 4) are
outside the hot path.
"""
from __future__ import annotations

import math
import sys

import numpy as np

from . import lattice, nrqcd
from .gaugeconfiguration_su3 import GaugeConfiguration
from .nrqcd import NRQCDField


def fortran_e(x: float, w: int, d: int, plus: bool = True) -> str:
    """Fortran 'SP,Ew.d' edit descriptor: sign, 0., d digits, exponent
    ('Ew.d' without SP when plus is False: no sign for positive values)."""
    sign = "-" if (x < 0 or (x == 0 and math.copysign(1.0, x) < 0)) else ("+" if plus else "")
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


def fortran_f(x: float, w: int, d: int) -> str:
    """Fortran 'Fw.d' edit descriptor: d decimals right-justified in w
    characters; the optional leading zero of |x| < 1 is dropped when the
    width needs it, and a value that does not fit prints w asterisks."""
    s = f"{abs(float(x)):.{d}f}" + ("." if d == 0 else "")
    neg = x < 0 and float(s.rstrip(".")) != 0.0
    if neg:
        s = "-" + s
    if len(s) > w and (s.startswith("0.") or s.startswith("-0.")):
        s = s.replace("0.", ".", 1)
    return s.rjust(w) if len(s) <= w else "*" * w


def _line(values, w: int, d: int) -> str:
    """One record of n(SP,Ew.d,1X): values separated by one blank."""
    return " ".join(fortran_e(v, w, d) for v in values)


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


def _correlators_run(ext, sp, smax, ksp_tol, mass, c, f_corr, f_norm, init_gauge, form=0, device=0):
    """The time loop shared by modes 32 and 33 (src/main.f90:330-371 and
    :66-110): point sources at the origin, nint(|smax|/a0) coupled steps
    (CN, then leapfrog), observables after each."""
    tsteps = _nint(abs(smax) / sp[0])
    lattice.InitModule(ext, sp, device=device)
    try:
        nrqcd.InitModule(mass, c, 1.0, ksp_tol, form=form)
        g = GaugeConfiguration()
        init_gauge(g)
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


def mode_correlators_free(args, form=0, device=0):
    ext = [int(a) for a in args[0:3]]
    sp = [float(a) for a in args[3:7]]
    smax = float(args[7])
    int(args[8])  # Seed: read, but the free mode draws no random numbers
    ksp_tol = float(args[9])
    mass = float(args[10])
    c = [complex(float(args[11 + 2 * k]), float(args[12 + 2 * k])) for k in range(4)]
    _correlators_run(ext, sp, smax, ksp_tol, mass, c, args[19], args[20], lambda g: g.ColdInit(), form, device)


def mode_correlators_equilibrium(args, form=0, device=0):
    """Mode 33 (src/main.f90:18-280): as mode 32 from a thermal configuration,
    EquilibriumInit(Beta, nefieldinit, nequilibriumtimesteps) with the
    default projection tolerance 1e-3 after random%InitModule(Seed)."""
    ext = [int(a) for a in args[0:3]]
    sp = [float(a) for a in args[3:7]]
    smax = float(args[7])
    seed = int(args[8])
    beta = float(args[9])
    nefieldinit, nequilibrium = int(args[10]), int(args[11])
    ksp_tol = float(args[12])
    mass = float(args[13])
    c = [complex(float(args[14 + 2 * k]), float(args[15 + 2 * k])) for k in range(4)]
    f_corr, f_norm = args[22], args[23]
    # MeasureEnergy, read with (I1): a missing argument reads as blank, i.e. 0
    measure = len(args) > 24 and int(args[24] or 0) != 0
    energy_file = args[25] if measure else None

    def init(g):
        g.EquilibriumInit(beta, nefieldinit, nequilibrium, MeasureEnergy=measure, filename=energy_file,
                          RandomSeed=seed)
    _correlators_run(ext, sp, smax, ksp_tol, mass, c, f_corr, f_norm, init, form, device)


def mode_correlators_one_t(args, form=0, device=0):
    """Mode 31, MeasureHeavyQuarkoniumCorrelators_oneT (src/main.f90:523-780):
    transverse-polarised box initial condition evolved to the time t; for
    it1 = 1 .. nint(|smax/2|/a0) a copy of the configuration (at
    t1 = t - (it1-1) a0) and of the point source runs 2 it1 coupled steps,
    its observables are written at s = 2 it1 a0, and the configuration then
    steps back by a0 (the reference's order, main.f90:601-617).  The
    observables at s = 0 come first.  Three files: the correlators, the
    norms and the _gconjg correlators."""
    ext = [int(a) for a in args[0:3]]
    sp = [float(a) for a in args[3:7]]
    tcom, smax = float(args[7]), float(args[8])
    seed = int(args[9])
    qs, amp, coupling = float(args[10]), float(args[11]), float(args[12])
    ksp_tol = float(args[13])
    mass = float(args[14])
    c = [complex(float(args[15 + 2 * k]), float(args[16 + 2 * k])) for k in range(4)]
    f_corr, f_norm, f_gconjg = args[23], args[24], args[25]
    t1steps = _nint(abs(smax / 2) / sp[0])
    nwork = sum(2 * it1 for it1 in range(1, t1steps + 1))
    lattice.InitModule(ext, sp, device=device)
    try:
        nrqcd.InitModule(mass, c, 1.0, ksp_tol, form=form)
        g1, g2 = GaugeConfiguration(), GaugeConfiguration()
        g1.TransversePolarisedOccupiedInit_Box(qs, amp, coupling, RandomSeed=seed, identity_links=False)
        h1, h2 = NRQCDField(), NRQCDField()
        h1.InitSinglePoint(1, 1)
        for _ in range(_nint(abs(tcom) / sp[0])):
            g1.Update(math.copysign(1.0, tcom))
        with open(f_corr, "w") as fc, open(f_norm, "w") as fn, open(f_gconjg, "w") as fg:
            fc.write(CORRELATOR_HEADER + "\n")
            fg.write(CORRELATOR_HEADER + "\n")
            fn.write(NORM_HEADER + "\n")

            def observables(s, h):
                fn.write(_line((s, h.GetNorm_Quark(), h.GetNorm_AntiQ()), 16, 9) + "\n")
                for f, cor in ((fc, h.GetMesoncorrelators()), (fg, h.GetMesoncorrelators_gconjg())):
                    vals = [s]
                    for key in ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1"):
                        vals += [cor[key].real, cor[key].imag]
                    f.write(_line(vals, 16, 9) + "\n")
            observables(0.0, h1)
            iwork = 0
            for it1 in range(1, t1steps + 1):
                t2steps = 2 * it1
                h2.Assign(h1)
                g2.assign(g1)
                for _ in range(t2steps):
                    iwork += 1
                    h2.Update(g2, mass, c, 1.0)
                    g2.Update(1.0)
                    # '(F7.3,A1)' of real(iwork)/nwork*100 in default (single) precision
                    pct = np.float32(iwork) / np.float32(nwork) * np.float32(100)
                    print(f"{float(pct):7.3f}%", flush=True)
                observables(sp[0] * t2steps, h2)
                g1.Update(-1.0)
        for o in (h1, h2):
            o.Destructor()
        for o in (g1, g2):
            o.Deallocate()
        nrqcd.FinalizeModule()
    finally:
        lattice.FinalizeModule()
    print(" Simulation completed", flush=True)


def write_gluondist(g, filename, max_iterations, tolerance, alpha):
    """PrintObservables of modes 1 and 11 (src/main.f90:3052-3170,
    2775-2895): a Coulomb-gauge-fixed copy of the configuration, its
    transverse AA and EE correlators, and per momentum site (lattice order)
    |p| and sqrt(AA EE), '(2(SP,E13.6,1X))'."""
    fixed = GaugeConfiguration()
    fixed.assign(g)
    fixed.CoulombGaugefixing(Tolerance_=tolerance, alpha_=alpha, MaxIterations_=max_iterations)
    aa, ee, mom = fixed.GetTransverseCorrelators()
    fixed.Deallocate()
    dist = np.sqrt(aa * ee)
    with open(filename, "w") as f:
        for p_, n_ in zip(mom, dist):
            f.write(_line((float(p_), float(n_)), 13, 6) + "\n")


def mode_gluondist(args, device=0):
    """Mode 1, MeasureGluondistribution (src/main.f90:3020-3296).  Arguments:
    Nx Ny Nz a0 ax ay az CoMTime Seed Qs Amplitude Coupling
    GaugefixingMaxIterations GaugefixingTolerance GaugefixingCoefficient
    FileGluondist.  Transverse-polarised box initial condition,
    ceiling(|CoMTime|/a0) leapfrog steps of sign(CoMTime), then the gluon
    distribution."""
    ext = [int(a) for a in args[0:3]]
    sp = [float(a) for a in args[3:7]]
    comtime = float(args[7])
    seed = int(args[8])
    qs, amp, coupling = float(args[9]), float(args[10]), float(args[11])
    gf_maxit, gf_tol, gf_alpha = int(args[12]), float(args[13]), float(args[14])
    f_out = args[15]
    steps = math.ceil(abs(comtime) / sp[0])
    lattice.InitModule(ext, sp, device=device)
    try:
        g = GaugeConfiguration()
        g.TransversePolarisedOccupiedInit_Box(qs, amp, coupling, RandomSeed=seed, identity_links=False)
        for _ in range(steps):
            g.Update(math.copysign(1.0, comtime))
        write_gluondist(g, f_out, gf_maxit, gf_tol, gf_alpha)
        g.Deallocate()
    finally:
        lattice.FinalizeModule()
    print(" Simulation completed", flush=True)


def mode_gluondist_equilibrium(args, device=0):
    """Mode 11, MeasureGluondistribution_Equilibrium (src/main.f90:2725-3012).
    Arguments: Nx Ny Nz a0 ax ay az TimeRange Seed Beta nefieldinit
    nequilibriumtimesteps TimeBetweenGluonMeasurements
    GaugefixingMaxIterations GaugefixingTolerance GaugefixingCoefficient
    FileGluondist MeasureEnergy [EnergyFilename].  EquilibriumInit, then the
    gluon distribution (TimeRange and TimeBetweenGluonMeasurements are read
    but unused, as in the reference)."""
    ext = [int(a) for a in args[0:3]]
    sp = [float(a) for a in args[3:7]]
    seed = int(args[8])
    beta = float(args[9])
    nefieldinit, nequilibrium = int(args[10]), int(args[11])
    gf_maxit, gf_tol, gf_alpha = int(args[13]), float(args[14]), float(args[15])
    f_out = args[16]
    measure = len(args) > 17 and int(args[17] or 0) != 0
    energy_file = args[18] if measure else None
    lattice.InitModule(ext, sp, device=device)
    try:
        g = GaugeConfiguration()
        g.EquilibriumInit(beta, nefieldinit, nequilibrium, MeasureEnergy=measure, filename=energy_file,
                          RandomSeed=seed)
        write_gluondist(g, f_out, gf_maxit, gf_tol, gf_alpha)
        g.Deallocate()
    finally:
        lattice.FinalizeModule()
    print(" Simulation completed", flush=True)


ZERO_TOL = 1e-12  # GetZeroTol() of the FP64 build, src/tolerances.f90:21-26


def ts_grid_schedule(a0: float, ds: float, tmin: float, tmax: float, smax: float):
    """The (t,s)-grid loop structure of mode 3 (src/main.f90:2244-2362),
    host arithmetic only.

    Returns (pre_sign, n_pre, rows): n_pre leapfrog steps of width pre_sign
    bring the configuration from t = 0 to t1min = tmin - smax/2; each row
    (it1, steps) starts from the configuration at t1 = it1*a0, and each entry
    (it2, point) of steps is one coupled step ending at t2 = it2*a0, with
    point = (is, it) where the reference records the sample and None
    otherwise.  As in the reference, the step that leaves [., tmax] is still
    taken before the row ends, and every entry counts as one unit of
    progress.
    """
    t1min = tmin - smax / 2
    t1max = tmax
    n_pre = _nint(abs(t1min) / a0)
    pre_sign = math.copysign(1.0, t1min)
    it2range = _nint(smax / a0)
    rows = []
    for it1 in range(_nint(t1min / a0), _nint(t1max / a0) + 1):
        t1 = it1 * a0
        steps = []
        for it2 in range(it1 + 1, it1 + it2range + 1):
            t2 = it2 * a0
            t = (t2 + t1) / 2
            s = t2 - t1
            itt, ist = _nint(t / ds), _nint(s / ds)
            on_grid = abs(itt * ds - t) <= ZERO_TOL and abs(ist * ds - s) <= ZERO_TOL
            if tmin <= t <= tmax and on_grid:
                steps.append((it2, (ist, itt)))
            else:
                steps.append((it2, None))
                if t > tmax:
                    break
        rows.append((it1, steps))
    return pre_sign, n_pre, rows


def ts_grid_bounds(ds: float, tmin: float, tmax: float, smax: float):
    """Index ranges of the result arrays: is in [0, ismax], it in [itmin, itmax]."""
    return 0, _nint(smax / ds), _nint(tmin / ds), _nint(tmax / ds)


def write_ts_grid(f_corr: str, f_norm: str, ds: float, itmin: int, corr, qnorm, anorm):
    """Output of mode 3 (src/main.f90:2366-2434).  corr, qnorm, anorm are
    indexed [is][it - itmin].  Header: 's', then per t 'Re'/'Im' (correlator)
    or 'Q'/'A' (norm) glued to t in F(w.d) with d = nint(-log10 ds) and
    w = d + p + 2, p = nint(log10|t|) for |t| > 1 else 0 (the reference
    writes w and d with I1, so both must be single digits)."""
    nt = len(corr[0])
    d = _nint(-math.log10(ds))
    hc, hn = ["s"], ["s"]
    for k in range(nt):
        t = (itmin + k) * ds
        p = _nint(math.log10(abs(t))) if abs(t) > 1 else 0
        w = d + p + 2
        if not (0 <= d <= 9 and 0 <= w <= 9):
            raise ValueError(f"(t,s)-grid header: F{w}.{d} is outside the reference's single-digit format")
        ft = fortran_f(t, w, d)
        hc += ["Re" + ft, "Im" + ft]
        hn += ["Q" + ft, "A" + ft]
    with open(f_corr, "w") as fc, open(f_norm, "w") as fn:
        fc.write(" ".join(hc) + "\n")
        fn.write(" ".join(hn) + "\n")
        for is_ in range(len(corr)):
            s = is_ * ds
            vc, vn = [s], [s]
            for k in range(nt):
                vc += [corr[is_][k].real, corr[is_][k].imag]
                vn += [qnorm[is_][k], anorm[is_][k]]
            fc.write(_line(vc, 16, 9) + "\n")
            fn.write(_line(vn, 16, 9) + "\n")


def mode_ts_grid(args, form=0, device=0):
    ext = [int(a) for a in args[0:3]]
    ds = float(args[3])
    sp = [ds / 2] + [float(a) for a in args[4:7]]
    tmin, tmax, smax = float(args[7]), float(args[8]), float(args[9])
    seed = int(args[10])
    qs, amp, coupling = float(args[11]), float(args[12]), float(args[13])
    ksp_tol = float(args[14])
    mass = float(args[15])
    c = [complex(float(args[16 + 2 * k]), float(args[17 + 2 * k])) for k in range(4)]
    f_corr, f_norm = args[24], args[25]
    ismin, ismax, itmin, itmax = ts_grid_bounds(ds, tmin, tmax, smax)
    nan = float("nan")
    ns, nt = ismax - ismin + 1, itmax - itmin + 1
    corr = [[complex(nan, nan)] * nt for _ in range(ns)]
    qnorm = [[nan] * nt for _ in range(ns)]
    corr[0] = [1j] * nt  # s = 0: the reference's preset row
    qnorm[0] = [1.0] * nt
    anorm = [row[:] for row in qnorm]
    pre_sign, n_pre, rows = ts_grid_schedule(sp[0], ds, tmin, tmax, smax)
    nprogress = sum(len(steps) for _, steps in rows)
    lattice.InitModule(ext, sp, device=device)
    try:
        nrqcd.InitModule(mass, c, 1.0, ksp_tol, form=form)
        g1, g2 = GaugeConfiguration(), GaugeConfiguration()
        g1.TransversePolarisedOccupiedInit_Box(qs, amp, coupling, RandomSeed=seed, identity_links=False)
        h1, h2 = NRQCDField(), NRQCDField()
        h1.InitSinglePoint(1, 1)
        for _ in range(n_pre):
            g1.Update(pre_sign)
        iprogress = 0
        for _, steps in rows:
            g2.assign(g1)
            h2.Assign(h1)
            for _, point in steps:
                iprogress += 1
                # '(E16.9,A1)' of real(iprogress)/nprogress*100 in default (single) precision
                pct = np.float32(iprogress) / np.float32(nprogress) * np.float32(100)
                print(fortran_e(float(pct), 16, 9, plus=False) + "%", flush=True)
                h2.Update(g2, mass, c, 1.0)
                g2.Update(1.0)
                if point is not None:
                    is_, it_ = point
                    if not (ismin <= is_ <= ismax and itmin <= it_ <= itmax):
                        raise RuntimeError(f"(t,s)-grid point ({is_}, {it_}) outside the result arrays")
                    corr[is_][it_ - itmin] = h2.GetMesoncorrelator_O1_3S1_ZeroMomentum()
                    qnorm[is_][it_ - itmin] = h2.GetNorm_Quark()
                    anorm[is_][it_ - itmin] = h2.GetNorm_AntiQ()
            g1.Update(1.0)
        write_ts_grid(f_corr, f_norm, ds, itmin, corr, qnorm, anorm)
        h1.Destructor()
        h2.Destructor()
        g1.Deallocate()
        g2.Deallocate()
        nrqcd.FinalizeModule()
    finally:
        lattice.FinalizeModule()
    print(" Simulation completed", flush=True)


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
    if mode == 1:
        mode_gluondist(argv[1:], device=device)
    elif mode == 11:
        mode_gluondist_equilibrium(argv[1:], device=device)
    elif mode == 2:
        mode_energy_gauss(argv[1:], device=device)
    elif mode == 3:
        mode_ts_grid(argv[1:], form=form, device=device)
    elif mode == 31:
        mode_correlators_one_t(argv[1:], form=form, device=device)
    elif mode == 32:
        mode_correlators_free(argv[1:], form=form, device=device)
    elif mode == 33:
        mode_correlators_equilibrium(argv[1:], form=form, device=device)
    else:
        raise SystemExit(f"Invalid simulation mode selected (this driver runs modes 1, 11, 2, 3, 31, 32 and 33): {mode}")


if __name__ == "__main__":
    main()
