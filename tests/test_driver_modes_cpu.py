"""CPU checks of the drop-in driver's argument handling and call sequence for
every mode, with the device classes replaced by recording stand-ins (the
numerics of each mode are checked against the oracle on the GPU)."""
import math

import numpy as np
import pytest

from nrqcd_b200 import driver


class Rec:
    calls = []


class FakeLattice:
    @staticmethod
    def InitModule(ext, sp, device=0):
        Rec.calls.append(("lattice", tuple(ext), tuple(sp)))

    @staticmethod
    def FinalizeModule():
        Rec.calls.append(("lattice_end",))


class FakeNrqcd:
    @staticmethod
    def InitModule(mass, c, step, tol, form=0):
        Rec.calls.append(("nrqcd", mass, tuple(c), step, tol, form))

    @staticmethod
    def FinalizeModule():
        Rec.calls.append(("nrqcd_end",))


class FakeGauge:
    V = 8

    def __init__(self):
        Rec.calls.append(("gauge_new",))

    def ColdInit(self):
        Rec.calls.append(("cold",))

    def TransversePolarisedOccupiedInit_Box(self, qs, amp, g, RandomSeed=1, identity_links=False):
        Rec.calls.append(("box", qs, amp, g, RandomSeed, identity_links))

    def EquilibriumInit(self, beta, nef, neq, MeasureEnergy=False, filename=None, RandomSeed=1, **kw):
        Rec.calls.append(("equilibrium", beta, nef, neq, MeasureEnergy, filename, RandomSeed))

    def Update(self, dt=1.0):
        Rec.calls.append(("leapfrog", dt))

    def assign(self, other):
        Rec.calls.append(("gauge_copy",))

    def CoulombGaugefixing(self, Tolerance_=1e-8, alpha_=0.08, MaxIterations_=100, verbose=True):
        Rec.calls.append(("gaugefix", Tolerance_, alpha_, MaxIterations_))
        return 3, np.zeros(3)

    def GetTransverseCorrelators(self):
        return np.full(self.V, 4.0), np.full(self.V, 9.0), np.arange(self.V, dtype=float)

    def GetDeviationFromGaussLaw(self):
        return 0.0

    def GetEnergy(self):
        return 1.0

    def Deallocate(self):
        pass


class FakeHeavy:
    def __init__(self):
        Rec.calls.append(("heavy_new",))

    def InitSinglePoint(self, lq, la):
        Rec.calls.append(("point", lq, la))

    def Update(self, g, mass, c, dt):
        Rec.calls.append(("cn", mass, tuple(c), dt))

    def Assign(self, other):
        Rec.calls.append(("heavy_copy",))

    def GetNorm_Quark(self):
        return 1.0

    def GetNorm_AntiQ(self):
        return 1.0

    def GetMesoncorrelators(self):
        return {k: 1j for k in ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1")}

    def GetMesoncorrelators_gconjg(self):
        return {k: 2j for k in ("o1_1s0", "o1_3s1", "o8_1s0", "o8_3s1")}

    def GetMesoncorrelator_O1_3S1_ZeroMomentum(self):
        return 0.5 + 0.25j

    def Destructor(self):
        pass


@pytest.fixture(autouse=True)
def fakes(monkeypatch):
    Rec.calls = []
    monkeypatch.setattr(driver, "lattice", FakeLattice)
    monkeypatch.setattr(driver, "nrqcd", FakeNrqcd)
    monkeypatch.setattr(driver, "GaugeConfiguration", FakeGauge)
    monkeypatch.setattr(driver, "NRQCDField", FakeHeavy)


def names(kind):
    return [c for c in Rec.calls if c[0] == kind]


C8 = ["1.0", "0.0", "2.0", "0.5", "3.0", "0.0", "4.0", "-1.0"]
CPLX = (1 + 0j, 2 + 0.5j, 3 + 0j, 4 - 1j)


def test_mode32(tmp_path):
    fc, fn = tmp_path / "c", tmp_path / "n"
    driver.main(["32", "2", "2", "2", "0.05", "1", "1", "1", "0.2", "7", "1e-11", "1.5"] + C8 + [str(fc), str(fn)])
    assert Rec.calls[0] == ("lattice", (2, 2, 2), (0.05, 1.0, 1.0, 1.0))
    assert names("nrqcd")[0] == ("nrqcd", 1.5, CPLX, 1.0, 1e-11, 0)
    assert names("cold") and len(names("cn")) == 4 and len(names("leapfrog")) == 4
    assert len(fc.read_text().splitlines()) == 6 and len(fn.read_text().splitlines()) == 6  # header, s = 0, 4 steps


def test_mode33_reads_thermal_arguments(tmp_path):
    fc, fn, fe = tmp_path / "c", tmp_path / "n", tmp_path / "e"
    driver.main(["33", "2", "2", "2", "0.05", "1", "1", "1", "0.1", "9", "6.5", "3", "4", "1e-10", "2.0"] + C8 +
                [str(fc), str(fn), "1", str(fe)])
    assert names("equilibrium") == [("equilibrium", 6.5, 3, 4, True, str(fe), 9)]
    assert names("nrqcd")[0] == ("nrqcd", 2.0, CPLX, 1.0, 1e-10, 0)
    assert len(names("cn")) == 2
    driver.main(["33", "2", "2", "2", "0.05", "1", "1", "1", "0.1", "9", "6.5", "3", "4", "1e-10", "2.0"] + C8 +
                [str(fc), str(fn), "0"])
    assert names("equilibrium")[-1][4:6] == (False, None)


def test_mode31_rows(tmp_path):
    fc, fn, fg = tmp_path / "c", tmp_path / "n", tmp_path / "g"
    driver.main(["31", "2", "2", "2", "0.05", "1", "1", "1", "-0.1", "0.3", "5", "0.8", "1.0", "0.5", "1e-12", "1.0"]
                + C8 + [str(fc), str(fn), str(fg)])
    assert names("box") == [("box", 0.8, 1.0, 0.5, 5, False)]
    # t = -0.1: two backward steps first; smax/2 = 0.15: t1steps = 3 rows of 2, 4, 6 coupled steps,
    # each row followed by one backward step of the configuration
    lf = [c[1] for c in names("leapfrog")]
    assert lf[:2] == [-1.0, -1.0] and lf.count(-1.0) == 2 + 3 and len(names("cn")) == 12
    for f in (fc, fn, fg):
        assert len(f.read_text().splitlines()) == 1 + 1 + 3


def test_mode3_grid(tmp_path):
    fc, fn = tmp_path / "c", tmp_path / "n"
    driver.main(["3", "2", "2", "2", "0.1", "1", "1", "1", "0.0", "0.1", "0.2", "3", "0.8", "1.0", "0.5", "1e-12",
                 "1.0"] + C8 + [str(fc), str(fn)])
    assert Rec.calls[0] == ("lattice", (2, 2, 2), (0.05, 1.0, 1.0, 1.0))  # a0 = ds / 2
    sign, n_pre, rows = driver.ts_grid_schedule(0.05, 0.1, 0.0, 0.1, 0.2)
    assert len(names("cn")) == sum(len(s) for _, s in rows)
    assert len(names("heavy_copy")) == len(rows) == len(names("gauge_copy"))
    lines = fc.read_text().splitlines()
    assert lines[0] == "s Re0.0 Im0.0 Re0.1 Im0.1" and len(lines) == 4
    vals = [float(v) for v in lines[2].split()]
    assert vals[1:3] == [0.5, 0.25]  # the O1(3S1) sample at (s = 0.1, t = 0)


def test_mode1_and_mode11_gluon_distribution(tmp_path):
    f = tmp_path / "g"
    driver.main(["1", "2", "2", "2", "0.05", "1", "1", "1", "-0.12", "4", "0.5", "1.0", "0.0", "77", "1e-9", "0.1",
                 str(f)])
    assert names("box") == [("box", 0.5, 1.0, 0.0, 4, False)]
    assert [c[1] for c in names("leapfrog")] == [-1.0] * math.ceil(0.12 / 0.05)
    assert names("gaugefix") == [("gaugefix", 1e-9, 0.1, 77)]
    lines = f.read_text().splitlines()
    assert len(lines) == 8 and [float(v) for v in lines[3].split()] == [3.0, 6.0]  # |p|, sqrt(AA EE)
    Rec.calls = []
    driver.main(["11", "2", "2", "2", "0.05", "1", "1", "1", "5.0", "4", "8.0", "2", "3", "1.0", "50", "1e-8",
                 "0.08", str(f), "0"])
    assert names("equilibrium") == [("equilibrium", 8.0, 2, 3, False, None, 4)]
    assert names("gaugefix") == [("gaugefix", 1e-8, 0.08, 50)]
    assert not names("leapfrog")


def test_mode2_energy_file(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    driver.main(["2", "2", "2", "2", "0.05", "1", "1", "1", "0.0", "0.1", "3", "0.8", "1.0", "0.0"])
    assert len((tmp_path / "energy_gauss.txt").read_text().splitlines()) == 3
    assert len(names("leapfrog")) == 3


def test_unknown_mode():
    with pytest.raises(SystemExit):
        driver.main(["5"])


# ---------------------------------------------------------------- the reference's run templates
def _templates():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "driver_argv.json")
    return json.load(open(path))


@pytest.mark.parametrize("mode", ["1", "11", "2", "3", "31", "32", "33"])
def test_reference_run_templates_parse(mode, tmp_path, monkeypatch):
    """Every run template of the reference (src/templates/*.sh, its argument
    order and values in tests/golden/driver_argv.json) runs through the
    driver: the lattice, spacings, solver and gauge-fixing parameters reach
    the library as the template sets them (the mode 33 template predates
    the MeasureEnergy argument; a missing one reads as 0, as in Fortran)."""
    monkeypatch.chdir(tmp_path)
    items = _templates()[mode]
    v = dict(items)
    driver.main([val for _, val in items])
    ext = (int(v["Nx"]), int(v["Ny"]), int(v["Nz"]))
    a0 = float(v["ds"]) / 2 if mode == "3" else float(v.get("TimeSpacing", v.get("at", 0)))
    assert Rec.calls[0] == ("lattice", ext, (a0, float(v["ax"]), float(v["ay"]), float(v["az"])))
    if mode in ("3", "31", "32", "33"):
        c = tuple(complex(float(v[f"c{k}_re"]), float(v[f"c{k}_im"])) for k in range(4))
        assert names("nrqcd")[0] == ("nrqcd", float(v["Mass"]), c, 1.0, float(v["iterativeTol"]), 0)
    if mode in ("1", "11"):
        assert names("gaugefix") == [("gaugefix", float(v["GaugefixingTolerance"]),
                                      float(v["GaugefixingCoefficient"]), int(v["GaugefixingMaxSteps"]))]
        assert (tmp_path / v["FileNameGluondist"]).exists()
    if mode in ("11", "33"):
        eq = names("equilibrium")[0]
        assert eq[1:4] == (float(v["Beta"]), int(v["nefieldinit"]), int(v["nequilibriumtimesteps"]))
        assert eq[6] == int(v["RandomSeed"])
    if mode in ("1", "2", "3", "31"):
        assert names("box")[0][1:5] == (float(v["InitialGluonSaturationScale"]),
                                        float(v["InitialGluonOccupationAmplitude"]), float(v["Coupling"]),
                                        int(v["RandomSeed"]))
    if mode == "32":
        assert len(names("cn")) == round(float(v["smax"]) / float(v["at"]))
