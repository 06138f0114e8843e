"""Writes tests/golden/driver_argv.json: for each run template of the
reference (src/templates/*.sh) that launches a mode this driver runs, the
template's argument list in its order (the variables of its mpiexec line
with the values the template assigns).  Run from the repository root with
the reference checked out at ../reference or given as the first argument:

    python tests/golden/make_driver_argv.py /path/to/NRQCD

Only the argument order and the template's values are kept, as test data
for the driver's parsing (tests/test_driver_modes_cpu.py)."""
import json
import os
import re
import sys

TEMPLATES = {
    1: "MeasureGluondistribution.sh",
    11: "MeasureGluondistribution_Equilibrium.sh",
    2: "MeasureEnergyAndGaussLawDeviation.sh",
    3: "MeasureHeavyMesonCorrelator.sh",
    31: "MeasureHeavyMesonCorrelator_oneT.sh",
    32: "MeasureHeavyMesonCorrelator_free.sh",
    33: "MeasureHeavyMesonCorrelator_equilibrium.sh",
}


def parse(path):
    text = open(path).read()
    values = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0]
        for stmt in line.split(";"):
            m = re.fullmatch(r"\s*([A-Za-z_][A-Za-z0-9_]*)=(\S*)\s*", stmt)
            if m:
                values[m.group(1)] = m.group(2).strip('"')
    launch = re.search(r"\$exename\s*\\?\s*\n?\s*(\$mode[^\n]*)", text)
    names = re.findall(r"\$([A-Za-z_][A-Za-z0-9_]*)", launch.group(1))
    return [(n, values[n]) for n in names]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.path.join("..", "reference")
    out = {}
    for mode, name in TEMPLATES.items():
        out[str(mode)] = parse(os.path.join(ref, "src", "templates", name))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "driver_argv.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(dst)


if __name__ == "__main__":
    main()
