"""The host generator of the device initial conditions (ranlxd, luxury
level 2, nrqcd_b200/csrc/ranlxd_host.h) against the CPU oracle's generator:
bit-identical streams over many refills, for several seeds (plain C++; no
GPU)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT

N = 40000  # about 3,400 refills of 12 words


@pytest.fixture(scope="module")
def host_stream(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("ranlxd")
    src = d / "gen.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cstdlib>
#include "ranlxd_host.h"
int main(int argc, char **argv) {
  const long seed = std::atol(argv[1]), n = std::atol(argv[2]);
  const int level = std::atoi(argv[3]);
  nrqh::Ranlxd r;
  if (!r.init(level, seed)) return 2;
  for (long k = 0; k < n; ++k) {
    double v = r.next();
    std::fwrite(&v, sizeof v, 1, stdout);
  }
  return 0;
}
''')
    exe = d / "gen"
    r = subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "nrqcd_b200", "csrc"), str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def run(seed, n, level=2):
        out = subprocess.run([str(exe), str(seed), str(n), str(level)], capture_output=True, check=True).stdout
        return np.frombuffer(out, dtype=np.float64)
    return run


@pytest.mark.parametrize("seed,level", [(1, 2), (3, 2), (2147483647, 2), (12345, 1)])
def test_host_stream_equals_oracle(oracle, host_stream, seed, level):
    got = host_stream(seed, N, level)
    want = oracle.Ranlxd(level, seed).draw(N)
    assert got.shape == want.shape and np.array_equal(got, want)
