"""The host generator of the device initial conditions (ranlxd, luxury
level 2, nrqcd_b200/csrc/ranlxd_host.h) against the CPU oracle's generator:
bit-identical streams over many refills, for several seeds (plain C++; no
GPU).  The jump (the recurrence as a congruential generator modulo
b^12 - b^5 + 1, b = 2^48) lands on the same numbers as sequential calls, and
the threaded pair draw of the initial conditions equals one sequential pass."""
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


JUMP_SRC = r'''
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>
#include "ranlxd_host.h"
// mode 0: numbers [n, n + k) after jump(n), for each n on the command line
// mode 1: jump(n) against jump(n - d) and d calls of next(), far into the stream
// mode 2: draw_pairs on several threads against one sequential pass
// mode 3: an exception thrown by the callback reaches the caller
// mode 4: block_states against jumps to the same blocks
int main(int argc, char **argv) {
  const int mode = std::atoi(argv[1]), level = std::atoi(argv[2]);
  const long seed = std::atol(argv[3]);
  if (mode == 0) {
    const long k = std::atol(argv[4]);
    for (int a = 5; a < argc; ++a) {
      nrqh::Ranlxd r;
      r.init(level, seed);
      if (!r.jump(std::strtoull(argv[a], nullptr, 10))) return 3;
      for (long i = 0; i < k; ++i) {
        double v = r.next();
        std::fwrite(&v, sizeof v, 1, stdout);
      }
    }
    return 0;
  }
  if (mode == 1) {
    long bad = 0;
    for (int a = 4; a < argc; ++a) {
      const unsigned long long n = std::strtoull(argv[a], nullptr, 10);
      nrqh::Ranlxd x, y;
      x.init(level, seed);
      y.init(level, seed);
      if (!x.jump(n) || !y.jump(n - 1000)) return 3;
      for (int i = 0; i < 1000; ++i) y.next();
      for (int i = 0; i < 600; ++i) bad += x.next() != y.next();
    }
    std::printf("%ld\n", bad);
    return 0;
  }
  const size_t count = std::atol(argv[4]);
  const unsigned long long first = std::strtoull(argv[5], nullptr, 10);
  if (mode == 4) {  // block_states: every state continues the stream at its block
    const unsigned long long first_block = count, stride = first;
    const size_t n = std::atol(argv[6]);
    std::vector<int64_t> w(12 * n);
    if (!nrqh::block_states(level, seed, first_block, stride, n, w.data(), 8)) return 3;
    long bad = 0;
    for (size_t t = 0; t < n; ++t) {
      nrqh::Ranlxd a, b;
      a.init(level, seed);
      b.init(level, seed);
      a.load_block_state(&w[12 * t]);
      if (!b.jump(12 * (first_block + stride * t))) return 3;
      for (int i = 0; i < 36; ++i) bad += a.next() != b.next();
    }
    std::printf("%ld\n", bad);
    return 0;
  }
  if (mode == 3) {  // the callback throws at pair argv[6]: caught here, after every worker joined
    const size_t bad_at = std::atol(argv[6]);
    try {
      nrqh::draw_pairs(level, seed, first, count, [&](size_t i, double, double) {
        if (i == bad_at) throw std::runtime_error("planted");
      }, 8);
    } catch (const std::runtime_error &e) {
      std::printf("caught %s\n", e.what());
      return 0;
    }
    return 4;
  }
  std::vector<double> got(2 * count), want(2 * count);
  if (!nrqh::draw_pairs(level, seed, first, count, [&](size_t i, double u1, double u2) {
        got[2 * i] = u1;
        got[2 * i + 1] = u2;
      }, 8))
    return 3;
  nrqh::Ranlxd r;
  r.init(level, seed);
  for (unsigned long long i = 0; i < first; ++i) r.next();
  for (size_t i = 0; i < 2 * count; ++i) want[i] = r.next();
  long bad = 0;
  for (size_t i = 0; i < 2 * count; ++i) bad += got[i] != want[i];
  std::printf("%ld\n", bad);
  return 0;
}
'''


@pytest.fixture(scope="module")
def jump_exe(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("ranlxd_jump")
    (d / "jump.cpp").write_text(JUMP_SRC)
    exe = d / "jump"
    r = subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "nrqcd_b200", "csrc"),
                        str(d / "jump.cpp"), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("seed,level", [(1, 2), (2147483647, 2), (12345, 1)])
def test_jump_lands_on_the_oracle_stream(oracle, jump_exe, seed, level):
    """Offsets at, before and after block boundaries (12 numbers per refill)
    and inside blocks, against the oracle's sequential stream."""
    k = 40
    offsets = [0, 1, 11, 12, 13, 23, 24, 143, 144, 145, 1001, 12347, 30000 - k]
    out = subprocess.run([str(jump_exe), "0", str(level), str(seed), str(k)] + [str(n) for n in offsets],
                         capture_output=True, check=True).stdout
    got = np.frombuffer(out, dtype=np.float64).reshape(len(offsets), k)
    want = oracle.Ranlxd(level, seed).draw(30000)
    for row, n in zip(got, offsets):
        assert np.array_equal(row, want[n:n + k]), n


def test_jump_far_into_the_stream(jump_exe):
    """jump(n) equals jump(n - 1000) followed by 1000 calls, up to 10^15."""
    offsets = [10 ** 6 + 7, 48 * 64 ** 3 * 3 + 5, 10 ** 12 + 11, 10 ** 15 + 3]
    r = subprocess.run([str(jump_exe), "1", "2", "7"] + [str(n) for n in offsets], capture_output=True, text=True,
                       check=True)
    assert r.stdout.split() == ["0"]


@pytest.mark.parametrize("count,first", [(600000, 0), (600000, 48 * 1000 * 2 + 1), (4097 * 3, 7), (5, 11), (0, 0)])
def test_threaded_pair_draw_equals_one_pass(jump_exe, count, first):
    """The initial conditions' threaded draw (up to 8 threads; shares of at
    least 4,096 pairs, so a few pairs run on one thread and an empty draw
    starts none) hands every pair the numbers one sequential pass would."""
    r = subprocess.run([str(jump_exe), "2", "2", "3", str(count), str(first)], capture_output=True, text=True,
                       check=True)
    assert r.stdout.split() == ["0"]


@pytest.mark.parametrize("seed,level,pr", [(1, 2, 397), (987654, 2, 397), (12345, 1, 202)])
def test_oracle_stream_is_the_published_recurrence(oracle, seed, level, pr):
    """The oracle's stream, read without its code: every block of 12
    delivered numbers is the ring of 48-bit words after a refill, and the
    subtract-with-borrow recurrence with lags (12, 5) in base b = 2^48 is the
    congruential generator Z -> Z / b modulo m = b^12 - b^5 + 1 (the borrow
    enters Z as -c b^12).  So consecutive blocks k, k+1 must satisfy
    Z_{k+1} = b^-pr Z_k (mod m) for one borrow c_k and one c_{k+1} in {0, 1}:
    this pins the lags, the borrow convention and the luxury level's pr
    steps per block with Python integers alone."""
    b = 1 << 48
    m = b ** 12 - b ** 5 + 1
    step = pow(pow(b, -1, m), pr, m)
    words = (oracle.Ranlxd(level, seed).draw(12 * 40) * b).astype(np.int64)
    assert np.array_equal(words.astype(np.float64) / b, oracle.Ranlxd(level, seed).draw(12 * 40))

    def lcg(h, c):
        h = [int(v) for v in h]
        z = sum(h[k] * b ** k for k in range(5)) + sum((h[k] - h[k - 5]) * b ** k for k in range(5, 12))
        return (z - c * b ** 12) % m

    blocks = words.reshape(40, 12)
    for k in range(39):
        here = {lcg(blocks[k], c) * step % m for c in (0, 1)}
        there = {lcg(blocks[k + 1], c) for c in (0, 1)}
        assert here & there, k
    # a wrong decimation or lag fails the same check
    wrong = pow(pow(b, -1, m), pr + 1, m)
    assert not any({lcg(blocks[k], c) * wrong % m for c in (0, 1)} & {lcg(blocks[k + 1], c) for c in (0, 1)}
                   for k in range(39))


@pytest.mark.parametrize("bad_at", [0, 4096 * 3 + 5, 40000 - 1])
def test_threaded_draw_passes_a_callback_exception_to_the_caller(jump_exe, bad_at):
    """An exception thrown by the callback on any worker thread (or on the
    calling thread's own share) is rethrown to the caller after every worker
    has joined, instead of terminating the process."""
    r = subprocess.run([str(jump_exe), "3", "2", "3", "40000", "0", str(bad_at)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.split() == ["caught", "planted"], (r.returncode, r.stdout, r.stderr)


@pytest.mark.parametrize("level,first_block,stride,n", [(2, 0, 37, 300), (2, 5, 1, 40), (1, 1000, 523, 70),
                                                       (2, 10 ** 9, 12345, 20)])
def test_block_states_continue_the_stream(jump_exe, level, first_block, stride, n):
    """The device draw's starting states (one jump per host thread, one
    modular multiplication per further state) continue the stream exactly
    where a jump to the same block does (the jumps themselves are checked
    against the oracle's stream above)."""
    r = subprocess.run([str(jump_exe), "4", str(level), "11", str(first_block), str(stride), str(n)],
                       capture_output=True, text=True, check=True)
    assert r.stdout.split() == ["0"]
