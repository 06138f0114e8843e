"""A second, independent restatement of the ranlxd seeding and stream.

The oracle's generator (oracle/ranlxd.c) and the product's host generator
(nrqcd_b200/csrc/ranlxd_host.h) are both compared with the oracle's stream
elsewhere, so the 31-bit shift register that fills the first twelve 48-bit
words would otherwise rest on one restatement only.  This file restates it
once more, in Python integers, from the reference's Fortran module
(src/ranlxd_generator.f90: ranlxd_init 251-317, update 70-219, ranlxd
324-350), which itself follows Luescher's "Double precision implementation of
the random number generator ranlux" (December 1997):

- the seed's 31 bits, least significant first, run through the shift
  register x_k <- x_k + x_{k+18} (mod 2) over 31 cells (ranlxd_init :287-311);
- each of the 12 words takes 48 complemented bits of the register, most
  significant first (:300-302: y = mod(xbit + 1, 2); x = 2x + y);
- the subtract-with-borrow recurrence with lags (12, 5) in base 2^48
  (x_i <- x_{i+7} - x_i - c, indices mod 12) runs pr = 202 (level 1) or 397
  (level 2) steps per block of 12 delivered numbers (update :70-219);
- delivery starts at ir = 11, jr = 7, ir_old = 0: the first draw refills
  (ranlxd :336-344).

Nothing here reads the oracle's or the product's code.
"""
import numpy as np
import pytest

B48 = 1 << 48


class RestatedRanlxd:
    def __init__(self, level, seed):
        if level not in (1, 2):
            raise ValueError("luxury level must be 1 or 2")
        if not 1 <= seed <= 2 ** 31 - 1:
            raise ValueError("seed must be between 1 and 2^31 - 1")
        self.pr = 202 if level == 1 else 397
        xbit = [(seed >> k) & 1 for k in range(31)]
        ibit, jbit = 0, 18
        self.x = []
        for _ in range(12):
            w = 0
            for _ in range(48):
                w = 2 * w + (xbit[ibit] + 1) % 2
                xbit[ibit] = (xbit[ibit] + xbit[jbit]) % 2
                ibit, jbit = (ibit + 1) % 31, (jbit + 1) % 31
            self.x.append(w)
        self.seeded = list(self.x)
        self.carry = 0
        self.ir, self.jr, self.ir_old = 11, 7, 0

    def _step(self):
        y = self.x[self.jr] - self.x[self.ir] - self.carry
        self.carry = 1 if y < 0 else 0
        self.x[self.ir] = y + B48 if y < 0 else y
        self.ir, self.jr = (self.ir + 1) % 12, (self.jr + 1) % 12

    def _update(self):
        # the reference unrolls the middle part in blocks of 12 starting at
        # ir = 0; one step at a time through the same cells is the same
        # recurrence, so pr single steps from the current (ir, jr) restate it
        for _ in range(self.pr):
            self._step()
        self.ir_old = self.ir

    def draw(self, n):
        out = np.empty(n)
        for k in range(n):
            self.ir = (self.ir + 1) % 12
            if self.ir == self.ir_old:
                # delivery moves ir alone and update() moves ir and jr
                # together, so jr is still seven cells ahead of ir_old here
                self.jr = (self.ir + 7) % 12
                self._update()
            out[k] = self.x[self.ir] / B48
        return out


def test_first_words_are_the_complemented_shift_register():
    """Seed 1: the register holds one set bit, so the first 18 output bits of
    word 0 are the complements of zeros (all ones) except the first."""
    r = RestatedRanlxd(2, 1)
    w0 = r.seeded[0]
    bits = [(w0 >> (47 - k)) & 1 for k in range(48)]
    assert bits[0] == 0 and all(b == 1 for b in bits[1:18])


@pytest.mark.parametrize("seed,level", [(1, 2), (2, 2), (2 ** 31 - 1, 2), (12345, 1), (1, 1), (987654321, 2)])
def test_restated_stream_equals_the_oracle(oracle, seed, level):
    n = 12 * 60
    got = RestatedRanlxd(level, seed).draw(n)
    want = oracle.Ranlxd(level, seed).draw(n)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("seed", [0, -1, 2 ** 31])
def test_seed_range(seed):
    with pytest.raises(ValueError):
        RestatedRanlxd(2, seed)
