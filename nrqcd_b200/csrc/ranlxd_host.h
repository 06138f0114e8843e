// Host random-number generator of the initial conditions (plain C++, no
// CUDA), kept in a header so that it can be checked on its own against the
// CPU oracle's generator.
#pragma once
#include <cmath>
#include <cstdint>

namespace nrqh {

// Double-precision RANLUX (M. Luescher, ranlxd v2.1): 12 words of 48-bit
// fractions, subtract-with-borrow x_n = x_{n-5} - x_{n-12} - c, pr recurrence
// steps per 12 delivered numbers (pr = 397 at luxury level 2), seeded from a
// 31-bit shift register — the generator of src/ranlxd_generator.f90:72-350
// as random%InitModule uses it (src/random.f90:126-140).
class Ranlxd {
 public:
  bool init(int level, int64_t seed) {
    if (level == 1) pr_ = 202;
    else if (level == 2) pr_ = 397;
    else return false;
    if (seed <= 0 || seed > 2147483647LL) return false;
    int bits[31];
    int64_t v = seed;
    for (int k = 0; k < 31; ++k) {
      bits[k] = (int)(v & 1);
      v >>= 1;
    }
    int ib = 0, jb = 18;
    const double unit = std::ldexp(1.0, -48);
    for (int k = 0; k < 12; ++k) {
      double acc = 0.0;
      for (int l = 0; l < 48; ++l) {
        acc = 2.0 * acc + (double)((bits[ib] + 1) & 1);
        bits[ib] = (bits[ib] + bits[jb]) & 1;
        ib = (ib + 1) % 31;
        jb = (jb + 1) % 31;
      }
      w_[k] = unit * acc;
    }
    borrow_ = 0.0;
    pos_ = 11;
    lag_ = 7;
    last_ = 0;
    return true;
  }
  double next() {
    pos_ = pos_ == 11 ? 0 : pos_ + 1;
    if (pos_ == last_) refill();
    return w_[pos_];
  }

 private:
  // pr_ subtract-with-borrow steps; the ring indices wrap by comparison (the
  // arithmetic of every step is unchanged)
  void refill() {
    const double unit = std::ldexp(1.0, -48);
    int i = pos_, j = lag_;
    double borrow = borrow_;
    for (int k = 0; k < pr_; ++k) {
      double y = (w_[j] - w_[i]) - borrow;
      const bool neg = y < 0.0;
      borrow = neg ? unit : 0.0;
      if (neg) y += 1.0;
      w_[i] = y;
      i = i == 11 ? 0 : i + 1;
      j = j == 11 ? 0 : j + 1;
    }
    borrow_ = borrow;
    pos_ = i;
    lag_ = j;
    last_ = i;
  }
  double w_[12];
  double borrow_ = 0.0;
  int pr_ = 397, pos_ = 11, lag_ = 7, last_ = 0;
};

}  // namespace nrqh
