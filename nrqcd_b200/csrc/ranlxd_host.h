// Host random-number generator of the initial conditions (plain C++, no
// CUDA), kept in a header so that it can be checked on its own against the
// CPU oracle's generator.
#pragma once
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <cstddef>
#include <exception>
#include <thread>
#include <vector>

namespace nrqh {

// Arithmetic modulo m = b^12 - b^5 + 1 (b = 2^48) on 12 base-b digits, least
// significant first.  The subtract-with-borrow recurrence of ranlxd with
// lags (12, 5) in base b is a linear congruential generator modulo m with
// multiplier 1/b (Marsaglia and Zaman 1991; Tezuka, L'Ecuyer and Couture
// 1993): for the words h_0 (oldest) .. h_11 (newest) and the borrow c,
//   Z = sum_{k<5} h_k b^k + sum_{5<=k<12} (h_k - h_{k-5}) b^k - c b^12  (mod m)
// advances as Z -> Z/b per step, so n steps are one multiplication by b^-n.
namespace swb {
constexpr int64_t kBase = int64_t(1) << 48;
struct Num {
  int64_t d[12];
};

// t[0..n) signed digits (|t_k| < 2^120), reduced into [0, m); uses
// b^12 = b^5 - 1 (mod m)
inline Num reduce(__int128 *t, int n) {
  for (int pass = 0; pass < 16; ++pass) {
    for (int k = n - 1; k >= 12; --k) {
      t[k - 7] += t[k];
      t[k - 12] -= t[k];
      t[k] = 0;
    }
    __int128 carry = 0;
    for (int k = 0; k < 12; ++k) {
      const __int128 v = t[k] + carry;
      carry = v >> 48;  // floor division: arithmetic shift
      t[k] = v - carry * kBase;
    }
    t[12] = carry;
    n = 13;
    if (carry == 0) break;
  }
  // the value is now in [0, b^12); subtract m once if it is not below it
  __int128 u[12];
  for (int k = 0; k < 12; ++k) u[k] = t[k];
  u[0] -= 1;
  u[5] += 1;
  __int128 carry = 0;
  for (int k = 0; k < 12; ++k) {
    const __int128 v = u[k] + carry;
    carry = v >> 48;
    u[k] = v - carry * kBase;
  }
  Num r;
  for (int k = 0; k < 12; ++k) r.d[k] = (int64_t)(carry > 0 ? u[k] : t[k]);
  return r;
}

inline Num mul(const Num &x, const Num &y) {
  __int128 t[24] = {};
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j) t[i + j] += (__int128)x.d[i] * y.d[j];
  return reduce(t, 24);
}

inline Num pow(Num x, uint64_t e) {
  Num r = {};
  r.d[0] = 1;
  while (e) {
    if (e & 1) r = mul(r, x);
    x = mul(x, x);
    e >>= 1;
  }
  return r;
}

// 1/b modulo m: b (b^11 - b^4) = -1 (mod m)
inline Num inverse_base() {
  __int128 t[13] = {};
  t[12] = 1;
  t[11] = -1;
  t[5] = -1;
  t[4] = 1;
  t[0] = 1;
  return reduce(t, 13);
}

// words h (oldest first, 48-bit integers) and borrow c -> Z
inline Num to_lcg(const int64_t *h, int c) {
  __int128 t[13] = {};
  for (int k = 0; k < 12; ++k) t[k] = h[k] - (k >= 5 ? h[k - 5] : 0);
  t[12] = -c;
  return reduce(t, 13);
}

inline bool equal(const Num &x, const Num &y) {
  for (int k = 0; k < 12; ++k)
    if (x.d[k] != y.d[k]) return false;
  return true;
}

// Z -> words h with borrow 0 that continue the same stream.  Z fixes only
// h_0 + c of the oldest word and the borrow, which the next step reads as a
// sum; h_11 may come out as b (the word 1.0), which the recurrence reads
// exactly as b - 1 with a borrow.  Of the candidates Z and Z - m, the one
// whose words lie in range and map back to Z is taken.
inline bool from_lcg(const Num &z, int64_t *h) {
  for (int cand = 0; cand < 2; ++cand) {
    __int128 t[13] = {};
    for (int k = 0; k < 12; ++k) t[k] = z.d[k];
    if (cand == 1) {  // Z - m = Z - b^12 + b^5 - 1
      t[12] = -1;
      t[5] += 1;
      t[0] -= 1;
      __int128 carry = 0;
      for (int k = 0; k < 13; ++k) {
        const __int128 v = t[k] + carry;
        carry = k < 12 ? v >> 48 : 0;
        t[k] = k < 12 ? v - carry * kBase : v;
      }
    }
    // Z_int = Q - b^5 (Q mod b^7) with Q = sum q_k b^k: the low five digits
    // are q_0..q_4, then q_{j+5} is digit j of R + sum_{i<=j} q_i b^i
    int64_t q[12];
    for (int k = 0; k < 5; ++k) q[k] = (int64_t)t[k];
    __int128 acc[8];
    for (int j = 0; j < 8; ++j) acc[j] = t[j + 5];
    for (int j = 0; j < 7; ++j) {
      acc[j] += q[j];
      __int128 carry = 0;
      for (int i = j; i < 8; ++i) {
        const __int128 v = acc[i] + carry;
        carry = i < 7 ? v >> 48 : 0;
        acc[i] = i < 7 ? v - carry * kBase : v;
      }
      q[j + 5] = (int64_t)acc[j];
      if (j == 6) q[11] = (int64_t)(acc[6] + acc[7] * kBase);
    }
    if (acc[7] < 0 || acc[7] > 1 || (acc[7] == 1 && acc[6] != 0)) continue;
    for (int k = 0; k < 12; ++k) h[k] = q[k];
    if (equal(to_lcg(h, 0), z)) return true;
  }
  return false;
}
}  // namespace swb

// Double-precision RANLUX (M. Luescher, ranlxd v2.1): 12 words of 48-bit
// fractions, subtract-with-borrow x_n = x_{n-5} - x_{n-12} - c, pr recurrence
// steps per 12 delivered numbers (pr = 397 at luxury level 2), seeded from a
// 31-bit shift register — the generator of src/ranlxd_generator.f90:72-350
// as random%InitModule uses it (src/random.f90:126-140).  The words are
// carried as 48-bit integers: the reference's double arithmetic on them is
// exact, so the integer recurrence delivers the same numbers, with a borrow
// chain of two integer operations per step instead of a floating-point
// subtract, compare and select.
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
    for (int k = 0; k < 12; ++k) {
      int64_t acc = 0;
      for (int l = 0; l < 48; ++l) {
        acc = 2 * acc + ((bits[ib] + 1) & 1);
        bits[ib] = (bits[ib] + bits[jb]) & 1;
        ib = (ib + 1) % 31;
        jb = (jb + 1) % 31;
      }
      x_[k] = seeded_[k] = acc;
    }
    carry_ = 0;
    next_ = 12;
    return true;
  }
  // Position the stream so that the next call of next() returns number n
  // (counted from 0 after init), as n sequential calls would: the state
  // before refill n/12 is the seeded state advanced by pr * (n/12)
  // recurrence steps, one multiplication modulo m; the refill then recomputes
  // every word, and n % 12 numbers of the block are skipped.
  bool jump(uint64_t n) {
    const uint64_t blocks = n / 12;
    if (blocks > UINT64_MAX / (uint64_t)pr_) return false;
    const swb::Num z = swb::mul(swb::pow(swb::inverse_base(), blocks * (uint64_t)pr_), swb::to_lcg(seeded_, 0));
    if (!swb::from_lcg(z, x_)) return false;
    carry_ = 0;
    refill();
    next_ = (int)(n % 12);
    return true;
  }
  double next() {
    if (next_ == 12) {
      refill();
      next_ = 0;
    }
    return out_[next_++];
  }
  // continue from a block-start state (words oldest first, borrow 0): the
  // next call of next() refills and returns that block's first number
  void load_block_state(const int64_t *w) {
    for (int k = 0; k < 12; ++k) x_[k] = w[k];
    carry_ = 0;
    next_ = 12;
  }
  const int64_t *seeded_words() const { return seeded_; }
  int steps_per_block() const { return pr_; }

 private:
  // one recurrence step on ring slot i (the oldest word) with lag slot j
  static inline void step(int64_t *x, int i, int j, int64_t &c) {
    int64_t y = x[j] - x[i] - c;
    c = (int64_t)((uint64_t)y >> 63);
    x[i] = y + (c << 48);
  }
  // pr_ steps over the ring held oldest-first from slot 0, then the ring
  // rotated back to oldest-first and the 12 newest words handed out oldest
  // first (the order ranlxd delivers them)
  void refill() {
    int64_t c = carry_;
    int64_t *x = x_;
    for (int rep = 0; rep < pr_ / 12; ++rep) {
#pragma GCC unroll 12
      for (int i = 0; i < 12; ++i) step(x, i, i < 5 ? i + 7 : i - 5, c);
    }
    const int rest = pr_ % 12;
    for (int i = 0; i < rest; ++i) step(x, i, i < 5 ? i + 7 : i - 5, c);
    int64_t r[12];
    for (int k = 0; k < 12; ++k) r[k] = x[(rest + k) % 12];
    const double unit = std::ldexp(1.0, -48);
    for (int k = 0; k < 12; ++k) {
      x[k] = r[k];
      out_[k] = unit * (double)r[k];
    }
    carry_ = c;
  }
  int64_t x_[12] = {};
  int64_t seeded_[12] = {};
  int64_t carry_ = 0;
  double out_[12] = {};
  int pr_ = 397, next_ = 12;
};

// The generator's state at the start of blocks first_block + t * stride
// (t < nstates) of the stream of (level, seed): for each t, the 12 words
// (oldest first, borrow 0) whose next refill delivers that block, into
// words[12 t .. 12 t + 12).  One jump per host thread and one modular
// multiplication per further state (Z_{t+1} = Z_t b^(-pr stride)), split
// over up to max_threads host threads.  False for a seed or level that init
// refuses, or a position the 64-bit step count cannot reach.
inline bool block_states(int level, int64_t seed, uint64_t first_block, uint64_t stride, size_t nstates,
                         int64_t *words, unsigned max_threads = 32) noexcept {
  try {
    Ranlxd probe;
    if (!probe.init(level, seed)) return false;
    const uint64_t pr = (uint64_t)probe.steps_per_block();
    if (nstates == 0) return true;
    const uint64_t last = first_block + stride * (uint64_t)(nstates - 1);
    if ((stride && (uint64_t)(nstates - 1) > (UINT64_MAX - first_block) / stride) || last > UINT64_MAX / pr)
      return false;
    const swb::Num z0 = swb::to_lcg(probe.seeded_words(), 0);
    const swb::Num inv = swb::inverse_base();
    const swb::Num step = swb::pow(inv, stride * pr);
    unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), max_threads));
    nt = (unsigned)std::min<size_t>(nt, (nstates + 63) / 64);
    std::vector<char> ok(nt, 1);
    auto share = [&](unsigned t) {
      const size_t lo = nstates * t / nt, hi = nstates * (t + 1) / nt;
      swb::Num z = swb::mul(swb::pow(inv, (first_block + stride * (uint64_t)lo) * pr), z0);
      for (size_t k = lo; k < hi; ++k) {
        if (!swb::from_lcg(z, words + 12 * k)) {
          ok[t] = 0;
          return;
        }
        z = swb::mul(z, step);
      }
    };
    std::vector<std::thread> pool;
    unsigned started = 1;
    try {
      pool.reserve(nt);
      for (; started < nt; ++started) pool.emplace_back(share, started);
    } catch (...) {  // no more threads: the remaining shares run here
    }
    share(0);
    for (unsigned t = started; t < nt; ++t) share(t);
    for (auto &th : pool) th.join();
    for (char c : ok)
      if (!c) return false;
    return true;
  } catch (...) {
    return false;
  }
}

// f(i, u[first + 2i], u[first + 2i + 1]) for i < count, u the stream of
// (level, seed), on up to max_threads host threads, each starting its share
// of the pairs with a jump: every f sees the numbers one sequential pass
// would hand it.  False for a seed or level that init refuses.
template <class F>
bool draw_pairs(int level, int64_t seed, uint64_t first, size_t count, F f, unsigned max_threads = 32) {
  Ranlxd probe;
  if (!probe.init(level, seed)) return false;
  const size_t min_share = 1 << 12;  // ~0.5 ms of drawing per thread at least
  unsigned nt = std::thread::hardware_concurrency();
  nt = std::max(1u, std::min(nt, max_threads));
  nt = (unsigned)std::min<size_t>(nt, (count + min_share - 1) / min_share);
  if (nt == 0) return true;
  // a share never throws: an exception from f (or from the generator) is
  // kept and rethrown on the calling thread once every worker has joined
  std::vector<std::exception_ptr> errs(nt);
  auto share = [&](unsigned t) -> char {
    try {
      const size_t lo = count * t / nt, hi = count * (t + 1) / nt;
      Ranlxd r;
      r.init(level, seed);
      if (!r.jump(first + 2 * (uint64_t)lo)) return 0;
      for (size_t i = lo; i < hi; ++i) {
        const double u1 = r.next(), u2 = r.next();
        f(i, u1, u2);
      }
      return 1;
    } catch (...) {
      errs[t] = std::current_exception();
      return 0;
    }
  };
  std::vector<std::thread> pool;
  std::vector<char> ok(nt, 1);
  unsigned started = 1;
  try {
    pool.reserve(nt);
    for (; started < nt; ++started) pool.emplace_back([&, started] { ok[started] = share(started); });
  } catch (...) {  // no more threads: the remaining shares run here
  }
  ok[0] = share(0);
  for (unsigned t = started; t < nt; ++t) ok[t] = share(t);
  for (auto &th : pool) th.join();
  for (auto &e : errs)
    if (e) std::rethrow_exception(e);
  for (char c : ok)
    if (!c) return false;
  return true;
}

// draw_pairs for callers behind the C ABI: an exception (from f, or a
// thread or vector that could not be created) becomes a false return
template <class F>
bool draw_pairs_noexcept(int level, int64_t seed, uint64_t first, size_t count, F f,
                         unsigned max_threads = 32) noexcept {
  try {
    return draw_pairs(level, seed, first, count, f, max_threads);
  } catch (...) {
    return false;
  }
}

}  // namespace nrqh
