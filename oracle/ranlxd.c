/*
 * Oracle (test infrastructure only): double-precision RANLUX generator and
 * Box-Muller normals.
 *
 * Restates M. Luescher's published ranlxd algorithm (v2.1, Dec 1997) as
 * carried by the reference in src/ranlxd_generator.f90:
 *   - seeding from a 31-bit shift register   (ranlxd_init, :251-317)
 *   - subtract-with-borrow x_n = x_{n-5} - x_{n-12} - c on 48-bit fractions
 *     with pr (=202 or 397) recurrence steps per 12 delivered numbers
 *     (update, :72-207; the 12-fold unrolled block there is arithmetically
 *     the same sequence of single steps used below)
 *   - delivery loop (ranlxd, :323-350), state get/reset (:355-438).
 * Box-Muller complex normals follow src/random.f90:238-255.
 */
#include <math.h>
#include "oracle.h"

static void define_constants(oc_ranlxd_state *s) {
  s->init = 1;
  s->one_bit = ldexp(1.0, -48);
  for (int k = 0; k < 12; ++k) s->next[k] = (k + 1) % 12;
}

int oc_ranlxd_init(oc_ranlxd_state *s, int64_t level, int64_t seed) {
  int64_t xbit[31];
  if (level == 1) s->pr = 202;
  else if (level == 2) s->pr = 397;
  else return -1;
  define_constants(s);
  int64_t i = seed;
  for (int k = 0; k < 31; ++k) {
    xbit[k] = ((i % 2) + 2) % 2;
    i /= 2;
  }
  if (seed <= 0 || i != 0) return -2;
  int ibit = 0, jbit = 18;
  for (int k = 0; k < 12; ++k) {
    double x = 0.0;
    for (int l = 0; l < 48; ++l) {
      double y = (double)((xbit[ibit] + 1) % 2);
      x = x + x + y;
      xbit[ibit] = (xbit[ibit] + xbit[jbit]) % 2;
      ibit = (ibit + 1) % 31;
      jbit = (jbit + 1) % 31;
    }
    s->xdbl[k] = s->one_bit * x;
  }
  s->carry = 0.0;
  s->ir = 11;
  s->jr = 7;
  s->ir_old = 0;
  return 0;
}

/* pr single steps of the borrow recurrence starting at ir (jr = ir+7). */
static void update(oc_ranlxd_state *s) {
  double *x = s->xdbl;
  int64_t ir = s->ir, jr = s->jr;
  double carry = s->carry;
  for (int64_t k = 0; k < s->pr; ++k) {
    double y = x[jr] - x[ir];
    y = y - carry;
    if (y < 0.0) {
      carry = s->one_bit;
      y = y + 1.0;
    } else {
      carry = 0.0;
    }
    x[ir] = y;
    ir = s->next[ir];
    jr = s->next[jr];
  }
  s->ir = ir;
  s->jr = jr;
  s->carry = carry;
  s->ir_old = ir;
}

void oc_ranlxd(oc_ranlxd_state *s, double *r, int64_t n) {
  if (!s->init) oc_ranlxd_init(s, 1, 1);
  for (int64_t k = 0; k < n; ++k) {
    s->ir = s->next[s->ir];
    if (s->ir == s->ir_old) update(s);
    r[k] = s->xdbl[s->ir];
  }
}

void oc_ranlxd_get(const oc_ranlxd_state *s, int64_t state[25]) {
  const double sbase = ldexp(1.0, 24), base = ldexp(1.0, 48);
  for (int k = 0; k < 12; ++k) {
    double x = sbase * s->xdbl[k];
    double y2 = trunc(x);
    double y1 = sbase * (x - y2);
    state[2 * k] = (int64_t)y1;
    state[2 * k + 1] = (int64_t)y2;
  }
  int64_t k = 12 * s->pr + s->ir;
  k = 12 * k + s->jr;
  k = 12 * k + s->ir_old;
  state[24] = 2 * k + (int64_t)(s->carry * base);
}

int oc_ranlxd_reset(oc_ranlxd_state *s, const int64_t state[25]) {
  const double sbase = ldexp(1.0, 24);
  define_constants(s);
  for (int k = 0; k < 24; ++k)
    if (state[k] >= (int64_t)sbase || state[k] < 0) return -5;
  int64_t k = state[24];
  if (k < 0) return -5;
  s->carry = s->one_bit * (double)(k % 2);
  k /= 2;
  s->ir_old = k % 12;
  k /= 12;
  s->jr = k % 12;
  k /= 12;
  s->ir = k % 12;
  s->pr = k / 12;
  if ((s->pr != 202 && s->pr != 397) || s->jr != (s->ir_old + 7) % 12) return -5;
  for (int j = 0; j < 12; ++j) {
    double y1 = (double)state[2 * j], y2 = (double)state[2 * j + 1];
    s->xdbl[j] = s->one_bit * (y1 + y2 * sbase);
  }
  return 0;
}

void oc_random_normal_cmplx(oc_ranlxd_state *s, int64_t n, double *out) {
  const double twopi = 2.0 * acos(-1.0);
  double r[2];
  for (int64_t i = 0; i < n; ++i) {
    oc_ranlxd(s, r, 2);
    double rad = sqrt(-2.0 * log(r[0]));
    out[2 * i] = rad * cos(twopi * r[1]);
    out[2 * i + 1] = rad * sin(twopi * r[1]);
  }
}
