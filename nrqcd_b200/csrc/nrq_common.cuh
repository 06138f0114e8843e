// Device-side building blocks shared by the gauge and heavy-quark kernels:
// FP64 complex arithmetic on double2, 3x3 colour matrices, the SU(3)
// generators as the reference defines them, and periodic lattice indexing.
//
// Generators: src/su3.f90:97-131 builds them with a column-major reshape,
// so T2, T5 and T7 are the transposes (= negatives) of the textbook
// lambda/2 matrices; the arrays below are the ones the reference holds.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nrq {

// ---------------------------------------------------------------- complex
struct cplx {
  double re, im;
};

__host__ __device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
__host__ __device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)};
}
__host__ __device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx operator*(cplx a, double s) { return {s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cplx conj(cplx a) { return {a.re, -a.im}; }
__host__ __device__ __forceinline__ cplx times_i(cplx a) { return {-a.im, a.re}; }
__host__ __device__ __forceinline__ double norm2(cplx a) { return fma(a.re, a.re, a.im * a.im); }
// acc += a*b
__host__ __device__ __forceinline__ void cmac(cplx &acc, cplx a, cplx b) {
  acc.re = fma(a.re, b.re, fma(-a.im, b.im, acc.re));
  acc.im = fma(a.re, b.im, fma(a.im, b.re, acc.im));
}
// acc += conj(a)*b
__host__ __device__ __forceinline__ void cmac_cj(cplx &acc, cplx a, cplx b) {
  acc.re = fma(a.re, b.re, fma(a.im, b.im, acc.re));
  acc.im = fma(a.re, b.im, fma(-a.im, b.re, acc.im));
}
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
// Smith's algorithm for a/b
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, den = b.re + b.im * r;
    return {(a.re + a.im * r) / den, (a.im - a.re * r) / den};
  } else {
    double r = b.re / b.im, den = b.re * r + b.im;
    return {(a.re * r + a.im) / den, (a.im * r - a.re) / den};
  }
}
// principal square root
__device__ __forceinline__ cplx csqrt_(cplx z) {
  double r = hypot(z.re, z.im);
  if (r == 0.0) return {0.0, 0.0};
  double t = sqrt(0.5 * (r + fabs(z.re)));
  if (z.re >= 0.0) return {t, z.im / (2.0 * t)};
  return {fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}

__device__ __forceinline__ cplx ld(const double2 *p) {
  double2 v = *p;
  return {v.x, v.y};
}
__device__ __forceinline__ cplx ldg(const double2 *p) {
  double2 v = __ldg(p);
  return {v.x, v.y};
}
__device__ __forceinline__ void st(double2 *p, cplx a) { *p = make_double2(a.re, a.im); }

// ---------------------------------------------------------------- 3x3
struct m3 {
  cplx e[9];  // row-major
};

__device__ __forceinline__ m3 m3_zero() {
  m3 r;
#pragma unroll
  for (int k = 0; k < 9; ++k) r.e[k] = {0.0, 0.0};
  return r;
}
__device__ __forceinline__ m3 m3_id() {
  m3 r = m3_zero();
  r.e[0].re = r.e[4].re = r.e[8].re = 1.0;
  return r;
}
__device__ __forceinline__ m3 mul(const m3 &a, const m3 &b) {
  m3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cplx acc = a.e[i * 3] * b.e[j];
      cmac(acc, a.e[i * 3 + 1], b.e[3 + j]);
      cmac(acc, a.e[i * 3 + 2], b.e[6 + j]);
      r.e[i * 3 + j] = acc;
    }
  return r;
}
// a * b^dagger
__device__ __forceinline__ m3 mul_nd(const m3 &a, const m3 &b) {
  m3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cplx acc = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        // a[i][k] * conj(b[j][k])
        cplx bc = conj(b.e[j * 3 + k]);
        cmac(acc, a.e[i * 3 + k], bc);
      }
      r.e[i * 3 + j] = acc;
    }
  return r;
}
// a^dagger * b
__device__ __forceinline__ m3 mul_dn(const m3 &a, const m3 &b) {
  m3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      cplx acc = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) cmac_cj(acc, a.e[k * 3 + i], b.e[k * 3 + j]);
      r.e[i * 3 + j] = acc;
    }
  return r;
}
__device__ __forceinline__ m3 dag(const m3 &a) {
  m3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.e[i * 3 + j] = conj(a.e[j * 3 + i]);
  return r;
}
__device__ __forceinline__ m3 add(const m3 &a, const m3 &b) {
  m3 r;
#pragma unroll
  for (int k = 0; k < 9; ++k) r.e[k] = a.e[k] + b.e[k];
  return r;
}
__device__ __forceinline__ m3 sub(const m3 &a, const m3 &b) {
  m3 r;
#pragma unroll
  for (int k = 0; k < 9; ++k) r.e[k] = a.e[k] - b.e[k];
  return r;
}
__device__ __forceinline__ m3 scale(const m3 &a, double s) {
  m3 r;
#pragma unroll
  for (int k = 0; k < 9; ++k) r.e[k] = s * a.e[k];
  return r;
}
__device__ __forceinline__ cplx trace(const m3 &a) { return a.e[0] + a.e[4] + a.e[8]; }

// ---------------------------------------------------------------- algebra
// M = sum_a alpha_a T^a with the reference's generators.
__device__ __forceinline__ m3 algebra_matrix(const double al[8]) {
  const double h = 0.5, s8 = 0.5 / 1.7320508075688772, d8 = 1.0 / 1.7320508075688772;
  m3 M;
  M.e[0] = {h * al[2] + s8 * al[7], 0.0};
  M.e[4] = {-h * al[2] + s8 * al[7], 0.0};
  M.e[8] = {-d8 * al[7], 0.0};
  // (0,1): T1 -> h ; T2 -> +i h
  M.e[1] = {h * al[0], h * al[1]};
  M.e[3] = {h * al[0], -h * al[1]};
  // (0,2): T4 -> h ; T5 -> +i h
  M.e[2] = {h * al[3], h * al[4]};
  M.e[6] = {h * al[3], -h * al[4]};
  // (1,2): T6 -> h ; T7 -> +i h
  M.e[5] = {h * al[5], h * al[6]};
  M.e[7] = {h * al[5], -h * al[6]};
  return M;
}

// Tr(T^a M) for all eight reference generators.
__device__ __forceinline__ void traces_with_generators(const m3 &M, cplx tr[8]) {
  const double h = 0.5, s8 = 0.5 / 1.7320508075688772, d8 = 1.0 / 1.7320508075688772;
  // Tr(T M) = sum_{rc} T[r][c] M[c][r]
  tr[0] = h * (M.e[3] + M.e[1]);                        // T1: (0,1),(1,0)
  tr[1] = h * (times_i(M.e[3]) - times_i(M.e[1]));      // T2: T[0][1]=+ih, T[1][0]=-ih
  tr[2] = h * (M.e[0] - M.e[4]);                        // T3
  tr[3] = h * (M.e[6] + M.e[2]);                        // T4
  tr[4] = h * (times_i(M.e[6]) - times_i(M.e[2]));      // T5: T[0][2]=+ih, T[2][0]=-ih
  tr[5] = h * (M.e[7] + M.e[5]);                        // T6
  tr[6] = h * (times_i(M.e[7]) - times_i(M.e[5]));      // T7: T[1][2]=+ih, T[2][1]=-ih
  tr[7] = s8 * (M.e[0] + M.e[4]) - d8 * M.e[8];         // T8
}

// exp(i Q) for hermitian traceless Q: exp(iQ) = f0 + f1 Q + f2 Q^2 with the
// coefficients from the Taylor series reduced by Cayley-Hamilton
// (Q^3 = c1 Q + c0, c1 = tr(Q^2)/2, c0 = det Q), after scaling Q by 2^-s
// so that |Q|_F <= 1/2, followed by s squarings in the same polynomial basis.
__device__ __forceinline__ m3 expi_herm(const m3 &Q) {
  m3 Q2 = mul(Q, Q);
  double c1 = 0.5 * (Q2.e[0].re + Q2.e[4].re + Q2.e[8].re);
  // det Q = tr(Q^3)/3 for traceless Q
  double t3 = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) t3 += Q.e[i * 3 + k].re * Q2.e[k * 3 + i].re - Q.e[i * 3 + k].im * Q2.e[k * 3 + i].im;
  double c0 = t3 / 3.0;
  double nf = sqrt(2.0 * c1);
  int s = 0;
  while (nf > 0.5 && s < 64) {
    nf *= 0.5;
    ++s;
  }
  double c1s = ldexp(c1, -2 * s), c0s = ldexp(c0, -3 * s);
  // Taylor: sum_n (i^n/n!) Q_s^n with Q_s^n = a I + b Q_s + d Q_s^2
  double a = 1.0, b = 0.0, d = 0.0;
  cplx f0 = {1.0, 0.0}, f1 = {0.0, 0.0}, f2 = {0.0, 0.0};
  double bound = 1.0;
  for (int n = 1; n <= 30; ++n) {
    bound *= nf / n;
    if (bound < 1e-20) break;
    double an = d * c0s, bn = fma(d, c1s, a), dn = b;
    double inv = 1.0 / n;
    a = an * inv;
    b = bn * inv;
    d = dn * inv;
    switch (n & 3) {
      case 0: f0.re += a; f1.re += b; f2.re += d; break;
      case 1: f0.im += a; f1.im += b; f2.im += d; break;
      case 2: f0.re -= a; f1.re -= b; f2.re -= d; break;
      default: f0.im -= a; f1.im -= b; f2.im -= d; break;
    }
  }
  for (int k = s; k >= 1; --k) {
    double c1k = ldexp(c1, -2 * k), c0k = ldexp(c0, -3 * k);
    cplx f12 = f1 * f2, f22 = f2 * f2;
    cplx g0 = f0 * f0 + (2.0 * c0k) * f12;
    cplx g1 = 2.0 * (f0 * f1) + (2.0 * c1k) * f12 + c0k * f22;
    cplx g2 = 2.0 * (f0 * f2) + f1 * f1 + c1k * f22;
    f0 = g0;
    f1 = 0.5 * g1;
    f2 = 0.25 * g2;
  }
  m3 G;
#pragma unroll
  for (int k = 0; k < 9; ++k) G.e[k] = f1 * Q.e[k] + f2 * Q2.e[k];
  G.e[0] = G.e[0] + f0;
  G.e[4] = G.e[4] + f0;
  G.e[8] = G.e[8] + f0;
  return G;
}

// ---------------------------------------------------------------- lattice
struct Lat {
  int64_t nx, ny, nz, V;
  double a0, a[3];
};

__device__ __forceinline__ void coords(const Lat &L, int64_t s, int64_t &x, int64_t &y, int64_t &z) {
  x = s % L.nx;
  int64_t t = s / L.nx;
  y = t % L.ny;
  z = t / L.ny;
}
// neighbour of site s in direction d (0..2) by +1 (sgn>0) or -1
__device__ __forceinline__ int64_t nb(const Lat &L, int64_t s, int d, int sgn) {
  int64_t x, y, z;
  coords(L, s, x, y, z);
  if (d == 0) {
    x += sgn;
    x = (x < 0) ? x + L.nx : (x >= L.nx ? x - L.nx : x);
  } else if (d == 1) {
    y += sgn;
    y = (y < 0) ? y + L.ny : (y >= L.ny ? y - L.ny : y);
  } else {
    z += sgn;
    z = (z < 0) ? z + L.nz : (z >= L.nz ? z - L.nz : z);
  }
  return x + L.nx * (y + L.ny * z);
}

// link U_d(s) from SoA planes: plane (d*9 + r*3 + c)
__device__ __forceinline__ m3 load_link(const double2 *__restrict__ U, int64_t V, int64_t s, int d) {
  m3 m;
  const double2 *p = U + (int64_t)d * 9 * V + s;
#pragma unroll
  for (int k = 0; k < 9; ++k) m.e[k] = ldg(p + k * V);
  return m;
}
__device__ __forceinline__ void store_link(double2 *__restrict__ U, int64_t V, int64_t s, int d, const m3 &m) {
  double2 *p = U + (int64_t)d * 9 * V + s;
#pragma unroll
  for (int k = 0; k < 9; ++k) st(p + k * V, m.e[k]);
}

}  // namespace nrq
