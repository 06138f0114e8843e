// Heavy-quark kernels of the hot path (FP64): the Crank-Nicolson step of
// src/nrqcd.f90:1053-1168 with the operator PETSc assembles in
// BuildSystemMatrix (src/nrqcd.f90:1175-1387) applied matrix-free.
//
// Operator.  With kappa = -i a0 dt/2 the source writes, per row site x,
// 6x6 blocks SubMat(x,y) = delta_xy 1 + kappa * (sum of terms); PETSc reads
// each column-major block row-major (src/nrqcd.f90:1014-1018), so the
// evolved operator holds SubMat^T.  Splitting the terms,
//   A = 1 + sum_t alpha_t G_t,  t in {kinetic, magnetic, Darwin, spin-orbit}
// with every G_t hermitian (c_t factored out), hence A^H = 1 + sum conj(alpha_t) G_t.
// Per site, with E_j(y) = -Re(E~_j^a(y) T^a)/(a0 a_j) (= -F_0j of
// gauge:1563-1581 for eigenphases inside the principal branch):
//   G_kin  psi(x) = sum_i 1/a_i^2 [psi(x) - 1/2 (U_i(x)^T x 1) psi(x+i)
//                                           - 1/2 (U_i(x-i)^* x 1) psi(x-i)]
//   G_mag  psi(x) = (B(x)^T x 1) psi(x),  B = sum_i F_jk (nrqcd:1669-1693: B_i x 1, no sigma)
//   G_dar  psi(x) = (D(x)^T x 1) psi(x),  D = sum_i [U_i E_i(x+i) U_i^+ - U_i(x-i)^+ E_i(x-i) U_i(x-i)]/(2a_i)
//   G_so   psi(x) = sum_i sum_(j,k,eps) eps i [(DE_ij(x)^T x s_k^T) psi(x+i)
//                                            - (DE_ij(x-i)^* x s_k^T) psi(x-i)]
//          DE_ij(x) = (E_j(x) U_i(x) + U_i(x) E_j(x+i))/(2 a_i)
//   alpha_kin = kappa c1/M, alpha_mag = -kappa c2/(2M), alpha_dar = -kappa c3/(8M^2),
//   alpha_so = -kappa c4/(8M^2); antiquark: M -> -M, c -> conj(c).
//
// Layout: propagator planes (species*36 + col*6 + row), V complex each.
// The stencil kernels live in cn_mv3.cu (TMA-staged) and cn_mv.cu
// (register-tiled); this file holds the per-step preparation, the BiCGStab
// vector updates and scalar stages, and the propagator I/O and observables.
#include <algorithm>

#include "nrq_eigen.cuh"
#include "nrq_kernels.cuh"

namespace nrq {

// Re(LogU(P)/i) = Im(S^+ diag(i theta) S) for unitary P (matrixoperations:510-531)
__device__ void field_strength_from_plaquette(const m3 &P, double scale_, double F[9]) {
  cplx ev[3];
  m3 S;
  eigenc3(P, ev, S);
  double th[3];
  for (int k = 0; k < 3; ++k) th[k] = atan2(ev[k].im, ev[k].re);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) {
        // Re(conj(S[k][r]) * S[k][c])
        cplx a = S.e[k * 3 + r], b = S.e[k * 3 + c];
        acc += th[k] * (a.re * b.re + a.im * b.im);
      }
      F[r * 3 + c] = acc * scale_;
    }
}

// Same quantity for plaquettes inside the principal branch with small
// angles, without an eigen-decomposition.  For unitary P = exp(iH) whose
// eigenphases satisfy |theta| < pi/2, K = (P - P^+)/(2i) = sin(H) and
// H = asin(K) = sum_n c_n K^(2n+1), c_n = (2n)!/(4^n (n!)^2 (2n+1)).  The
// powers of K are reduced with Cayley-Hamilton (K^3 = t1 K^2 - t2 K + t3 1
// with the real invariants of the hermitian K), so the series runs on three
// real coefficients and H = f0 1 + f1 K + f2 K^2 is assembled once.  Used
// when |K|_F <= 0.3 and Re Tr P > 2 (all eigenphases then lie within
// |theta| < 0.31); the Jacobi route handles every other plaquette.  Both
// return Re(LogU(P)/i) to rounding.
__device__ bool field_strength_small_angle(const m3 &P, double scale_, double F[9]) {
  const double trP = P.e[0].re + P.e[4].re + P.e[8].re;
  m3 K;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      // (P[r][c] - conj(P[c][r])) / (2i)
      cplx d = P.e[r * 3 + c] - conj(P.e[c * 3 + r]);
      K.e[r * 3 + c] = {0.5 * d.im, -0.5 * d.re};
    }
  double nf2 = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) nf2 += norm2(K.e[k]);
  if (!(trP > 2.0) || !(nf2 <= 0.09)) return false;
  const double rho = sqrt(nf2);
  const m3 K2 = mul(K, K);
  const double t1 = K.e[0].re + K.e[4].re + K.e[8].re;
  const double trK2 = K2.e[0].re + K2.e[4].re + K2.e[8].re;
  const double t2 = 0.5 * (t1 * t1 - trK2);
  // det K (real for hermitian K)
  const cplx det = K.e[0] * (K.e[4] * K.e[8] - K.e[5] * K.e[7]) - K.e[1] * (K.e[3] * K.e[8] - K.e[5] * K.e[6]) +
                   K.e[2] * (K.e[3] * K.e[7] - K.e[4] * K.e[6]);
  const double t3 = det.re;
  // K^m = a 1 + b K + d K^2 ; start m = 1
  double a = 0.0, b = 1.0, d = 0.0;
  double f0 = 0.0, f1 = 1.0, f2 = 0.0;  // c_0 K
  double cn = 1.0, pw = rho;            // c_n (n = 0) and rho^(2n+1)
  for (int n = 1; n <= 40; ++n) {
    // two multiplications by K: K^(2n+1) from K^(2n-1)
    for (int rep = 0; rep < 2; ++rep) {
      const double an = d * t3, bn = a - d * t2, dn = b + d * t1;
      a = an;
      b = bn;
      d = dn;
    }
    cn *= (double)(2 * n - 1) * (double)(2 * n - 1) / ((double)(2 * n) * (double)(2 * n + 1));
    pw *= nf2;
    f0 += cn * a;
    f1 += cn * b;
    f2 += cn * d;
    if (cn * pw < 1e-19 * rho) break;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double h = f1 * K.e[k].re + f2 * K2.e[k].re + ((k % 4 == 0) ? f0 : 0.0);
    F[k] = h * scale_;
  }
  return true;
}

// E_j(y) entering the CN operator: -Re(sum_a E~^a T^a)/a0/a_j (real symmetric)
__device__ __forceinline__ m3 efield_cn(const Lat &L, const double *__restrict__ E, int64_t y, int j) {
  const int64_t V = L.V;
  const double h = 0.5, s8 = 0.5 / 1.7320508075688772, d8 = 1.0 / 1.7320508075688772;
  const double *e = E + (int64_t)(j * 8) * V + y;
  double e1 = __ldg(e), e3 = __ldg(e + 2 * V), e4 = __ldg(e + 3 * V), e6 = __ldg(e + 5 * V),
         e8 = __ldg(e + 7 * V);
  const double f = -1.0 / L.a0 / L.a[j];
  m3 M = m3_zero();
  M.e[0].re = (h * e3 + s8 * e8) * f;
  M.e[4].re = (-h * e3 + s8 * e8) * f;
  M.e[8].re = (-d8 * e8) * f;
  M.e[1].re = M.e[3].re = (h * e1) * f;
  M.e[2].re = M.e[6].re = (h * e4) * f;
  M.e[5].re = M.e[7].re = (h * e6) * f;
  return M;
}

__global__ void __launch_bounds__(128) k_cn_prepare(Lat L, const double2 *__restrict__ U,
                                                    const double *__restrict__ E, double2 *__restrict__ Dsum,
                                                    double *__restrict__ Bsum, double2 *__restrict__ DE) {
  int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (x >= L.V) return;
  const int64_t V = L.V;
  // Darwin
  m3 D = m3_zero();
  for (int i = 0; i < 3; ++i) {
    int64_t xp = nb(L, x, i, +1), xm = nb(L, x, i, -1);
    m3 u = load_link(U, V, x, i), um = load_link(U, V, xm, i);
    m3 t1 = mul_nd(mul(u, efield_cn(L, E, xp, i)), u);
    m3 t2 = mul(mul_dn(um, efield_cn(L, E, xm, i)), um);
    D = add(D, scale(sub(t1, t2), 1.0 / (2.0 * L.a[i])));
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) st(Dsum + (int64_t)k * V + x, D.e[k]);
  // magnetic: B_i = F_jk with (i,j,k) cyclic
  double B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3, k = (i + 2) % 3;
    // P_jk = U_j(x) U_k(x+j) U_j(x+k)^+ U_k(x)^+
    m3 P = mul_nd(mul_nd(mul(load_link(U, V, x, j), load_link(U, V, nb(L, x, j, +1), k)),
                         load_link(U, V, nb(L, x, k, +1), j)),
                  load_link(U, V, x, k));
    double F[9];
    if (!field_strength_small_angle(P, 1.0 / L.a[j] / L.a[k], F))
      field_strength_from_plaquette(P, 1.0 / L.a[j] / L.a[k], F);
    for (int m = 0; m < 9; ++m) B[m] += F[m];
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) Bsum[(int64_t)k * V + x] = B[k];
  // spin-orbit colour matrices
  for (int i = 0; i < 3; ++i) {
    int64_t xp = nb(L, x, i, +1);
    m3 u = load_link(U, V, x, i);
    for (int perm = 0; perm < 2; ++perm) {
      int j = perm == 0 ? (i + 1) % 3 : (i + 2) % 3;
      m3 d = scale(add(mul(efield_cn(L, E, x, j), u), mul(u, efield_cn(L, E, xp, j))), 0.5 / L.a[i]);
      double2 *dst = DE + (int64_t)((i * 2 + perm) * 9) * V + x;
#pragma unroll
      for (int k = 0; k < 9; ++k) st(dst + (int64_t)k * V, d.e[k]);
    }
  }
}

void launch_cn_prepare(Lat L, const double2 *U, const double *E, double2 *Dsum, double *Bsum, double2 *DE,
                       cudaStream_t st) {
  int64_t nb_ = (L.V + 127) / 128;
  k_cn_prepare<<<(unsigned)nb_, 128, 0, st>>>(L, U, E, Dsum, Bsum, DE);
}

__device__ __forceinline__ cplx scal_c(const double *sc, int col, int slot) {
  return {sc[col * SC_STRIDE + slot], sc[col * SC_STRIDE + slot + 1]};
}


// ------------------------------------------------------------ BiCGStab vector updates
// s = r - alpha v ; x += alpha p + omega s ; r = s - omega t ; partials (rh.r), (r.r)
__global__ void __launch_bounds__(384) k_vec_xr(int64_t V, double2 *__restrict__ X, double2 *__restrict__ R,
                                                const double2 *__restrict__ P, const double2 *__restrict__ Vv,
                                                const double2 *__restrict__ T, const double2 *__restrict__ RH,
                                                const double *__restrict__ scal, double *__restrict__ partials) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t x0 = (int64_t)blockIdx.x * CN_SITES_PER_BLOCK + lane;
  const bool active = x0 < V;
  const int64_t pb = (int64_t)(w * 6) * V;
  const cplx al = scal_c(scal, w, SC_ALPHA), om = scal_c(scal, w, SC_OMEGA);
  double q[3] = {0.0, 0.0, 0.0};
  if (active) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int64_t o = pb + (int64_t)r * V + x0;
      cplx s = ld(R + o) - al * ldg(Vv + o);
      cplx xn = ld(X + o) + al * ldg(P + o) + om * s;
      cplx rn = s - om * ldg(T + o);
      st(X + o, xn);
      st(R + o, rn);
      cplx d = {0.0, 0.0};
      cmac_cj(d, ldg(RH + o), rn);
      q[0] += d.re;
      q[1] += d.im;
      q[2] += norm2(rn);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q[k] += __shfl_down_sync(0xffffffffu, q[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) partials[((int64_t)blockIdx.x * CN_COLS + w) * 3 + k] = q[k];
}

// p = r + beta (p - omega v)
__global__ void __launch_bounds__(384) k_vec_p(int64_t V, double2 *__restrict__ P, const double2 *__restrict__ R,
                                               const double2 *__restrict__ Vv, const double *__restrict__ scal) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t x0 = (int64_t)blockIdx.x * CN_SITES_PER_BLOCK + lane;
  if (x0 >= V) return;
  const int64_t pb = (int64_t)(w * 6) * V;
  const cplx be = scal_c(scal, w, SC_BETA), om = scal_c(scal, w, SC_OMEGA);
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const int64_t o = pb + (int64_t)r * V + x0;
    st(P + o, ldg(R + o) + be * (ld(P + o) - om * ldg(Vv + o)));
  }
}

// s = r - alpha v (materialised for the TMA-staged and tensor-core
// stencils); with partials, also the per-column partial sums of |s|^2 for
// the half-step convergence check
__global__ void __launch_bounds__(384) k_vec_s(int64_t V, double2 *__restrict__ S, const double2 *__restrict__ R,
                                               const double2 *__restrict__ Vv, const double *__restrict__ scal,
                                               double *__restrict__ partials) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t x0 = (int64_t)blockIdx.x * CN_SITES_PER_BLOCK + lane;
  const int64_t pb = (int64_t)(w * 6) * V;
  const cplx al = scal_c(scal, w, SC_ALPHA);
  double q = 0.0;
  if (x0 < V) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int64_t o = pb + (int64_t)r * V + x0;
      const cplx s = ldg(R + o) - al * ldg(Vv + o);
      st(S + o, s);
      q += norm2(s);
    }
  }
  if (!partials) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) q += __shfl_down_sync(0xffffffffu, q, o);
  if (lane == 0) partials[(int64_t)blockIdx.x * CN_COLS + w] = q;
}

// x += alpha p: the solution after a half step that met the tolerance
__global__ void __launch_bounds__(384) k_vec_xp(int64_t V, double2 *__restrict__ X, const double2 *__restrict__ P,
                                                const double *__restrict__ scal) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t x0 = (int64_t)blockIdx.x * CN_SITES_PER_BLOCK + lane;
  if (x0 >= V) return;
  const int64_t pb = (int64_t)(w * 6) * V;
  const cplx al = scal_c(scal, w, SC_ALPHA);
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const int64_t o = pb + (int64_t)r * V + x0;
    st(X + o, ld(X + o) + al * ldg(P + o));
  }
}

// x += alpha p + omega s ; r = s - omega t ; partials (rh.r), (r.r)   (s materialised)
__global__ void __launch_bounds__(384) k_vec_xr_s(int64_t V, double2 *__restrict__ X, double2 *__restrict__ R,
                                                  const double2 *__restrict__ P, const double2 *__restrict__ S,
                                                  const double2 *__restrict__ T, const double2 *__restrict__ RH,
                                                  const double *__restrict__ scal, double *__restrict__ partials) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t x0 = (int64_t)blockIdx.x * CN_SITES_PER_BLOCK + lane;
  const bool active = x0 < V;
  const int64_t pb = (int64_t)(w * 6) * V;
  const cplx al = scal_c(scal, w, SC_ALPHA), om = scal_c(scal, w, SC_OMEGA);
  double q[3] = {0.0, 0.0, 0.0};
  if (active) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int64_t o = pb + (int64_t)r * V + x0;
      const cplx s = ldg(S + o);
      const cplx xn = ld(X + o) + al * ldg(P + o) + om * s;
      const cplx rn = s - om * ldg(T + o);
      st(X + o, xn);
      st(R + o, rn);
      cplx d = {0.0, 0.0};
      cmac_cj(d, ldg(RH + o), rn);
      q[0] += d.re;
      q[1] += d.im;
      q[2] += norm2(rn);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q[k] += __shfl_down_sync(0xffffffffu, q[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) partials[((int64_t)blockIdx.x * CN_COLS + w) * 3 + k] = q[k];
}

// The merged update after t = A^H s (MV_T2 left omega and beta):
// x += alpha p + omega s ; r = s - omega t ; p = r + beta (p - omega v) ;
// partials (r.r).  One pass of 5 reads and 3 writes in place of the x, r
// update (5 reads, rh included, 2 writes) and the p update (3 reads, 1 write).
__global__ void __launch_bounds__(384) k_vec_xrp(int64_t V, double2 *__restrict__ X, double2 *__restrict__ R,
                                                 double2 *__restrict__ P, const double2 *__restrict__ S,
                                                 const double2 *__restrict__ T, const double2 *__restrict__ Vv,
                                                 const double *__restrict__ scal, double *__restrict__ partials) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t x0 = (int64_t)blockIdx.x * CN_SITES_PER_BLOCK + lane;
  const int64_t pb = (int64_t)(w * 6) * V;
  const cplx al = scal_c(scal, w, SC_ALPHA), om = scal_c(scal, w, SC_OMEGA), be = scal_c(scal, w, SC_BETA);
  double q = 0.0;
  if (x0 < V) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const int64_t o = pb + (int64_t)r * V + x0;
      const cplx s = ldg(S + o), p = ld(P + o);
      const cplx rn = s - om * ldg(T + o);
      st(X + o, ld(X + o) + al * p + om * s);
      st(R + o, rn);
      st(P + o, rn + be * (p - om * ldg(Vv + o)));
      q += norm2(rn);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) q += __shfl_down_sync(0xffffffffu, q, o);
  if (lane == 0) partials[(int64_t)blockIdx.x * CN_COLS + w] = q;
}

void launch_vec_xrp(Lat L, double2 *x, double2 *r, double2 *p, const double2 *s, const double2 *t,
                    const double2 *v, const double *scal, double *partials, cudaStream_t st) {
  unsigned nb_ = (unsigned)((L.V + CN_SITES_PER_BLOCK - 1) / CN_SITES_PER_BLOCK);
  k_vec_xrp<<<nb_, 32 * CN_COLS, 0, st>>>(L.V, x, r, p, s, t, v, scal, partials);
}

void launch_vec_s(Lat L, double2 *s, const double2 *r, const double2 *v, const double *scal, cudaStream_t st,
                  double *partials) {
  unsigned nb_ = (unsigned)((L.V + CN_SITES_PER_BLOCK - 1) / CN_SITES_PER_BLOCK);
  k_vec_s<<<nb_, 32 * CN_COLS, 0, st>>>(L.V, s, r, v, scal, partials);
}
void launch_vec_xp(Lat L, double2 *x, const double2 *p, const double *scal, cudaStream_t st) {
  unsigned nb_ = (unsigned)((L.V + CN_SITES_PER_BLOCK - 1) / CN_SITES_PER_BLOCK);
  k_vec_xp<<<nb_, 32 * CN_COLS, 0, st>>>(L.V, x, p, scal);
}
void launch_vec_xr_s(Lat L, double2 *x, double2 *r, const double2 *p, const double2 *s, const double2 *t,
                     const double2 *rh, const double *scal, double *partials, cudaStream_t st) {
  unsigned nb_ = (unsigned)((L.V + CN_SITES_PER_BLOCK - 1) / CN_SITES_PER_BLOCK);
  k_vec_xr_s<<<nb_, 32 * CN_COLS, 0, st>>>(L.V, x, r, p, s, t, rh, scal, partials);
}

void launch_vec_xr(Lat L, double2 *x, double2 *r, const double2 *p, const double2 *v, const double2 *t,
                   const double2 *rh, const double *scal, double *partials, cudaStream_t st) {
  unsigned nb_ = (unsigned)((L.V + CN_SITES_PER_BLOCK - 1) / CN_SITES_PER_BLOCK);
  k_vec_xr<<<nb_, 32 * CN_COLS, 0, st>>>(L.V, x, r, p, v, t, rh, scal, partials);
}
void launch_vec_p(Lat L, double2 *p, const double2 *r, const double2 *v, const double *scal, cudaStream_t st) {
  unsigned nb_ = (unsigned)((L.V + CN_SITES_PER_BLOCK - 1) / CN_SITES_PER_BLOCK);
  k_vec_p<<<nb_, 32 * CN_COLS, 0, st>>>(L.V, p, r, v, scal);
}

// ------------------------------------------------------------ scalar stages
__device__ __forceinline__ cplx cdiv_safe(cplx a, cplx b) { return cdiv(a, b); }

__global__ void k_cn_finalize(int stage, int64_t nblocks, const double *__restrict__ partials,
                              double *__restrict__ scal, double tol) {
  const int col = blockIdx.x;
  const int nq = (stage == 4 || stage == 6) ? 1 : stage == 5 ? 5 : stage == 7 ? 4 : (stage == 0 || stage == 1) ? 2 : 3;
  __shared__ double sh[5][256];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int k = 0; k < nq; ++k) acc[k] += partials[(b * CN_COLS + col) * nq + k];
  for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int wd = blockDim.x / 2; wd > 0; wd >>= 1) {
    if (threadIdx.x < wd)
      for (int k = 0; k < 5; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + wd];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double *sc = scal + col * SC_STRIDE;
  const double q0 = sh[0][0], q1 = sh[1][0], q2 = sh[2][0];
  const bool conv = sc[SC_CONV] != 0.0;
  if (stage == 0 || stage == 7) {  // rr, bb after a (re)start; rho = rh.r (7: FP32 shadow rh)
    sc[SC_RR] = q0;
    sc[SC_BB] = q1;
    sc[SC_RHO] = stage == 7 ? q2 : q0;
    sc[SC_RHO + 1] = stage == 7 ? sh[3][0] : 0.0;
    sc[SC_CONV] = (q0 <= tol * tol * q1 || q1 == 0.0) ? 1.0 : 0.0;
    sc[SC_BREAK] = 0.0;
    sc[SC_NONFIN] = (isfinite(q0) && isfinite(q1)) ? 0.0 : 1.0;
    sc[SC_ALPHA] = sc[SC_ALPHA + 1] = sc[SC_OMEGA] = sc[SC_OMEGA + 1] = sc[SC_BETA] = sc[SC_BETA + 1] = 0.0;
  } else if (stage == 1) {  // alpha = rho / (rh . v)
    cplx den = {q0, q1};
    cplx rho = {sc[SC_RHO], sc[SC_RHO + 1]};
    cplx al = {0.0, 0.0};
    if (!conv) {
      if (den.re == 0.0 && den.im == 0.0) sc[SC_BREAK] = 1.0;
      else al = cdiv(rho, den);
    }
    sc[SC_ALPHA] = al.re;
    sc[SC_ALPHA + 1] = al.im;
  } else if (stage == 2) {  // omega = (t.s)/(t.t)
    cplx om = {0.0, 0.0};
    if (!conv && q2 > 0.0) om = (1.0 / q2) * cplx{q0, q1};
    sc[SC_OMEGA] = om.re;
    sc[SC_OMEGA + 1] = om.im;
  } else if (stage == 5) {  // omega = (t.s)/(t.t) and beta, ahead of the merged update
    // rh.s = rh.r - alpha rh.v = 0 by the choice of alpha, so
    // rho_new = rh.(s - omega t) = -omega rh.t, and beta =
    // (rho_new / rho)(alpha / omega) = -alpha (rh.t) / rho
    if (!conv) {
      cplx om = {0.0, 0.0};
      if (q2 > 0.0) om = (1.0 / q2) * cplx{q0, q1};
      const cplx rht = {sh[3][0], sh[4][0]};
      const cplx rho = {sc[SC_RHO], sc[SC_RHO + 1]};
      const cplx al = {sc[SC_ALPHA], sc[SC_ALPHA + 1]};
      cplx be = {0.0, 0.0}, rhon = {0.0, 0.0};
      if ((om.re == 0.0 && om.im == 0.0) || (rho.re == 0.0 && rho.im == 0.0)) {
        sc[SC_BREAK] = 1.0;
      } else {
        rhon = -(om * rht);
        be = -cdiv(al * rht, rho);
      }
      if (!isfinite(rht.re) || !isfinite(rht.im)) sc[SC_NONFIN] = 1.0;
      sc[SC_OMEGA] = om.re;
      sc[SC_OMEGA + 1] = om.im;
      sc[SC_BETA] = be.re;
      sc[SC_BETA + 1] = be.im;
      sc[SC_RHO] = rhon.re;
      sc[SC_RHO + 1] = rhon.im;
    } else {
      sc[SC_OMEGA] = sc[SC_OMEGA + 1] = sc[SC_BETA] = sc[SC_BETA + 1] = 0.0;
    }
  } else if (stage == 6) {  // rr = r.r after the merged update
    if (!conv) {
      sc[SC_RR] = q0;
      if (!isfinite(q0)) sc[SC_NONFIN] = 1.0;
      if (q0 <= tol * tol * sc[SC_BB]) sc[SC_CONV] = 1.0;
    }
  } else if (stage == 4) {  // half step: |s|^2 against the tolerance
    sc[SC_SS] = q0;
    sc[SC_HALF] = (!conv && q0 <= tol * tol * sc[SC_BB]) ? 1.0 : 0.0;
    if (!isfinite(q0)) sc[SC_NONFIN] = 1.0;
  } else {  // stage 3: rho_new = rh.r, rr = r.r
    if (!conv) {
      sc[SC_RR] = q2;
      if (!isfinite(q2)) sc[SC_NONFIN] = 1.0;
      bool cv = q2 <= tol * tol * sc[SC_BB];
      cplx rho = {sc[SC_RHO], sc[SC_RHO + 1]};
      cplx rhon = {q0, q1};
      cplx al = {sc[SC_ALPHA], sc[SC_ALPHA + 1]}, om = {sc[SC_OMEGA], sc[SC_OMEGA + 1]};
      cplx be = {0.0, 0.0};
      if (cv) {
        sc[SC_CONV] = 1.0;
      } else if ((om.re == 0.0 && om.im == 0.0) || (rho.re == 0.0 && rho.im == 0.0)) {
        sc[SC_BREAK] = 1.0;
      } else {
        be = cdiv(rhon, rho) * cdiv(al, om);
      }
      sc[SC_BETA] = be.re;
      sc[SC_BETA + 1] = be.im;
      sc[SC_RHO] = rhon.re;
      sc[SC_RHO + 1] = rhon.im;
    } else {
      sc[SC_BETA] = sc[SC_BETA + 1] = 0.0;
    }
  }
}

void launch_cn_finalize(int stage, int64_t nblocks, const double *partials, double *scal, double tol,
                        cudaStream_t st) {
  k_cn_finalize<<<CN_COLS, 256, 0, st>>>(stage, nblocks, partials, scal, tol);
}

// ------------------------------------------------------------ batched scalars
// Chebyshev coefficients of every field of a batch from the spectral
// enclosure of its mass (the device-side counterpart of the host recurrence
// of the single-field precision form): theta = 1 + i tau (lo+hi)/2,
// delta = i |tau| (hi-lo)/2, sigma = theta/delta, rho_0 = 1/sigma,
// rho_{k+1} = 1/(2 sigma - rho_k), c1 = rho_{k+1} rho_k, c2 = 2 rho_{k+1}/delta.
__global__ void k_batch_coef(BatchField *__restrict__ tab, int nfields, int *__restrict__ flags) {
  const int fi = blockIdx.x * blockDim.x + threadIdx.x;
  if (fi >= nfields) return;
  BatchField &f = tab[fi];
  int bad = 0;
  for (int sp = 0; sp < 2; ++sp) {
    double lo = f.bounds[2 * sp], hi = f.bounds[2 * sp + 1];
    if (!(isfinite(lo) && isfinite(hi) && hi >= lo)) {
      bad = 1;
      lo = hi = 0.0;
    }
    const cplx one = {1.0, 0.0};
    const cplx theta = {1.0, f.tau * 0.5 * (lo + hi)};
    const cplx delta = {0.0, fmax(fabs(f.tau) * 0.5 * (hi - lo), 1e-14)};
    const cplx sigma = cdiv(theta, delta);
    f.inv_theta[sp] = cdiv(one, theta);
    cplx rho = cdiv(one, sigma);
    // rho_k = T_k(sigma) / T_{k+1}(sigma), so m steps gain 1/|rho_0 ... rho_{m-1}|
    cplx prod = one;
    f.gain[sp][0] = 1.0;
    for (int k = 0; k < BATCH_MAX_CHEB; ++k) {
      prod = prod * rho;
      f.gain[sp][k + 1] = 1.0 / sqrt(norm2(prod));
      const cplx rn = cdiv(one, 2.0 * sigma - rho);
      f.cheb[k].c1[sp] = rn * rho;
      f.cheb[k].c2[sp] = cdiv(2.0 * rn, delta);
      rho = rn;
    }
  }
  flags[fi] = bad;
}
void launch_batch_coef(BatchField *tab, int nfields, int *flags, cudaStream_t st) {
  k_batch_coef<<<(unsigned)((nfields + 63) / 64), 64, 0, st>>>(tab, nfields, flags);
}

// (r.r, b.b) of every column of every field from the residual stencil's
// partial rows; sets the convergence and non-finite flags of each column.
__global__ void k_batch_finalize(const BatchField *__restrict__ tab, int64_t nrows, double tol, int skip_done) {
  const int col = blockIdx.x;
  const BatchField &f = tab[blockIdx.y];
  // a field the residual launch skipped keeps its scalars (another column's
  // block may mark its column converged meanwhile: then this column had
  // converged before, and keeps its scalars too)
  if (skip_done && batch_field_done(f)) return;
  __shared__ double sh[2][256];
  double acc[2] = {0.0, 0.0};
  for (int64_t b = threadIdx.x; b < nrows; b += blockDim.x)
    for (int k = 0; k < 2; ++k) acc[k] += f.partials[(b * CN_COLS + col) * 2 + k];
  for (int k = 0; k < 2; ++k) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int wd = blockDim.x / 2; wd > 0; wd >>= 1) {
    if (threadIdx.x < wd)
      for (int k = 0; k < 2; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + wd];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double *sc = f.scal + col * SC_STRIDE;
  const double q0 = sh[0][0], q1 = sh[1][0];
  sc[SC_RR] = q0;
  sc[SC_BB] = q1;
  sc[SC_CONV] = (q0 <= tol * tol * q1 || q1 == 0.0) ? 1.0 : 0.0;
  sc[SC_NONFIN] = (isfinite(q0) && isfinite(q1)) ? 0.0 : 1.0;
}
void launch_batch_finalize(const BatchField *tab, int nfields, int64_t nrows, double tol, int skip_done,
                           cudaStream_t st) {
  k_batch_finalize<<<dim3(CN_COLS, (unsigned)nfields), 256, 0, st>>>(tab, nrows, tol, skip_done);
}

__global__ void k_batch_predict(const BatchField *__restrict__ tab, int nfields, int m, double tol,
                                const double *__restrict__ pstate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nfields * CN_COLS) return;
  const BatchField &f = tab[i / CN_COLS];
  const int col = i % CN_COLS;
  double *sc = f.scal + col * SC_STRIDE;
  sc[SC_HALF] = 0.0;
  if (sc[SC_CONV] != 0.0 || !(sc[SC_BB] > 0.0)) return;
  const double ratio = pstate[0];
  const bool on = ratio >= 0.0 && fmod(pstate[1], 16.0) != 0.0;
  const double pred = sqrt(sc[SC_RR] / sc[SC_BB]) / f.gain[col / 6][m];
  const double scale = fmax(1.0, ratio);
  sc[SC_SS] = pred;
  if (on && 2.0 * scale * pred <= tol) {
    sc[SC_CONV] = 1.0;
    sc[SC_HALF] = 1.0;
    sc[SC_RR] = (scale * pred) * (scale * pred) * sc[SC_BB];
  } else {
    sc[SC_HALF] = 2.0;
  }
}
void launch_batch_predict(const BatchField *tab, int nfields, int m, double tol, const double *pstate,
                          cudaStream_t st) {
  const int n = nfields * CN_COLS;
  m = m < 0 ? 0 : (m > BATCH_MAX_CHEB ? BATCH_MAX_CHEB : m);
  k_batch_predict<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(tab, nfields, m, tol, pstate);
}

// one block: the largest true-to-predicted ratio of the columns the
// residual check measured (SC_HALF = 2) into pstate[0]; pstate[1] += 1
__global__ void k_batch_calibrate(const BatchField *__restrict__ tab, int nfields, double *__restrict__ pstate) {
  __shared__ double sh[256];
  double mx = -1.0;
  for (int i = threadIdx.x; i < nfields * CN_COLS; i += blockDim.x) {
    double *sc = tab[i / CN_COLS].scal + (i % CN_COLS) * SC_STRIDE;
    if (sc[SC_HALF] == 2.0 && sc[SC_BB] > 0.0 && sc[SC_SS] > 0.0)
      mx = fmax(mx, sqrt(sc[SC_RR] / sc[SC_BB]) / sc[SC_SS]);
    sc[SC_HALF] = 0.0;
  }
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (sh[0] >= 0.0) pstate[0] = fmax(pstate[0], sh[0]);
    pstate[1] += 1.0;
  }
}
void launch_batch_calibrate(const BatchField *tab, int nfields, double *pstate, cudaStream_t st) {
  k_batch_calibrate<<<1, 256, 0, st>>>(tab, nfields, pstate);
}

__global__ void k_batch_hist_start(int64_t n, const BatchField *__restrict__ tab) {
  const BatchField &f = tab[blockIdx.y];
  const float2 *h[4] = {f.h1, f.h2, f.h3, f.h4};
  int d = 0;
  while (d < 4 && h[d]) ++d;
  const double cf[5][4] = {{0, 0, 0, 0}, {1, 0, 0, 0}, {2, -1, 0, 0}, {3, -3, 1, 0}, {4, -6, 4, -1}};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double dx = 0.0, dy = 0.0;
    for (int k = 0; k < d; ++k) {  // read before hnew (which may be the oldest slot) is written
      const float2 a = h[k][i];
      dx += cf[d][k] * (double)a.x;
      dy += cf[d][k] * (double)a.y;
    }
    const double2 x = f.x[i];
    f.x[i] = make_double2(x.x + dx, x.y + dy);
    f.hnew[i] = make_float2((float)dx, (float)dy);
  }
}
void launch_batch_hist_start(int64_t V, const BatchField *tab, int nfields, cudaStream_t st) {
  const int64_t n = 72 * V;
  k_batch_hist_start<<<dim3((unsigned)std::min<int64_t>((n + 255) / 256, 2048), (unsigned)nfields), 256, 0, st>>>(
      n, tab);
}

// ------------------------------------------------------------ propagator I/O, norms, correlators
// Fortran prop(6,6,V): (site*6 + col)*6 + row ; f holds quark then antiquark (2*V*36)
__global__ void k_prop_f2soa(const double2 *__restrict__ f, double2 *__restrict__ P, int64_t V) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  for (int sp = 0; sp < 2; ++sp)
#pragma unroll
    for (int k = 0; k < 36; ++k) P[(int64_t)(sp * 36 + k) * V + s] = f[(int64_t)sp * 36 * V + s * 36 + k];
}
__global__ void k_prop_soa2f(const double2 *__restrict__ P, double2 *__restrict__ f, int64_t V) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  for (int sp = 0; sp < 2; ++sp)
#pragma unroll
    for (int k = 0; k < 36; ++k) f[(int64_t)sp * 36 * V + s * 36 + k] = P[(int64_t)(sp * 36 + k) * V + s];
}
void launch_prop_f2soa(const double2 *f, double2 *P, int64_t V, cudaStream_t st) {
  k_prop_f2soa<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(f, P, V);
}
void launch_prop_soa2f(const double2 *P, double2 *f, int64_t V, cudaStream_t st) {
  k_prop_soa2f<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(P, f, V);
}

__global__ void k_single_point(double2 *__restrict__ P, int64_t V, int64_t sq, int64_t sa) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  const double v = 1.0 / sqrt(6.0);
  for (int sp = 0; sp < 2; ++sp) {
    const int64_t src = sp == 0 ? sq : sa;
#pragma unroll
    for (int k = 0; k < 36; ++k) {
      const int col = k / 6, row = k % 6;
      P[(int64_t)(sp * 36 + k) * V + s] = make_double2((s == src && col == row) ? v : 0.0, 0.0);
    }
  }
}
void launch_single_point(double2 *P, int64_t V, int64_t sq, int64_t sa, cudaStream_t st) {
  k_single_point<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(P, V, sq, sa);
}

__global__ void __launch_bounds__(256) k_norms(const double2 *__restrict__ P, int64_t V, double *partials) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (s < V)
    for (int sp = 0; sp < 2; ++sp)
      for (int k = 0; k < 36; ++k) v[sp] += norm2(ldg(P + (int64_t)(sp * 36 + k) * V + s));
  __shared__ double sh[8][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 2; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0) {
    sh[warp][0] = v[0];
    sh[warp][1] = v[1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += sh[k][0];
      b += sh[k][1];
    }
    partials[blockIdx.x * 2] = a;
    partials[blockIdx.x * 2 + 1] = b;
  }
}
void launch_norms(const double2 *P, int64_t V, double *partials, int64_t &nblk, cudaStream_t st) {
  nblk = (V + 255) / 256;
  k_norms<<<(unsigned)nblk, 256, 0, st>>>(P, V, partials);
}

// Sparse Gamma tables for the zero-momentum meson correlators
// (src/nrqcd.f90:1484-1661): entries (row, col, re, im) of Gamma = T^a x s_k,
// 1 x s_k or T^a x 1 (index 2*colour + spin), with the reference's matrices.
struct GamEntry {
  double re, im;
  int r, c;
};
struct GamTable {
  int ngam[3];       // O1_3S1, O8_1S0, O8_3S1
  int start[3][24];  // entry offset per Gamma
  int count[3][24];
  GamEntry e[3 * 24 * 8];
};
__constant__ GamTable c_gam;

// GCONJ: the _gconjg variants (src/nrqcd.f90:1728-1905), conj(A) in place of
// A^+, i.e. A's indices swapped in every product below
template <bool GCONJ>
__global__ void __launch_bounds__(128) k_correlators(const double2 *__restrict__ P, int64_t V, double *partials) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (s < V) {
    // Q[r][c] = quark (row r, col c), A likewise
    auto q = [&](int r, int c) { return ldg(P + (int64_t)(c * 6 + r) * V + s); };
    auto a = [&](int r, int c) {
      return GCONJ ? ldg(P + (int64_t)(36 + r * 6 + c) * V + s) : ldg(P + (int64_t)(36 + c * 6 + r) * V + s);
    };
    // O1_1S0 = i Tr(A^+ Q) = i sum_{rc} conj(A[r][c]) Q[r][c]
    cplx t = {0.0, 0.0};
    for (int r = 0; r < 6; ++r)
      for (int c = 0; c < 6; ++c) cmac_cj(t, a(r, c), q(r, c));
    cplx o = times_i(t);
    v[0] = o.re;
    v[1] = o.im;
    const double wts[3] = {1.0 / 3.0, 6.0 / 8.0, 6.0 / 24.0};
    for (int kind = 0; kind < 3; ++kind) {
      cplx sum = {0.0, 0.0};
      for (int g = 0; g < c_gam.ngam[kind]; ++g) {
        const int st0 = c_gam.start[kind][g], n = c_gam.count[kind][g];
        // Tr(A^+ G Q G) = sum conj(A[d1][d0]) G[d1][d2] Q[d2][d3] G[d3][d0]
        for (int e1 = 0; e1 < n; ++e1) {
          const GamEntry ga = c_gam.e[st0 + e1];  // (d1, d2)
          for (int e2 = 0; e2 < n; ++e2) {
            const GamEntry gb = c_gam.e[st0 + e2];  // (d3, d0)
            cplx gg = cplx{ga.re, ga.im} * cplx{gb.re, gb.im};
            cplx qa = q(ga.c, gb.r);
            cplx term = {0.0, 0.0};
            cmac_cj(term, a(ga.r, gb.c), qa);
            cmac(sum, gg, term);
          }
        }
      }
      cplx ov = times_i(sum) * wts[kind];
      v[2 + 2 * kind] = ov.re;
      v[3 + 2 * kind] = ov.im;
    }
  }
  __shared__ double sh[4][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 8; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
    for (int k = 0; k < 8; ++k) sh[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < 8) {
    double acc = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) acc += sh[k][threadIdx.x];
    partials[blockIdx.x * 8 + threadIdx.x] = acc;
  }
}

static void build_gamma_table(GamTable &T) {
  // reference generators (row-major) and Pauli matrices (su2.f90 arrays)
  double Tre[8][9] = {{0}}, Tim[8][9] = {{0}};
  const double h = 0.5, s8 = 0.5 / 1.7320508075688772, d8 = 1.0 / 1.7320508075688772;
  Tre[0][1] = Tre[0][3] = h;
  Tim[1][1] = h; Tim[1][3] = -h;
  Tre[2][0] = h; Tre[2][4] = -h;
  Tre[3][2] = Tre[3][6] = h;
  Tim[4][2] = h; Tim[4][6] = -h;
  Tre[5][5] = Tre[5][7] = h;
  Tim[6][5] = h; Tim[6][7] = -h;
  Tre[7][0] = s8; Tre[7][4] = s8; Tre[7][8] = -d8;
  double Sre[3][4] = {{0, 1, 1, 0}, {0, 0, 0, 0}, {1, 0, 0, -1}};
  double Sim[3][4] = {{0, 0, 0, 0}, {0, 1, -1, 0}, {0, 0, 0, 0}};
  int ne = 0;
  auto add_gamma = [&](int kind, int g, const double *Are, const double *Aim, const double *Bre,
                       const double *Bim) {
    T.start[kind][g] = ne;
    int cnt = 0;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        for (int s = 0; s < 2; ++s)
          for (int t = 0; t < 2; ++t) {
            double ar = Are[r * 3 + c], ai = Aim[r * 3 + c], br = Bre[s * 2 + t], bi = Bim[s * 2 + t];
            double vr = ar * br - ai * bi, vi = ar * bi + ai * br;
            if (vr != 0.0 || vi != 0.0) {
              T.e[ne++] = GamEntry{vr, vi, 2 * r + s, 2 * c + t};
              ++cnt;
            }
          }
    T.count[kind][g] = cnt;
  };
  double I3re[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, I3im[9] = {0};
  double I2re[4] = {1, 0, 0, 1}, I2im[4] = {0};
  T.ngam[0] = 3;
  for (int k = 0; k < 3; ++k) add_gamma(0, k, I3re, I3im, Sre[k], Sim[k]);
  T.ngam[1] = 8;
  for (int a = 0; a < 8; ++a) add_gamma(1, a, Tre[a], Tim[a], I2re, I2im);
  T.ngam[2] = 24;
  int g = 0;
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 8; ++a) add_gamma(2, g++, Tre[a], Tim[a], Sre[k], Sim[k]);
}

void launch_correlators(const double2 *P, int64_t V, double *partials, int64_t &nblk, cudaStream_t st,
                        bool gconjg) {
  static GamTable T;
  static bool built = false;
  if (!built) {
    build_gamma_table(T);
    built = true;
  }
  cudaMemcpyToSymbolAsync(c_gam, &T, sizeof(T), 0, cudaMemcpyHostToDevice, st);
  nblk = (V + 127) / 128;
  if (gconjg) k_correlators<true><<<(unsigned)nblk, 128, 0, st>>>(P, V, partials);
  else k_correlators<false><<<(unsigned)nblk, 128, 0, st>>>(P, V, partials);
}

// ------------------------------------------------------------ history-extrapolated start
// The plain solve's start 2b - psi misses t = x - (2b - psi); consecutive
// steps' t vary smoothly, so the start adds t extrapolated from the last d
// steps by the polynomial of degree d - 1 through them: x0 = 2b - psi +
// sum_k c_k t_k, c = (1), (2, -1), (3, -3, 1), (4, -6, 4, -1) (t_1 the
// newest).  The history is kept in FP32.
struct HistExtrap {
  const float2 *t[4];
  double c[4];
};
__global__ void k_hist_extrapolate(int64_t n, double2 *__restrict__ X, const HistExtrap H) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dx = 0.0, dy = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (H.t[k]) {
      const float2 a = H.t[k][i];
      dx += H.c[k] * (double)a.x;
      dy += H.c[k] * (double)a.y;
    }
  const double2 x = X[i];
  X[i] = make_double2(x.x + dx, x.y + dy);
}
// t = x - (2b - psi) of the step just solved
__global__ void k_hist_store(int64_t n, const double2 *__restrict__ X, const double2 *__restrict__ B,
                             const double2 *__restrict__ Psi, float2 *__restrict__ T) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 x = X[i], b = B[i], p = Psi[i];
  T[i] = make_float2((float)(x.x - (2.0 * b.x - p.x)), (float)(x.y - (2.0 * b.y - p.y)));
}
void launch_hist_extrapolate(int64_t n, double2 *X, const float2 *const *t, int d, cudaStream_t st) {
  static const double kCoef[4][4] = {{1, 0, 0, 0}, {2, -1, 0, 0}, {3, -3, 1, 0}, {4, -6, 4, -1}};
  HistExtrap H{};
  d = d < 1 ? 1 : (d > 4 ? 4 : d);
  for (int k = 0; k < 4; ++k) {
    H.t[k] = k < d ? t[k] : nullptr;
    H.c[k] = kCoef[d - 1][k];
  }
  k_hist_extrapolate<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, X, H);
}
void launch_hist_store(int64_t n, const double2 *X, const double2 *B, const double2 *Psi, float2 *T, cudaStream_t st) {
  k_hist_store<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, X, B, Psi, T);
}

}  // namespace nrq
