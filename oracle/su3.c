/*
 * Oracle (test infrastructure only): SU(3) algebra, Jacobi eigensolvers,
 * matrix exponential and logarithm, as the reference computes them.
 *
 *   generators        src/su3.f90:97-131  (the arrays the reference holds:
 *                     Fortran reshape is column-major, so T2, T5, T7 are the
 *                     transposes of the textbook lambda/2 matrices)
 *   GetAlgebraMatrix  src/su3.f90:287-301
 *   GetGroupExp       src/su3.f90:235-274 -> ExpAH_diaglibrary
 *                     src/matrixoperations.f90:547-567
 *   EigenH            src/matrixoperations.f90:187-312 (cyclic complex Jacobi
 *                     for hermitian matrices, Wilkinson-Reinsch handbook p.202)
 *   EigenC            src/matrixoperations.f90:327-459 (complex Jacobi for
 *                     general matrices; eigenvector rows normalised)
 *   LogU              src/matrixoperations.f90:510-531
 * Matrices are 3x3 complex, row-major, interleaved (re,im).
 */
#include <complex.h>
#include <math.h>
#include <string.h>
#include "oracle.h"
#include "oracle_internal.h"

void oc_generator(int a, double T_[18]) {
  cplx *T = (cplx *)T_;
  for (int k = 0; k < 9; ++k) T[k] = 0;
  const double h = 0.5;
  switch (a) {
    case 1: T[0 * 3 + 1] = h; T[1 * 3 + 0] = h; break;
    case 2: T[0 * 3 + 1] = h * I; T[1 * 3 + 0] = -h * I; break;
    case 3: T[0] = h; T[4] = -h; break;
    case 4: T[0 * 3 + 2] = h; T[2 * 3 + 0] = h; break;
    case 5: T[0 * 3 + 2] = h * I; T[2 * 3 + 0] = -h * I; break;
    case 6: T[1 * 3 + 2] = h; T[2 * 3 + 1] = h; break;
    case 7: T[1 * 3 + 2] = h * I; T[2 * 3 + 1] = -h * I; break;
    case 8: {
      double s = 0.5 / sqrt(3.0);
      T[0] = s; T[4] = s; T[8] = -1.0 / sqrt(3.0);
    } break;
    default: for (int k = 0; k < 9; ++k) T[k] = -1; break;
  }
}

/* Pauli matrices as held by src/su2.f90:68-79 (sigma_2 transposed). */
void oc_pauli(int k, cplx S[4]) {
  S[0] = S[1] = S[2] = S[3] = 0;
  if (k == 1) { S[1] = 1; S[2] = 1; }
  else if (k == 2) { S[1] = I; S[2] = -I; }
  else { S[0] = 1; S[3] = -1; }
}

void m3_mul(const cplx A[9], const cplx B[9], cplx C[9]) {
  cplx R[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      cplx acc = 0;
      for (int k = 0; k < 3; ++k) acc += A[i * 3 + k] * B[k * 3 + j];
      R[i * 3 + j] = acc;
    }
  memcpy(C, R, sizeof(R));
}

void m3_dag(const cplx A[9], cplx B[9]) {
  cplx R[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i * 3 + j] = conj(A[j * 3 + i]);
  memcpy(B, R, sizeof(R));
}

cplx m3_trace(const cplx A[9]) { return A[0] + A[4] + A[8]; }

void oc_algebra_matrix(const double alpha[8], double M_[18]) {
  cplx *M = (cplx *)M_;
  cplx T[9];
  for (int k = 0; k < 9; ++k) M[k] = 0;
  for (int a = 1; a <= 8; ++a) {
    oc_generator(a, (double *)T);
    for (int k = 0; k < 9; ++k) M[k] = M[k] + alpha[a - 1] * T[k];
  }
}

cplx trace_with_generator(int a, const cplx M[9]) {
  cplx T[9], P[9];
  oc_generator(a, (double *)T);
  m3_mul(T, M, P);
  return m3_trace(P);
}

static inline double fsign(double a, double b) { return b >= 0.0 ? fabs(a) : -fabs(a); }

void oc_eigenh3(const double A_[18], double d[3], double U_[18]) {
  const int n = 3;
  const double SYM_EPS = ldexp(1.0, -103);
  cplx A[3][3], (*U)[3] = (cplx(*)[3])U_;
  memcpy(A, A_, sizeof(A));
  double ev[3][2];
  for (int p = 0; p < n; ++p) {
    ev[p][0] = 0;
    ev[p][1] = creal(A[p][p]);
    d[p] = ev[p][1];
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) U[i][j] = (i == j) ? 1.0 : 0.0;
  const double red = 0.04 / (double)(n * n * n * n);
  for (int sweep = 1; sweep <= 50; ++sweep) {
    double off = 0;
    for (int q = 1; q < n; ++q)
      for (int p = 0; p < q; ++p) off += creal(A[p][q] * conj(A[p][q]));
    if (off <= SYM_EPS) break;
    double thresh = (sweep < 4) ? off * red : 0.0;
    for (int q = 1; q < n; ++q) {
      for (int p = 0; p < q; ++p) {
        cplx Apq = A[p][q];
        off = creal(Apq * conj(Apq));
        if (sweep > 4 && off < SYM_EPS * (ev[p][1] * ev[p][1] + ev[q][1] * ev[q][1])) {
          A[p][q] = 0;
        } else if (off > thresh) {
          double t = 0.5 * (ev[p][1] - ev[q][1]);
          t = 1.0 / (t + fsign(sqrt(t * t + off), t));
          double delta = t * off;
          ev[p][0] = ev[p][0] + delta;
          ev[p][1] = d[p] + ev[p][0];
          ev[q][0] = ev[q][0] - delta;
          ev[q][1] = d[q] + ev[q][0];
          double invc = sqrt(delta * t + 1.0);
          double s = t / invc;
          t = delta / (invc + 1.0);
          for (int j = 0; j < p; ++j) {
            cplx x = A[j][p], y = A[j][q];
            A[j][p] = x + s * (conj(Apq) * y - t * x);
            A[j][q] = y - s * (Apq * x + t * y);
          }
          for (int j = p + 1; j < q; ++j) {
            cplx x = A[p][j], y = A[j][q];
            A[p][j] = x + s * (Apq * conj(y) - t * x);
            A[j][q] = y - s * (Apq * conj(x) + t * y);
          }
          for (int j = q + 1; j < n; ++j) {
            cplx x = A[p][j], y = A[q][j];
            A[p][j] = x + s * (Apq * y - t * x);
            A[q][j] = y - s * (conj(Apq) * x + t * y);
          }
          A[p][q] = 0;
          for (int j = 0; j < n; ++j) {
            cplx x = U[p][j], y = U[q][j];
            U[p][j] = x + s * (Apq * y - t * x);
            U[q][j] = y - s * (conj(Apq) * x + t * y);
          }
        }
      }
    }
    for (int p = 0; p < n; ++p) {
      ev[p][0] = 0;
      d[p] = ev[p][1];
    }
  }
}

void oc_eigenc3(const double A_[18], double d_[6], double U_[18]) {
  const int n = 3;
  const double EPS = ldexp(1.0, -103);
  cplx A[3][3], (*U)[3] = (cplx(*)[3])U_, *d = (cplx *)d_;
  memcpy(A, A_, sizeof(A));
  cplx ev[3][2];
  for (int p = 0; p < n; ++p) {
    ev[p][0] = 0;
    ev[p][1] = A[p][p];
    d[p] = ev[p][1];
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) U[i][j] = (i == j) ? 1.0 : 0.0;
  const double red = 0.01 / (double)(n * n * n * n);
  for (int sweep = 1; sweep <= 50; ++sweep) {
    double off = 0;
    for (int q = 1; q < n; ++q)
      for (int p = 0; p < q; ++p) {
        double a1 = cabs(A[p][q]), a2 = cabs(A[q][p]);
        off = off + a1 * a1 + a2 * a2;
      }
    if (off <= EPS) break;
    double thresh = (sweep < 4) ? off * red : 0.0;
    for (int q = 1; q < n; ++q) {
      for (int p = 0; p < q; ++p) {
        double a1 = cabs(A[p][q]), a2 = cabs(A[q][p]);
        off = a1 * a1 + a2 * a2;
        double e1 = cabs(ev[p][1]), e2 = cabs(ev[q][1]);
        if (sweep > 4 && off < EPS * (e1 * e1 + e2 * e2)) {
          A[p][q] = 0;
          A[q][p] = 0;
        } else if (off > thresh) {
          cplx delta = A[p][q] * A[q][p];
          cplx x = 0.5 * (ev[p][1] - ev[q][1]);
          cplx y = csqrt(x * x + delta);
          cplx t = x - y;
          cplx s = x + y;
          if (cabs(t) < cabs(s)) t = s;
          t = 1.0 / t;
          delta = delta * t;
          ev[p][0] = ev[p][0] + delta;
          ev[p][1] = d[p] + ev[p][0];
          ev[q][0] = ev[q][0] - delta;
          ev[q][1] = d[q] + ev[q][0];
          cplx invc = csqrt(delta * t + 1.0);
          s = t / invc;
          t = t / (invc + 1.0);
          cplx sx = s * A[p][q], ty = t * A[p][q];
          cplx sy = s * A[q][p], tx = t * A[q][p];
          for (int j = 0; j < n; ++j) {
            x = A[j][p];
            y = A[j][q];
            A[j][p] = x + sy * (y - ty * x);
            A[j][q] = y - sx * (x + tx * y);
            x = A[p][j];
            y = A[q][j];
            A[p][j] = x + sx * (y - tx * x);
            A[q][j] = y - sy * (x + ty * y);
          }
          A[p][q] = 0;
          A[q][p] = 0;
          for (int j = 0; j < n; ++j) {
            x = U[p][j];
            y = U[q][j];
            U[p][j] = x + sx * (y - tx * x);
            U[q][j] = y - sy * (x + ty * y);
          }
        }
      }
    }
    for (int p = 0; p < n; ++p) {
      ev[p][0] = 0;
      d[p] = ev[p][1];
    }
  }
  for (int p = 0; p < n; ++p) {
    double norm = 0;
    for (int q = 0; q < n; ++q) {
      double a = cabs(U[p][q]);
      norm = norm + a * a;
    }
    norm = 1.0 / sqrt(norm);
    for (int q = 0; q < n; ++q) U[p][q] = U[p][q] * norm;
  }
}

/* exp(i A) for hermitian A via EigenH: A = S^+ diag(ev) S */
void expi_hermitian(const cplx A[9], cplx G[9]) {
  double ev[3];
  cplx S[9], Sd[9], D[9];
  oc_eigenh3((const double *)A, ev, (double *)S);
  for (int k = 0; k < 9; ++k) D[k] = 0;
  for (int i = 0; i < 3; ++i) D[i * 4] = cos(ev[i]) + I * sin(ev[i]);
  m3_dag(S, Sd);
  m3_mul(Sd, D, G);
  m3_mul(G, S, G);
}

void oc_group_exp(const double alpha[8], double G_[18]) {
  cplx M[9];
  oc_algebra_matrix(alpha, (double *)M);
  expi_hermitian(M, (cplx *)G_);
}

void oc_logu3(const double P_[18], double L_[18]) {
  cplx ev[3], S[9], Sd[9], D[9];
  cplx *L = (cplx *)L_;
  oc_eigenc3(P_, (double *)ev, (double *)S);
  for (int k = 0; k < 9; ++k) D[k] = 0;
  for (int i = 0; i < 3; ++i) D[i * 4] = I * atan2(cimag(ev[i]), creal(ev[i]));
  m3_dag(S, Sd);
  m3_mul(Sd, D, L);
  m3_mul(L, S, L);
}
