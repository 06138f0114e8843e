// Complex Jacobi eigen-decomposition of a general 3x3 matrix on the device,
// shared by the CN preparation (field strength via LogU) and the gluon
// observables (ArgLogU of the links).
#pragma once
#include "nrq_common.cuh"

namespace nrq {

// ------------------------------------------------------------ Jacobi log
// Complex Jacobi eigen-decomposition of a general 3x3 matrix, the algorithm
// of src/matrixoperations.f90:327-459 (d = U A U^+, rows of U normalised).
__device__ inline void eigenc3(const m3 &Ain, cplx d[3], m3 &U) {
  const double EPS = 9.860761315262648e-32;  // 2^-103
  m3 A = Ain;
  cplx ev0[3], ev1[3];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    ev0[p] = {0.0, 0.0};
    ev1[p] = A.e[p * 4];
    d[p] = ev1[p];
  }
  U = m3_id();
  const double red = 0.01 / 81.0;
  for (int sweep = 1; sweep <= 50; ++sweep) {
    double off = 0.0;
    for (int q = 1; q < 3; ++q)
      for (int p = 0; p < q; ++p) {
        double a1 = cabs_(A.e[p * 3 + q]), a2 = cabs_(A.e[q * 3 + p]);
        off = off + a1 * a1 + a2 * a2;
      }
    if (off <= EPS) break;
    double thresh = (sweep < 4) ? off * red : 0.0;
    for (int q = 1; q < 3; ++q) {
      for (int p = 0; p < q; ++p) {
        double a1 = cabs_(A.e[p * 3 + q]), a2 = cabs_(A.e[q * 3 + p]);
        off = a1 * a1 + a2 * a2;
        double e1 = cabs_(ev1[p]), e2 = cabs_(ev1[q]);
        if (sweep > 4 && off < EPS * (e1 * e1 + e2 * e2)) {
          A.e[p * 3 + q] = {0.0, 0.0};
          A.e[q * 3 + p] = {0.0, 0.0};
        } else if (off > thresh) {
          cplx delta = A.e[p * 3 + q] * A.e[q * 3 + p];
          cplx x = 0.5 * (ev1[p] - ev1[q]);
          cplx y = csqrt_(x * x + delta);
          cplx t = x - y;
          cplx s = x + y;
          if (cabs_(t) < cabs_(s)) t = s;
          t = cdiv({1.0, 0.0}, t);
          delta = delta * t;
          ev0[p] = ev0[p] + delta;
          ev1[p] = d[p] + ev0[p];
          ev0[q] = ev0[q] - delta;
          ev1[q] = d[q] + ev0[q];
          cplx invc = csqrt_(delta * t + cplx{1.0, 0.0});
          s = cdiv(t, invc);
          t = cdiv(t, invc + cplx{1.0, 0.0});
          cplx sx = s * A.e[p * 3 + q], ty = t * A.e[p * 3 + q];
          cplx sy = s * A.e[q * 3 + p], tx = t * A.e[q * 3 + p];
          for (int j = 0; j < 3; ++j) {
            x = A.e[j * 3 + p];
            y = A.e[j * 3 + q];
            A.e[j * 3 + p] = x + sy * (y - ty * x);
            A.e[j * 3 + q] = y - sx * (x + tx * y);
            x = A.e[p * 3 + j];
            y = A.e[q * 3 + j];
            A.e[p * 3 + j] = x + sx * (y - tx * x);
            A.e[q * 3 + j] = y - sy * (x + ty * y);
          }
          A.e[p * 3 + q] = {0.0, 0.0};
          A.e[q * 3 + p] = {0.0, 0.0};
          for (int j = 0; j < 3; ++j) {
            x = U.e[p * 3 + j];
            y = U.e[q * 3 + j];
            U.e[p * 3 + j] = x + sx * (y - tx * x);
            U.e[q * 3 + j] = y - sy * (x + ty * y);
          }
        }
      }
    }
    for (int p = 0; p < 3; ++p) {
      ev0[p] = {0.0, 0.0};
      d[p] = ev1[p];
    }
  }
  for (int p = 0; p < 3; ++p) {
    double nrm = 0.0;
    for (int q = 0; q < 3; ++q) nrm += norm2(U.e[p * 3 + q]);
    nrm = 1.0 / sqrt(nrm);
    for (int q = 0; q < 3; ++q) U.e[p * 3 + q] = nrm * U.e[p * 3 + q];
  }
}

}  // namespace nrq
