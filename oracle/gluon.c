/* CPU oracle (test infrastructure only) of the gluon-distribution
 * observables: Coulomb gauge fixing and the transverse AA/EE correlators.
 *
 *   CoulombGaugefixing_Links      src/gaugeconfiguration_su3.f90:2297-2456
 *   GetDivergenceOfGaugeField_M   src/gaugeconfiguration_su3.f90:2460-2478
 *   GetTransverseAA/EECorrelator  src/gaugeconfiguration_su3.f90:1825-1905
 *   GetTransverseCorrelator       src/gaugeconfiguration_su3.f90:1907-1945
 *   GetTransverseField_usingProjector  src/gaugeconfiguration_su3.f90:1953-1972
 *   GetMomentum_G (backward derivative), GetNorm2Momentum_G,
 *   FindMaxNorm2Momentum, GetTransverseProjector  src/lattice.f90:422-465,
 *                                                 963-979, 1081-1089, 1184-1198
 *   ExpAH (EigenH of -iA), ArgLogU (EigenC)  src/matrixoperations.f90:474-495, 547-567
 *   x2p / p2x scales (a1 a2 a3 forward, 1/Volume backward)  src/xpfft.f90:129-139
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_internal.h"

/* backward-derivative lattice momentum of a site and its norm */
static double momentum(const oc_lattice *L, int64_t s, cplx p[3]) {
  const double pi = acos(-1.0);
  const int64_t pos[3] = {s % L->n[0], (s / L->n[0]) % L->n[1], s / (L->n[0] * L->n[1])};
  double n2 = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double ph = pi * (double)pos[i] / (double)L->n[i];
    p[i] = 2.0 * sin(ph) / L->a[i + 1] * (cos(ph) - I * sin(ph));
    n2 += creal(p[i] * conj(p[i]));
  }
  return sqrt(n2);
}

double oc_norm2_momentum(const oc_lattice *L, int64_t s) {
  cplx p[3];
  return momentum(L, s, p);
}

/* D(x) = sum_i AH(U_i(x - i) - U_i(x)), AH(M) = (M - M^+)/2 */
static void divergence(const oc_lattice *L, const double *links, int64_t s, cplx D[9]) {
  for (int k = 0; k < 9; ++k) D[k] = 0;
  for (int i = 1; i <= 3; ++i) {
    cplx U[9], Um[9], d[9];
    oc_load_link(links, s, i, U);
    oc_load_link(links, oc_neib(L, s, i, -1), i, Um);
    for (int k = 0; k < 9; ++k) d[k] = -U[k] + Um[k];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) D[r * 3 + c] += (d[r * 3 + c] - conj(d[c * 3 + r])) / 2.0;
  }
}

/* Coulomb gauge fixing of the links (the electric field is not transformed,
 * as in the reference).  Returns the reference's loop counter after the loop
 * (the iteration at which the divergence met the tolerance, or
 * max_iterations + 1); deviations[k] (may be NULL) gets the maximum
 * Frobenius norm / 9 of the divergence checked at iteration k + 1. */
int64_t oc_gauge_coulomb_gaugefix(const oc_lattice *L, double *links, double tol, double alpha,
                                  int64_t max_iterations, double *deviations) {
  const int64_t V = oc_volume(L);
  cplx *D = (cplx *)malloc(sizeof(cplx) * (size_t)V * 9); /* [r*3+c][site] */
  cplx *G = (cplx *)malloc(sizeof(cplx) * (size_t)V * 9); /* [site][r*3+c] */
  double pmax = 0.0;
  for (int64_t s = 0; s < V; ++s) {
    const double pn = oc_norm2_momentum(L, s);
    if (pn > pmax) pmax = pn;
  }
  const double fwd = L->a[1] * L->a[2] * L->a[3];
  const double bwd = 1.0 / ((double)V * fwd);
  int64_t it;
  for (it = 1; it <= max_iterations; ++it) {
    double mx = -1.0;
    for (int64_t s = 0; s < V; ++s) {
      cplx d[9];
      divergence(L, links, s, d);
      double f = 0.0;
      for (int k = 0; k < 9; ++k) {
        D[(int64_t)k * V + s] = d[k];
        f += creal(d[k] * conj(d[k]));
      }
      f = sqrt(f) / 9.0;
      if (f > mx) mx = f;
    }
    if (deviations) deviations[it - 1] = mx;
    if (!(mx > tol)) break;
    for (int k = 0; k < 9; ++k) oc_fft3d((double *)(D + (int64_t)k * V), L->n, -1, fwd);
    for (int64_t s = 0; s < V; ++s) {
      const double pn = oc_norm2_momentum(L, s);
      if (pn > 1e-12) {
        const double f = (pmax / pn) * (pmax / pn);
        for (int k = 0; k < 9; ++k) D[(int64_t)k * V + s] *= f;
      }
    }
    for (int k = 0; k < 9; ++k) oc_fft3d((double *)(D + (int64_t)k * V), L->n, +1, bwd);
    for (int64_t s = 0; s < V; ++s) {
      /* ExpAH(alpha D) = exp(i H), H = -i alpha D */
      cplx H[9];
      for (int k = 0; k < 9; ++k) H[k] = -I * (alpha * D[(int64_t)k * V + s]);
      expi_hermitian(H, G + s * 9);
    }
    for (int64_t s = 0; s < V; ++s)
      for (int i = 1; i <= 3; ++i) {
        cplx U[9], T[9], Gd[9];
        oc_load_link(links, s, i, U);
        m3_dag(G + oc_neib(L, s, i, +1) * 9, Gd);
        m3_mul(G + s * 9, U, T);
        m3_mul(T, Gd, T);
        oc_store_link(links, s, i, T);
      }
  }
  free(D);
  free(G);
  return it;
}

/* aa[s], ee[s]: the transverse AA and EE correlators at momentum site s
 * (averaged over the eight generators), momenta[s] = |p(s)| (any output
 * may be NULL) */
void oc_gauge_transverse_correlators(const oc_lattice *L, const double *links, const double *efield, double *aa,
                                     double *ee, double *momenta) {
  const int64_t V = oc_volume(L);
  const double fwd = L->a[1] * L->a[2] * L->a[3];
  const double volume = (double)V * fwd;
  cplx *F = (cplx *)malloc(sizeof(cplx) * (size_t)V * 48); /* [(field*3 + i)*8 + a][site] */
  for (int64_t s = 0; s < V; ++s)
    for (int i = 1; i <= 3; ++i) {
      cplx U[9], Lg[9];
      oc_load_link(links, s, i, U);
      oc_logu3((const double *)U, (double *)Lg); /* i ArgLogU */
      const double *e = oc_efield_at(efield, s, i);
      for (int a = 1; a <= 8; ++a) {
        cplx H[9];
        for (int k = 0; k < 9; ++k) H[k] = -I * Lg[k]; /* ArgLogU */
        const double A = 2.0 * creal(trace_with_generator(a, H)) / L->a[i];
        const double E = e[a - 1] / L->a[i] / L->a[0];
        F[((int64_t)(0 * 3 + (i - 1)) * 8 + (a - 1)) * V + s] = A;
        F[((int64_t)(1 * 3 + (i - 1)) * 8 + (a - 1)) * V + s] = E;
      }
    }
  for (int k = 0; k < 48; ++k) oc_fft3d((double *)(F + (int64_t)k * V), L->n, -1, fwd);
  for (int64_t s = 0; s < V; ++s) {
    cplx p[3];
    const double pn = momentum(L, s, p);
    if (momenta) momenta[s] = pn;
    /* GetTransverseProjector is declared real: the real part of
       (delta_ij - conj(p_i) p_j / |p|^2) / 2 */
    double P[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        cplx v = 0;
        if (!(pn < 1e-12)) v = ((i == j ? 1.0 : 0.0) - conj(p[i]) * p[j] / (pn * pn)) / 2.0;
        P[i][j] = creal(v);
      }
    for (int field = 0; field < 2; ++field) {
      double acc = 0.0;
      for (int a = 0; a < 8; ++a) {
        cplx f[3], res = 0;
        for (int i = 0; i < 3; ++i) f[i] = F[((int64_t)(field * 3 + i) * 8 + a) * V + s];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) res += f[i] * P[i][j] * conj(f[j]);
        acc += (creal(res) / volume) / 8.0;
      }
      double *out = field == 0 ? aa : ee;
      if (out) out[s] = acc;
    }
  }
  free(F);
}
