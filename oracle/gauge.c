/*
 * Oracle (test infrastructure only): gauge-field part of the hot path.
 *
 *   ColdInit                           src/gaugeconfiguration_su3.f90:363-378
 *   TransversePolarisedOccupiedInit_Box  :906-951 -> ...Init :1263-1446,
 *                                      GetBoxOccupation :1455-1471,
 *                                      momenta src/lattice.f90:963-979,
 *                                      polarisations src/lattice.f90:1120-1176
 *   Update_Leapfrog                    :2082-2111
 *   Update_Links_Leapfrog              :2118-2140
 *   Update_Efield_Leapfrog + staples   :2147-2259
 *   GetEnergy                          :1769-1817 (plaquette :1591-1615)
 *   GetDeviationFromGaussLaw           :1480-1531
 *   GetGdeviation / GetG               :724-813
 *   Gauss projection loop              :494-540
 *   GetFieldStrengthTensor_M           :1563-1581 (temporal plaquette :1656-1679)
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_internal.h"

void oc_gauge_cold(const oc_lattice *L, double *links, double *efield) {
  int64_t V = oc_volume(L);
  memset(efield, 0, sizeof(double) * (size_t)V * 24);
  cplx Id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int64_t s = 0; s < V; ++s)
    for (int d = 1; d <= 3; ++d) oc_store_link(links, s, d, Id);
}

/* ---------------- initial condition ---------------- */

static void momentum_backward(const oc_lattice *L, int64_t site, cplx p[3]) {
  const double pi = acos(-1.0);
  int64_t pos[3] = {site % L->n[0], (site / L->n[0]) % L->n[1], site / (L->n[0] * L->n[1])};
  for (int i = 0; i < 3; ++i) {
    double ang = pi * (double)pos[i] / (double)L->n[i];
    double mag = 2.0 * sin(ang) / L->a[i + 1];
    p[i] = mag * (cos(-ang) + I * sin(-ang));
  }
}

static double norm2_abs(const cplx *v, int n) {
  double s = 0;
  for (int i = 0; i < n; ++i) {
    double a = cabs(v[i]);
    s += a * a;
  }
  return sqrt(s);
}

/* polarisation vectors as columns: eps[i][pol] */
static void polarisation_vectors(const cplx p[3], cplx eps[3][3]) {
  const double tol = 1e-12;
  double abs_p = norm2_abs(p, 3);
  memset(eps, 0, sizeof(cplx) * 9);
  if (abs_p < tol) return;
  if (cabs(p[0]) > tol) {
    double n12 = norm2_abs(p, 2);
    eps[0][0] = -p[1] / n12;
    eps[1][0] = +p[0] / n12;
    eps[2][0] = 0;
    eps[0][1] = conj(p[0]) * p[2] / (abs_p * n12);
    eps[1][1] = conj(p[1]) * p[2] / (abs_p * n12);
    eps[2][1] = -n12 / abs_p;
  } else {
    double n23 = norm2_abs(p + 1, 2);
    eps[0][0] = 0;
    eps[1][0] = +p[2] / n23;
    eps[2][0] = -p[1] / n23;
    eps[0][1] = 1;
    eps[1][1] = 0;
    eps[2][1] = 0;
  }
  for (int i = 0; i < 3; ++i) eps[i][2] = p[i] / abs_p;
}

int oc_gauge_transverse_box(const oc_lattice *L, double Q, double n0, double g,
                            int64_t seed, int identity_links, double *links,
                            double *efield) {
  const int64_t V = oc_volume(L);
  oc_ranlxd_state rng;
  memset(&rng, 0, sizeof(rng));
  if (oc_ranlxd_init(&rng, 2, seed) != 0) return -1;

  /* r(site, a, pol): real part of complex normals, drawn per site, per pol */
  cplx *r = (cplx *)calloc((size_t)V * 16, sizeof(cplx)); /* [pol][a][site] */
  double buf[16];
  for (int64_t s = 0; s < V; ++s)
    for (int pol = 0; pol < 2; ++pol) {
      oc_random_normal_cmplx(&rng, 8, buf);
      for (int a = 0; a < 8; ++a) r[((int64_t)pol * 8 + a) * V + s] = buf[2 * a];
    }
  double fwd_scale = L->a[1] * L->a[2] * L->a[3];
  double volume = (double)V * fwd_scale;
  for (int k = 0; k < 16; ++k) oc_fft3d((double *)(r + (int64_t)k * V), L->n, -1, fwd_scale);

  cplx *af = (cplx *)calloc((size_t)V * 24, sizeof(cplx)); /* [i][a][site] */
  cplx *ef = (cplx *)calloc((size_t)V * 24, sizeof(cplx));
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    cplx p[3], eps[3][3];
    momentum_backward(L, s, p);
    double pn = norm2_abs(p, 3);
    if (!(pn > 1e-12)) continue;
    double occ = (pn < Q) ? n0 : g * g / 2.0;
    polarisation_vectors(p, eps);
    cplx pa = sqrt(occ / pn * 2.0);
    cplx pe = I * sqrt(occ * pn * 2.0);
    for (int a = 0; a < 8; ++a) {
      cplx r1 = r[(0 * 8 + a) * V + s], r2 = r[(1 * 8 + a) * V + s];
      for (int i = 0; i < 3; ++i) {
        af[((int64_t)i * 8 + a) * V + s] = pa * (r1 * eps[i][0] + r2 * eps[i][1]);
        ef[((int64_t)i * 8 + a) * V + s] = pe * (r1 * eps[i][0] + r2 * eps[i][1]);
      }
    }
  }
  free(r);
  for (int k = 0; k < 24; ++k) {
    oc_fft3d((double *)(af + (int64_t)k * V), L->n, +1, 1.0 / volume);
    oc_fft3d((double *)(ef + (int64_t)k * V), L->n, +1, 1.0 / volume);
  }
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    for (int i = 1; i <= 3; ++i) {
      double as[8], es[8];
      for (int a = 0; a < 8; ++a) {
        as[a] = creal(af[((int64_t)(i - 1) * 8 + a) * V + s]) * L->a[i];
        es[a] = creal(ef[((int64_t)(i - 1) * 8 + a) * V + s]) * L->a[0] * L->a[i];
      }
      cplx G[9];
      if (identity_links) {
        for (int k = 0; k < 9; ++k) G[k] = (k % 4 == 0) ? 1.0 : 0.0;
      } else {
        oc_group_exp(as, (double *)G);
      }
      oc_store_link(links, s, i, G);
      memcpy(efield + (s * 3 + (i - 1)) * 8, es, sizeof(es));
    }
  }
  free(af);
  free(ef);
  return 0;
}

/* ---------------- leapfrog ---------------- */

static void update_links(const oc_lattice *L, double *links, const double *efield, double dt) {
  const int64_t V = oc_volume(L);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    for (int i = 1; i <= 3; ++i) {
      double alpha[8];
      const double *e = oc_efield_at(efield, s, i);
      for (int a = 0; a < 8; ++a) alpha[a] = e[a] * dt;
      cplx G[9], U[9];
      oc_group_exp(alpha, (double *)G);
      oc_load_link(links, s, i, U);
      m3_mul(G, U, U);
      oc_store_link(links, s, i, U);
    }
  }
}

static void ustaple(const oc_lattice *L, const double *links, int i, int k, int64_t s, cplx S[9]) {
  cplx A[9], B[9], C[9];
  oc_load_link(links, oc_neib(L, s, i, +1), k, A);
  oc_load_link(links, oc_neib(L, s, k, +1), i, B);
  oc_load_link(links, s, k, C);
  m3_dag(B, B);
  m3_dag(C, C);
  m3_mul(A, B, S);
  m3_mul(S, C, S);
}

static void dstaple(const oc_lattice *L, const double *links, int i, int k, int64_t s, cplx S[9]) {
  int64_t nk = oc_neib(L, s, k, -1);
  int64_t nik = oc_neib(L, nk, i, +1);
  cplx A[9], B[9], C[9];
  oc_load_link(links, nik, k, A);
  oc_load_link(links, nk, i, B);
  oc_load_link(links, nk, k, C);
  m3_dag(A, A);
  m3_dag(B, B);
  m3_mul(A, B, S);
  m3_mul(S, C, S);
}

static void update_efield(const oc_lattice *L, const double *links, double *efield, double dt) {
  const int64_t V = oc_volume(L);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    for (int i = 1; i <= 3; ++i) {
      cplx sum[9] = {0};
      for (int k = 1; k <= 3; ++k) {
        if (k == i) continue;
        double r = L->a[0] / L->a[k];
        double coef = dt * (r * r);
        cplx SU[9], SD[9];
        ustaple(L, links, i, k, s, SU);
        dstaple(L, links, i, k, s, SD);
        for (int m = 0; m < 9; ++m) sum[m] = sum[m] + coef * (SU[m] + SD[m]);
      }
      cplx U[9], LS[9];
      oc_load_link(links, s, i, U);
      m3_mul(U, sum, LS);
      double *e = efield + (s * 3 + (i - 1)) * 8;
      for (int a = 1; a <= 8; ++a) e[a - 1] = e[a - 1] - 2.0 * cimag(trace_with_generator(a, LS));
    }
  }
}

void oc_gauge_update(const oc_lattice *L, double *links, double *efield, double dt) {
  if (dt > 0) {
    update_links(L, links, efield, dt);
    update_efield(L, links, efield, dt);
  } else {
    update_efield(L, links, efield, dt);
    update_links(L, links, efield, dt);
  }
}

/* ---------------- observables ---------------- */

static void spatial_plaquette(const oc_lattice *L, const double *links, int i, int j, int64_t s,
                              cplx P[9]) {
  cplx l1[9], l2[9], l3[9], l4[9];
  oc_load_link(links, s, i, l1);
  oc_load_link(links, oc_neib(L, s, i, +1), j, l2);
  oc_load_link(links, oc_neib(L, s, j, +1), i, l3);
  oc_load_link(links, s, j, l4);
  m3_dag(l3, l3);
  m3_dag(l4, l4);
  m3_mul(l1, l2, P);
  m3_mul(P, l3, P);
  m3_mul(P, l4, P);
}

static void plaquette(const oc_lattice *L, const double *links, const double *efield, int i,
                      int j, int64_t s, cplx P[9]) {
  if (i == 0 || j == 0) {
    double e[8];
    if (i == 0 && j != 0) {
      const double *ee = oc_efield_at(efield, s, j);
      for (int a = 0; a < 8; ++a) e[a] = +ee[a];
      oc_group_exp(e, (double *)P);
    } else if (i != 0 && j == 0) {
      const double *ee = oc_efield_at(efield, s, i);
      for (int a = 0; a < 8; ++a) e[a] = -ee[a];
      oc_group_exp(e, (double *)P);
    } else {
      for (int k = 0; k < 9; ++k) P[k] = (k % 4 == 0) ? 1.0 : 0.0;
    }
  } else {
    spatial_plaquette(L, links, i, j, s, P);
  }
}

void oc_field_strength(const oc_lattice *L, const double *links, const double *efield, int i,
                       int j, int64_t site, double F[9]) {
  cplx P[9], Lg[9];
  plaquette(L, links, efield, i, j, site, P);
  oc_logu3((const double *)P, (double *)Lg);
  for (int k = 0; k < 9; ++k) {
    /* real( LogU(P)/a_i/a_j/i ) */
    cplx z = Lg[k] / L->a[i] / L->a[j];
    F[k] = cimag(z);
  }
}

double oc_gauge_energy(const oc_lattice *L, const double *links, const double *efield) {
  const int64_t V = oc_volume(L);
  double total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    double local = 0;
    for (int i = 1; i <= 3; ++i) {
      const double *e = oc_efield_at(efield, s, i);
      double sq = 0;
      for (int a = 0; a < 8; ++a) {
        double ea = e[a] / L->a[i] / L->a[0];
        sq += ea * ea;
      }
      local += sq / 2.0;
      for (int j = i + 1; j <= 3; ++j) {
        cplx P[9];
        spatial_plaquette(L, links, i, j, s, P);
        double pot = (1.0 - creal(m3_trace(P)) / 3.0) / L->a[i] / L->a[j];
        local += 2.0 * 3.0 * pot;
      }
    }
    total += local;
  }
  return total;
}

double oc_gauge_gauss_ref(const oc_lattice *L, const double *links, const double *efield) {
  const int64_t V = oc_volume(L);
  double total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    for (int i = 1; i <= 3; ++i) {
      int64_t nb = oc_neib(L, s, i, -1);
      cplx E[9], En[9], Un[9], Und[9], D[9];
      oc_algebra_matrix(oc_efield_at(efield, s, i), (double *)E);
      oc_algebra_matrix(oc_efield_at(efield, nb, i), (double *)En);
      oc_load_link(links, nb, i, Un);
      m3_dag(Un, Und);
      m3_mul(Und, En, D);
      m3_mul(D, Un, D);
      for (int k = 0; k < 9; ++k) D[k] = (E[k] - D[k]) / (L->a[i] * L->a[i]) / L->a[0];
      for (int a = 1; a <= 8; ++a) total += 2.0 * fabs(cimag(trace_with_generator(a, D)));
    }
  }
  return total;
}

static void gauss_G(const oc_lattice *L, const double *links, const double *efield, int64_t s,
                    cplx G[9]) {
  for (int k = 0; k < 9; ++k) G[k] = 0;
  for (int i = 1; i <= 3; ++i) {
    int64_t nb = oc_neib(L, s, i, -1);
    cplx Un[9], Und[9], En[9], E[9], T[9];
    oc_load_link(links, nb, i, Un);
    oc_algebra_matrix(oc_efield_at(efield, nb, i), (double *)En);
    oc_algebra_matrix(oc_efield_at(efield, s, i), (double *)E);
    m3_dag(Un, Und);
    m3_mul(Und, En, T);
    m3_mul(T, Un, T);
    for (int k = 0; k < 9; ++k) G[k] = G[k] + (E[k] - T[k]) / L->a[i];
  }
  for (int k = 0; k < 9; ++k) G[k] = G[k] / L->a[0];
}

double oc_gauge_gauss_maxnorm(const oc_lattice *L, const double *links, const double *efield) {
  const int64_t V = oc_volume(L);
  double mx = 0;
#pragma omp parallel for reduction(max : mx) schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    cplx G[9];
    gauss_G(L, links, efield, s, G);
    for (int a = 1; a <= 8; ++a) {
      double v = 2.0 * cabs(trace_with_generator(a, G));
      if (v > mx) mx = v;
    }
  }
  return mx;
}

int64_t oc_gauge_gauss_project(const oc_lattice *L, double *links, double *efield, double tol,
                               int64_t max_sweeps) {
  const int64_t V = oc_volume(L);
  const double kdt = 0.01 * L->a[0];
  double dev = oc_gauge_gauss_maxnorm(L, links, efield);
  int64_t it = 0;
  double *prev = (double *)malloc(sizeof(double) * (size_t)V * 24);
  while (dev > tol && it < max_sweeps) {
    ++it;
    memcpy(prev, efield, sizeof(double) * (size_t)V * 24);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < V; ++s) {
      cplx G[9];
      gauss_G(L, links, prev, s, G);
      for (int k = 1; k <= 3; ++k) {
        cplx U[9], Ud[9], E[9], Gn[9], T[9];
        oc_load_link(links, s, k, U);
        oc_algebra_matrix(oc_efield_at(prev, s, k), (double *)E);
        gauss_G(L, links, prev, oc_neib(L, s, k, +1), Gn);
        m3_dag(U, Ud);
        m3_mul(U, G, T);
        m3_mul(T, Ud, T);
        m3_mul(T, Gn, T);
        for (int m = 0; m < 9; ++m) T[m] = kdt * (T[m] - G[m]) + E[m];
        double *e = efield + (s * 3 + (k - 1)) * 8;
        for (int a = 1; a <= 8; ++a) e[a - 1] = 2.0 * creal(trace_with_generator(a, T));
      }
    }
    dev = oc_gauge_gauss_maxnorm(L, links, efield);
  }
  free(prev);
  return it;
}

/* EquilibriumInit without charges (gauge:380-814; the measurement branches
   after the projection are jumped over there): cold links, then nefieldinit
   rounds of a thermal E (sigma = sqrt(4/beta); E^a_k(x) = Re(sigma r) a0 for
   complex normals r drawn per site and direction, gauge:432-444), Gauss
   projection to tol, nequilibrium leapfrog steps (gauge:667-672).  Per
   round: projection sweeps, energy and max-norm deviation after the steps
   (any output may be NULL).  Returns -1 for a bad seed, -2 when a projection
   did not converge within max_sweeps. */
int oc_gauge_equilibrium_init(const oc_lattice *L, double beta, int64_t nefieldinit, int64_t nequilibrium,
                              double tol, int64_t seed, int64_t max_sweeps, double *links, double *efield,
                              int64_t *sweeps, double *energies, double *deviations) {
  const int64_t V = oc_volume(L);
  oc_ranlxd_state rng;
  memset(&rng, 0, sizeof(rng));
  if (oc_ranlxd_init(&rng, 2, seed) != 0) return -1;
  const double sigma = sqrt(4.0 / beta);
  oc_gauge_cold(L, links, efield);
  double buf[16];
  for (int64_t r = 0; r < nefieldinit; ++r) {
    for (int64_t s = 0; s < V; ++s)
      for (int k = 0; k < 3; ++k) {
        oc_random_normal_cmplx(&rng, 8, buf);
        for (int a = 0; a < 8; ++a) efield[(s * 3 + k) * 8 + a] = (sigma * buf[2 * a]) * L->a[0];
      }
    int64_t it = oc_gauge_gauss_project(L, links, efield, tol, max_sweeps);
    if (sweeps) sweeps[r] = it;
    if (oc_gauge_gauss_maxnorm(L, links, efield) > tol) return -2;
    for (int64_t t = 0; t < nequilibrium; ++t) oc_gauge_update(L, links, efield, 1.0);
    if (energies) energies[r] = oc_gauge_energy(L, links, efield);
    if (deviations) deviations[r] = oc_gauge_gauss_maxnorm(L, links, efield);
  }
  return 0;
}
