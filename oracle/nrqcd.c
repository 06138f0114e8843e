/*
 * Oracle (test infrastructure only): NRQCD heavy-quark part of the hot path.
 *
 *   InitSinglePoint            src/nrqcd.f90:324-350
 *   GetNorm_Propagator         src/nrqcd.f90:573-611
 *   C2CS / S2CS / GetKronProd  src/nrqcd.f90:452-491, src/matrixoperations.f90:81-104
 *   GetMagneticField_CS_G      src/nrqcd.f90:1669-1693
 *   BuildSystemMatrix          src/nrqcd.f90:1175-1387
 *   AddMatrixToSystem          src/nrqcd.f90:996-1025: the column-major 6x6
 *                              block handed to PETSc MatSetValues is read
 *                              row-major (PETSc default, MAT_ROW_ORIENTED
 *                              never changed), so the operator actually
 *                              assembled holds the TRANSPOSE of every block
 *   Update_CrankNicholson      src/nrqcd.f90:1053-1168:
 *                              RHS = A psi_col; solve A^H psi'_col = RHS,
 *                              quark (+M, c), antiquark (-M, conj c)
 *   meson correlators          src/nrqcd.f90:1484-1661
 *
 * The PETSc KSP (GMRES(30)+ILU(0), left preconditioned, rtol=kspTol) is
 * replaced by an unpreconditioned GMRES(30) on the true residual, run to a
 * tighter tolerance; only converged solutions are comparable.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_internal.h"

#ifdef _OPENMP
#include <omp.h>
#endif

int oc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* threads of the following parallel regions (a launcher may have set
   OMP_NUM_THREADS=1 before the OpenMP runtime loaded) */
void oc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

void oc_heavy_init_single_point(const oc_lattice *L, int64_t lat_index_1based, double *prop_) {
  const int64_t V = oc_volume(L);
  cplx *prop = (cplx *)prop_;
  memset(prop, 0, sizeof(cplx) * (size_t)V * 36);
  int64_t s = lat_index_1based - 1;
  for (int d = 0; d < 6; ++d) prop[s * 36 + d * 6 + d] = 1.0 / sqrt(6.0);
}

double oc_heavy_norm(const oc_lattice *L, const double *prop_) {
  const int64_t V = oc_volume(L);
  const cplx *prop = (const cplx *)prop_;
  double total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    /* Tr Re(psi psi^+) = sum_{row,col} |psi(row,col)|^2 */
    double loc = 0;
    for (int d = 0; d < 6; ++d) {
      cplx acc = 0;
      for (int k = 0; k < 6; ++k) {
        cplx v = prop[s * 36 + k * 6 + d]; /* psi(d,k) */
        acc += v * conj(v);
      }
      loc += creal(acc);
    }
    total += loc;
  }
  return sqrt(total);
}

/* ---------------- system matrix blocks ---------------- */

/* E-field entering the CN operator: -F_{0i}(y) (nrqcd.f90:1254-1255) */
static void efield_cn(const oc_lattice *L, const double *links, const double *efield, int i,
                      int64_t y, cplx E[9]) {
  double F[9];
  oc_field_strength(L, links, efield, 0, i, y, F);
  for (int k = 0; k < 9; ++k) E[k] = -F[k];
}

/* Kron(A 3x3, B 2x2) -> 6x6 with index 2*colour + spin */
static void kron32(const cplx A[9], const cplx B[4], cplx K[36]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      for (int s = 0; s < 2; ++s)
        for (int t = 0; t < 2; ++t) K[(2 * r + s) * 6 + (2 * c + t)] = A[r * 3 + c] * B[s * 2 + t];
}

static void c2cs(const cplx A[9], cplx K[36]) {
  cplx Id[4] = {1, 0, 0, 1};
  kron32(A, Id, K);
}

/* block storage: per site 7 blocks (0 diag, 1+2(i-1) = +i, 2+2(i-1) = -i) */
typedef struct {
  cplx *b; /* V * 7 * 36 */
} blocks_t;

static void add_block(cplx *dst, cplx coef, const cplx M[36], int transpose) {
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) {
      cplx v = coef * M[r * 6 + c];
      if (transpose) dst[c * 6 + r] += v;
      else dst[r * 6 + c] += v;
    }
}

static void build_blocks(const oc_lattice *L, const double *links, const double *efield,
                         double mass, const cplx c[4], double dt, int transpose, blocks_t *B) {
  const int64_t V = oc_volume(L);
  const double a0 = L->a[0];
  const cplx kappa = 0.0 + I * (-dt / 2 * a0);
  memset(B->b, 0, sizeof(cplx) * (size_t)V * 7 * 36);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t x = 0; x < V; ++x) {
    cplx *blk = B->b + x * 7 * 36;
    cplx Id6[36] = {0};
    for (int d = 0; d < 6; ++d) Id6[d * 7] = 1;
    /* O(dt^0) identity */
    add_block(blk, 1.0, Id6, transpose);
    /* kinetic  -c1/2m D^2  (1211-1243) */
    for (int i = 1; i <= 3; ++i) {
      double ai = L->a[i];
      cplx coef = kappa * c[0] / mass / (ai * ai);
      add_block(blk, coef, Id6, transpose);
      cplx U[9], K[36];
      oc_load_link(links, x, i, U);
      c2cs(U, K);
      cplx coefo = kappa * (-c[0]) / 2 / mass / (ai * ai);
      add_block(blk + (1 + 2 * (i - 1)) * 36, coefo, K, transpose);
      int64_t xm = oc_neib(L, x, i, -1);
      cplx Um[9], Umd[9];
      oc_load_link(links, xm, i, Um);
      m3_dag(Um, Umd);
      c2cs(Umd, K);
      add_block(blk + (2 + 2 * (i - 1)) * 36, coefo, K, transpose);
    }
    /* Darwin -c3/8m^2 [D_i, g a_t E_i]  (1245-1269) */
    for (int i = 1; i <= 3; ++i) {
      int64_t xp = oc_neib(L, x, i, +1), xm = oc_neib(L, x, i, -1);
      cplx Ep[9], Em[9], U[9], Um[9], Ud[9], Umd[9], T1[9], T2[9], D[9], K[36];
      efield_cn(L, links, efield, i, xp, Ep);
      efield_cn(L, links, efield, i, xm, Em);
      oc_load_link(links, x, i, U);
      oc_load_link(links, xm, i, Um);
      m3_dag(U, Ud);
      m3_dag(Um, Umd);
      m3_mul(U, Ep, T1);
      m3_mul(T1, Ud, T1);
      m3_mul(Umd, Em, T2);
      m3_mul(T2, Um, T2);
      for (int k = 0; k < 9; ++k) D[k] = (T1[k] - T2[k]) / (2 * L->a[i]);
      c2cs(D, K);
      cplx coef = kappa * (-c[2]) / 8 / (mass * mass);
      add_block(blk, coef, K, transpose);
    }
    /* magnetic -c2 g/2m B (as written: B_i x 1, no sigma)  (1272-1282, 1669-1693) */
    for (int i = 1; i <= 3; ++i) {
      int j = i % 3 + 1, k = (i + 1) % 3 + 1;
      double Fjk[9], Fkj[9];
      cplx Bm[9], K[36];
      oc_field_strength(L, links, efield, j, k, x, Fjk);
      oc_field_strength(L, links, efield, k, j, x, Fkj);
      for (int m = 0; m < 9; ++m) Bm[m] = (Fjk[m] - Fkj[m]) / 2;
      c2cs(Bm, K);
      cplx coef = kappa * (-c[1]) / 2 / mass;
      add_block(blk, coef, K, transpose);
    }
    /* spin-orbit -c4 i/8m^2 eps_ijk sigma_k {D_i, g a_t E_j}  (1285-1381) */
    for (int i = 1; i <= 3; ++i) {
      int64_t xp = oc_neib(L, x, i, +1), xm = oc_neib(L, x, i, -1);
      for (int perm = 0; perm < 2; ++perm) {
        int j, k, eps;
        if (perm == 0) { j = i % 3 + 1; k = (i + 1) % 3 + 1; eps = +1; }
        else { j = (i + 1) % 3 + 1; k = i % 3 + 1; eps = -1; }
        cplx sig[4];
        oc_pauli(k, sig);
        cplx E0[9], Ep[9], Em[9], U[9], Umd[9], T1[9], T2[9], D[9], K[36];
        /* +i neighbour */
        efield_cn(L, links, efield, j, x, E0);
        efield_cn(L, links, efield, j, xp, Ep);
        oc_load_link(links, x, i, U);
        m3_mul(E0, U, T1);
        m3_mul(U, Ep, T2);
        for (int m = 0; m < 9; ++m) D[m] = (T1[m] + T2[m]) / 2 / L->a[i];
        kron32(D, sig, K);
        cplx coefp = kappa * (double)eps * (-c[3]) / 8 / (mass * mass) * I;
        add_block(blk + (1 + 2 * (i - 1)) * 36, coefp, K, transpose);
        /* -i neighbour */
        efield_cn(L, links, efield, j, xm, Em);
        cplx Um[9];
        oc_load_link(links, xm, i, Um);
        m3_dag(Um, Umd);
        m3_mul(E0, Umd, T1);
        m3_mul(Umd, Em, T2);
        for (int m = 0; m < 9; ++m) D[m] = (T1[m] + T2[m]) / 2 / L->a[i];
        kron32(D, sig, K);
        cplx coefm = kappa * (double)eps * (+c[3]) / 8 / (mass * mass) * I;
        add_block(blk + (2 + 2 * (i - 1)) * 36, coefm, K, transpose);
      }
    }
  }
}

static int64_t block_col(const oc_lattice *L, int64_t x, int b) {
  if (b == 0) return x;
  int i = (b - 1) / 2 + 1;
  int sgn = ((b - 1) % 2 == 0) ? +1 : -1;
  return oc_neib(L, x, i, sgn);
}

/* y = A v  (herm=0) or y = A^H v (herm=1) for one 6V-vector v (site-major, 6 dofs) */
static void apply_vec(const oc_lattice *L, const blocks_t *B, int herm, const cplx *v, cplx *y) {
  const int64_t V = oc_volume(L);
#pragma omp parallel for schedule(static)
  for (int64_t x = 0; x < V; ++x) {
    cplx acc[6] = {0};
    for (int b = 0; b < 7; ++b) {
      const cplx *M;
      int64_t src;
      if (!herm) {
        M = B->b + (x * 7 + b) * 36;
        src = block_col(L, x, b);
        for (int r = 0; r < 6; ++r) {
          cplx s = 0;
          for (int c = 0; c < 6; ++c) s += M[r * 6 + c] * v[src * 6 + c];
          acc[r] += s;
        }
      } else {
        /* (A^H)_{x,y} = (A_{y,x})^H ; y = x for diag, y = x -/+ i for block +/-i */
        int bb;
        if (b == 0) { src = x; bb = 0; }
        else {
          int i = (b - 1) / 2 + 1;
          int sgn = ((b - 1) % 2 == 0) ? +1 : -1;
          src = oc_neib(L, x, i, -sgn);
          bb = b;
        }
        M = B->b + (src * 7 + bb) * 36;
        for (int r = 0; r < 6; ++r) {
          cplx s = 0;
          for (int c = 0; c < 6; ++c) s += conj(M[c * 6 + r]) * v[src * 6 + c];
          acc[r] += s;
        }
      }
    }
    for (int r = 0; r < 6; ++r) y[x * 6 + r] = acc[r];
  }
}

static cplx vdot(const cplx *a, const cplx *b, int64_t n) {
  double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
  for (int64_t k = 0; k < n; ++k) {
    cplx p = conj(a[k]) * b[k];
    re += creal(p);
    im += cimag(p);
  }
  return re + I * im;
}

static double vnorm(const cplx *a, int64_t n) { return sqrt(creal(vdot(a, a, n))); }

/* restarted GMRES(m), zero initial guess, unpreconditioned; returns iterations */
static int64_t gmres(const oc_lattice *L, const blocks_t *B, int herm, const cplx *b, cplx *x,
                     double tol, int64_t maxits, int m, double *relres) {
  const int64_t n = oc_volume(L) * 6;
  cplx *Vk = (cplx *)malloc(sizeof(cplx) * (size_t)n * (m + 1));
  cplx *w = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  cplx *H = (cplx *)calloc((size_t)(m + 1) * m, sizeof(cplx));
  cplx *cs = (cplx *)malloc(sizeof(cplx) * m), *g = (cplx *)malloc(sizeof(cplx) * (m + 1));
  double *sn = (double *)malloc(sizeof(double) * m);
  memset(x, 0, sizeof(cplx) * (size_t)n);
  double bnorm = vnorm(b, n);
  if (bnorm == 0.0) {
    *relres = 0;
    free(Vk); free(w); free(H); free(cs); free(g); free(sn);
    return 0;
  }
  int64_t its = 0;
  double res = bnorm;
  while (its < maxits) {
    /* r = b - A x */
    apply_vec(L, B, herm, x, w);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) w[k] = b[k] - w[k];
    double beta = vnorm(w, n);
    res = beta;
    if (beta <= tol * bnorm) break;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) Vk[k] = w[k] / beta;
    memset(g, 0, sizeof(cplx) * (m + 1));
    g[0] = beta;
    int j;
    for (j = 0; j < m && its < maxits; ++j) {
      ++its;
      cplx *vj = Vk + (int64_t)j * n, *vn = Vk + (int64_t)(j + 1) * n;
      apply_vec(L, B, herm, vj, vn);
      for (int i = 0; i <= j; ++i) { /* modified Gram-Schmidt */
        cplx h = vdot(Vk + (int64_t)i * n, vn, n);
        H[i * m + j] = h;
        const cplx *vi = Vk + (int64_t)i * n;
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < n; ++k) vn[k] -= h * vi[k];
      }
      double hn = vnorm(vn, n);
      H[(j + 1) * m + j] = hn;
      if (hn > 0) {
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < n; ++k) vn[k] /= hn;
      }
      for (int i = 0; i < j; ++i) { /* apply previous rotations */
        cplx h0 = H[i * m + j], h1 = H[(i + 1) * m + j];
        H[i * m + j] = conj(cs[i]) * h0 + sn[i] * h1;
        H[(i + 1) * m + j] = -sn[i] * h0 + cs[i] * h1;
      }
      cplx h0 = H[j * m + j];
      double h1 = creal(H[(j + 1) * m + j]);
      double den = sqrt(creal(h0 * conj(h0)) + h1 * h1);
      cplx c_ = (den > 0) ? h0 / den : 1.0;
      double s_ = (den > 0) ? h1 / den : 0.0;
      cs[j] = c_;
      sn[j] = s_;
      H[j * m + j] = conj(c_) * h0 + s_ * h1;
      H[(j + 1) * m + j] = 0;
      cplx gj = g[j];
      g[j] = conj(c_) * gj;
      g[j + 1] = -s_ * gj;
      res = cabs(g[j + 1]);
      if (res <= tol * bnorm) { ++j; break; }
    }
    /* solve upper-triangular H y = g and update x */
    int kk = j;
    cplx *y = (cplx *)malloc(sizeof(cplx) * (kk > 0 ? kk : 1));
    for (int i = kk - 1; i >= 0; --i) {
      cplx s = g[i];
      for (int l = i + 1; l < kk; ++l) s -= H[i * m + l] * y[l];
      y[i] = s / H[i * m + i];
    }
    for (int i = 0; i < kk; ++i) {
      const cplx *vi = Vk + (int64_t)i * n;
      cplx yi = y[i];
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < n; ++k) x[k] += yi * vi[k];
    }
    free(y);
    if (res <= tol * bnorm) {
      /* confirm with the true residual on the next loop iteration */
      apply_vec(L, B, herm, x, w);
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < n; ++k) w[k] = b[k] - w[k];
      res = vnorm(w, n);
      if (res <= tol * bnorm) break;
    }
  }
  *relres = res / bnorm;
  free(Vk); free(w); free(H); free(cs); free(g); free(sn);
  return its;
}

void oc_cn_apply(const oc_lattice *L, const double *links, const double *efield, double mass,
                 const double c_[8], double dt, int herm, int transpose_blocks,
                 const double *psi_in, double *psi_out) {
  const int64_t V = oc_volume(L);
  const cplx *c = (const cplx *)c_;
  blocks_t B;
  B.b = (cplx *)malloc(sizeof(cplx) * (size_t)V * 7 * 36);
  build_blocks(L, links, efield, mass, c, dt, transpose_blocks, &B);
  cplx *v = (cplx *)malloc(sizeof(cplx) * (size_t)V * 6), *y = (cplx *)malloc(sizeof(cplx) * (size_t)V * 6);
  const cplx *pin = (const cplx *)psi_in;
  cplx *pout = (cplx *)psi_out;
  for (int col = 0; col < 6; ++col) {
    for (int64_t s = 0; s < V; ++s)
      for (int r = 0; r < 6; ++r) v[s * 6 + r] = pin[s * 36 + col * 6 + r];
    apply_vec(L, &B, herm, v, y);
    for (int64_t s = 0; s < V; ++s)
      for (int r = 0; r < 6; ++r) pout[s * 36 + col * 6 + r] = y[s * 6 + r];
  }
  free(v); free(y); free(B.b);
}

static int cn_species(const oc_lattice *L, const double *links, const double *efield,
                      double mass, const cplx c[4], double dt, double tol, int64_t maxits,
                      int transpose, cplx *prop, int64_t *iters, double *relres) {
  const int64_t V = oc_volume(L);
  blocks_t B;
  B.b = (cplx *)malloc(sizeof(cplx) * (size_t)V * 7 * 36);
  build_blocks(L, links, efield, mass, c, dt, transpose, &B);
  cplx *v = (cplx *)malloc(sizeof(cplx) * (size_t)V * 6), *rhs = (cplx *)malloc(sizeof(cplx) * (size_t)V * 6);
  cplx *x = (cplx *)malloc(sizeof(cplx) * (size_t)V * 6);
  int ok = 1;
  for (int col = 0; col < 6; ++col) {
    for (int64_t s = 0; s < V; ++s)
      for (int r = 0; r < 6; ++r) v[s * 6 + r] = prop[s * 36 + col * 6 + r];
    apply_vec(L, &B, 0, v, rhs);                 /* RHS = A psi        */
    iters[col] = gmres(L, &B, 1, rhs, x, tol, maxits, 30, &relres[col]); /* A^H x = RHS */
    if (!(relres[col] <= tol)) ok = 0;
    for (int64_t s = 0; s < V; ++s)
      for (int r = 0; r < 6; ++r) prop[s * 36 + col * 6 + r] = x[s * 6 + r];
  }
  free(v); free(rhs); free(x); free(B.b);
  return ok;
}

int oc_cn_update(const oc_lattice *L, const double *links, const double *efield, double mass,
                 const double c_[8], double dt, double tol, int64_t maxits,
                 int transpose_blocks, double *prop_q, double *prop_a, oc_cn_stats *stats) {
  const cplx *c = (const cplx *)c_;
  cplx cc[4];
  for (int k = 0; k < 4; ++k) cc[k] = conj(c[k]);
  oc_cn_stats st;
  memset(&st, 0, sizeof(st));
  int ok1 = cn_species(L, links, efield, +mass, c, dt, tol, maxits, transpose_blocks,
                       (cplx *)prop_q, st.iterations, st.rel_residual);
  int ok2 = cn_species(L, links, efield, -mass, cc, dt, tol, maxits, transpose_blocks,
                       (cplx *)prop_a, st.iterations + 6, st.rel_residual + 6);
  st.converged = ok1 && ok2;
  if (stats) *stats = st;
  return st.converged ? 0 : 1;
}

/* ---------------- meson correlators ---------------- */

static void m6_mul(const cplx *A, const cplx *B, cplx *C) {
  cplx R[36];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      cplx acc = 0;
      for (int k = 0; k < 6; ++k) acc += A[i * 6 + k] * B[k * 6 + j];
      R[i * 6 + j] = acc;
    }
  memcpy(C, R, sizeof(R));
}

static void load_prop(const double *p, int64_t s, cplx M[36]) {
  const cplx *q = (const cplx *)p + s * 36;
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) M[r * 6 + c] = q[c * 6 + r];
}

/* sum_x Tr( i * adag(x) Gam q(x) Gam ) * w over a list of Gamma matrices;
   gconjg replaces adag = conjg(transpose(a)) by conjg(a) (the _gconjg
   variants, src/nrqcd.f90:1728-1905) */
static void correlator_any(const oc_lattice *L, const double *q, const double *a, int ngam,
                           const cplx *gams, double weight_num, double weight_den, int noGam, int gconjg,
                           double out[2]) {
  const int64_t V = oc_volume(L);
  double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    cplx Q[36], A[36], Ad[36], C[36] = {0}, T[36];
    load_prop(q, s, Q);
    load_prop(a, s, A);
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) Ad[i * 6 + j] = gconjg ? conj(A[i * 6 + j]) : conj(A[j * 6 + i]);
    if (noGam) {
      m6_mul(Ad, Q, T);
      for (int k = 0; k < 36; ++k) C[k] = I * T[k];
    } else {
      for (int g = 0; g < ngam; ++g) {
        const cplx *G = gams + g * 36;
        m6_mul(Ad, G, T);
        m6_mul(T, Q, T);
        m6_mul(T, G, T);
        for (int k = 0; k < 36; ++k) C[k] = C[k] + I * T[k] * weight_num / weight_den;
      }
    }
    cplx tr = 0;
    for (int d = 0; d < 6; ++d) tr += C[d * 7];
    re += creal(tr);
    im += cimag(tr);
  }
  out[0] = re;
  out[1] = im;
}

static void meson_o1_1s0(const oc_lattice *L, const double *q, const double *a, int gconjg, double out[2]) {
  correlator_any(L, q, a, 0, NULL, 1, 1, 1, gconjg, out);
}

static void meson_o1_3s1(const oc_lattice *L, const double *q, const double *a, int gconjg, double out[2]) {
  cplx G[3 * 36];
  cplx Id3[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 1; i <= 3; ++i) {
    cplx s[4];
    oc_pauli(i, s);
    kron32(Id3, s, G + (i - 1) * 36);
  }
  correlator_any(L, q, a, 3, G, 1, 3, 0, gconjg, out);
}

static void meson_o8_1s0(const oc_lattice *L, const double *q, const double *a, int gconjg, double out[2]) {
  cplx G[8 * 36];
  for (int g = 1; g <= 8; ++g) {
    cplx T[9];
    oc_generator(g, (double *)T);
    c2cs(T, G + (g - 1) * 36);
  }
  correlator_any(L, q, a, 8, G, 6, 8, 0, gconjg, out);
}

static void meson_o8_3s1(const oc_lattice *L, const double *q, const double *a, int gconjg, double out[2]) {
  cplx G[24 * 36];
  int n = 0;
  for (int i = 1; i <= 3; ++i)
    for (int g = 1; g <= 8; ++g) {
      cplx T[9], s[4];
      oc_generator(g, (double *)T);
      oc_pauli(i, s);
      kron32(T, s, G + (n++) * 36);
    }
  correlator_any(L, q, a, 24, G, 6, 24, 0, gconjg, out);
}

void oc_meson_o1_1s0(const oc_lattice *L, const double *q, const double *a, double out[2]) {
  meson_o1_1s0(L, q, a, 0, out);
}
void oc_meson_o1_3s1(const oc_lattice *L, const double *q, const double *a, double out[2]) {
  meson_o1_3s1(L, q, a, 0, out);
}
void oc_meson_o8_1s0(const oc_lattice *L, const double *q, const double *a, double out[2]) {
  meson_o8_1s0(L, q, a, 0, out);
}
void oc_meson_o8_3s1(const oc_lattice *L, const double *q, const double *a, double out[2]) {
  meson_o8_3s1(L, q, a, 0, out);
}

/* the four _gconjg correlators (src/nrqcd.f90:1728-1905): out[8] = re/im of
   O1(1S0), O1(3S1), O8(1S0), O8(3S1) with conjg(AntiQProp) in place of its
   hermitian conjugate */
void oc_meson_gconjg(const oc_lattice *L, const double *q, const double *a, double out[8]) {
  meson_o1_1s0(L, q, a, 1, out);
  meson_o1_3s1(L, q, a, 1, out + 2);
  meson_o8_1s0(L, q, a, 1, out + 4);
  meson_o8_3s1(L, q, a, 1, out + 6);
}
