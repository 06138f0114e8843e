/* Oracle (test infrastructure only): shared internal helpers. */
#ifndef NRQCD_ORACLE_INTERNAL_H
#define NRQCD_ORACLE_INTERNAL_H
#include <complex.h>
#include <stdint.h>
#include "oracle.h"

typedef double complex cplx;

void m3_mul(const cplx A[9], const cplx B[9], cplx C[9]);
void m3_dag(const cplx A[9], cplx B[9]);
cplx m3_trace(const cplx A[9]);
cplx trace_with_generator(int a, const cplx M[9]);
void expi_hermitian(const cplx A[9], cplx G[9]);
void oc_pauli(int k, cplx S[4]);

static inline int64_t oc_volume(const oc_lattice *L) { return L->n[0] * L->n[1] * L->n[2]; }

/* periodic neighbour: dir in 1..3, sgn = +1/-1 (src/lattice.f90:846-947) */
static inline int64_t oc_neib(const oc_lattice *L, int64_t site, int dir, int sgn) {
  int64_t x = site % L->n[0];
  int64_t y = (site / L->n[0]) % L->n[1];
  int64_t z = site / (L->n[0] * L->n[1]);
  if (dir == 1) x = (x + sgn + L->n[0]) % L->n[0];
  else if (dir == 2) y = (y + sgn + L->n[1]) % L->n[1];
  else z = (z + sgn + L->n[2]) % L->n[2];
  return x + L->n[0] * (y + L->n[1] * z);
}

/* link U_dir(site) (dir 1..3) from the Fortran layout links(3,3,3,V) */
static inline void oc_load_link(const double *links, int64_t site, int dir, cplx U[9]) {
  const cplx *l = (const cplx *)links + (site * 3 + (dir - 1)) * 9;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) U[r * 3 + c] = l[c * 3 + r];
}
static inline void oc_store_link(double *links, int64_t site, int dir, const cplx U[9]) {
  cplx *l = (cplx *)links + (site * 3 + (dir - 1)) * 9;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) l[c * 3 + r] = U[r * 3 + c];
}
static inline const double *oc_efield_at(const double *efield, int64_t site, int dir) {
  return efield + (site * 3 + (dir - 1)) * 8;
}

#endif
