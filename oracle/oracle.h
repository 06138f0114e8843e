/*
 * CPU oracle for the two per-timestep hot paths of the NRQCD simulation
 * (classical-statistical SU(3) leapfrog and the NRQCD Crank-Nicolson step).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark link it.  No
 * product code path may call it.
 *
 * FP64 restatement of the Fortran reference (alexanderlehmann/NRQCD).  Every
 * function cites the reference file:line it follows.  Array layouts are the
 * reference's Fortran column-major layouts flattened with site slowest:
 *   links(3,3,3,V)  complex(8): index ((site*3 + dir)*3 + col)*3 + row
 *   efield(8,3,V)   real(8)   : index (site*3 + dir)*8 + a
 *   prop(6,6,V)     complex(8): index (site*6 + col)*6 + row
 * Site index (0-based) = x + Nx*(y + Ny*z), i.e. lattice index - 1
 * (src/lattice.f90:883-898) with x fastest.
 *
 * Parity pinning: the reference ships no golden data and cannot be built here
 * (Fortran/MPI/PETSc/MKL absent).  The oracle is pinned by the reference's
 * own physics checks (energy, Gauss law, norm, reversibility) and by the
 * exact free-propagation known answer; the ranlxd stream is a faithful
 * restatement that no reference output pins ("parity unpinned" for the RNG).
 */
#ifndef NRQCD_ORACLE_H
#define NRQCD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t n[3];   /* lattice extents Nx, Ny, Nz                    */
  double a[4];    /* spacings a0 (temporal), ax, ay, az            */
} oc_lattice;

/* ---- ranlxd (src/ranlxd_generator.f90) ---------------------------------- */
typedef struct {
  int64_t pr, ir, jr, ir_old, init;
  int64_t next[12];
  double one_bit, carry;
  double xdbl[12];
} oc_ranlxd_state;

int  oc_ranlxd_init(oc_ranlxd_state *s, int64_t level, int64_t seed);
void oc_ranlxd(oc_ranlxd_state *s, double *r, int64_t n);
void oc_ranlxd_get(const oc_ranlxd_state *s, int64_t state[25]);
int  oc_ranlxd_reset(oc_ranlxd_state *s, const int64_t state[25]);
/* Box-Muller complex normals (src/random.f90:238-255): out[2i]=re, out[2i+1]=im */
void oc_random_normal_cmplx(oc_ranlxd_state *s, int64_t n, double *out);

/* ---- FFT with the reference's MKL conventions (src/xpfft.f90:129-139) ---- */
/* data: interleaved complex, x fastest.  sign=-1 forward, +1 backward.      */
void oc_fft3d(double *data, const int64_t n[3], int sign, double scale);

/* ---- SU(3) / matrix operations (src/su3.f90, src/matrixoperations.f90) -- */
/* matrices are interleaved complex, ROW-major m[(r*3+c)*2 + re/im]           */
void oc_generator(int a, double T[18]);                     /* a = 1..8       */
void oc_algebra_matrix(const double alpha[8], double M[18]);
void oc_eigenh3(const double A[18], double d[3], double U[18]);
void oc_eigenc3(const double A[18], double d[6], double U[18]);
void oc_group_exp(const double alpha[8], double G[18]);      /* exp(i a^a T^a) */
void oc_logu3(const double P[18], double L[18]);             /* log via EigenC  */

/* ---- gauge field (src/gaugeconfiguration_su3.f90) ---------------------- */
void   oc_gauge_cold(const oc_lattice *L, double *links, double *efield);
int    oc_gauge_transverse_box(const oc_lattice *L, double Q, double n0, double g,
                               int64_t seed, int identity_links,
                               double *links, double *efield);
void   oc_gauge_update(const oc_lattice *L, double *links, double *efield, double dt);
double oc_gauge_energy(const oc_lattice *L, const double *links, const double *efield);
double oc_gauge_gauss_ref(const oc_lattice *L, const double *links, const double *efield);
double oc_gauge_gauss_maxnorm(const oc_lattice *L, const double *links, const double *efield);
void   oc_field_strength(const oc_lattice *L, const double *links, const double *efield,
                         int i, int j, int64_t site, double F[9]);
/* Gauss projection loop of EquilibriumInit (gauge:494-540); returns sweeps */
int64_t oc_gauge_gauss_project(const oc_lattice *L, double *links, double *efield,
                               double tol, int64_t max_sweeps);
int     oc_gauge_equilibrium_init(const oc_lattice *L, double beta, int64_t nefieldinit, int64_t nequilibrium,
                                  double tol, int64_t seed, int64_t max_sweeps, double *links, double *efield,
                                  int64_t *sweeps, double *energies, double *deviations);

/* ---- heavy quarks (src/nrqcd.f90) -------------------------------------- */
void   oc_heavy_init_single_point(const oc_lattice *L, int64_t lat_index_1based, double *prop);
double oc_heavy_norm(const oc_lattice *L, const double *prop);

/* CN operator as PETSc assembles it.  herm=0: A_eff ; herm=1: A_eff^H.
 * transpose_blocks=1 reproduces PETSc's row-oriented reading of the
 * column-major block (the evolved operator); 0 gives the operator as the
 * Fortran source writes it.  Applies to all 6 propagator columns.          */
void oc_cn_apply(const oc_lattice *L, const double *links, const double *efield,
                 double mass, const double c[8], double dt, int herm,
                 int transpose_blocks, const double *psi_in, double *psi_out);

typedef struct {
  int64_t iterations[12];   /* per species*6 + column                      */
  double  rel_residual[12]; /* true residual ||b - A x|| / ||b||          */
  int     converged;        /* 1 if all columns reached tol               */
} oc_cn_stats;

/* One Crank-Nicolson step of quark and antiquark (nrqcd.f90:1053-1168).
 * c = WilsonCoeffs(4) interleaved complex.  GMRES(restart) on the
 * unpreconditioned residual to rel. tolerance tol. */
int oc_cn_update(const oc_lattice *L, const double *links, const double *efield,
                 double mass, const double c[8], double dt, double tol,
                 int64_t maxits, int transpose_blocks,
                 double *prop_q, double *prop_a, oc_cn_stats *stats);

/* Meson correlators at zero momentum (nrqcd.f90:1484-1661); out[2] */
void oc_meson_o1_1s0(const oc_lattice *L, const double *q, const double *a, double out[2]);
void oc_meson_o1_3s1(const oc_lattice *L, const double *q, const double *a, double out[2]);
void oc_meson_o8_1s0(const oc_lattice *L, const double *q, const double *a, double out[2]);
void oc_meson_o8_3s1(const oc_lattice *L, const double *q, const double *a, double out[2]);
/* the _gconjg correlators (nrqcd.f90:1728-1905); out[8] */
void oc_meson_gconjg(const oc_lattice *L, const double *q, const double *a, double out[8]);

/* ---- gluon distribution (src/gaugeconfiguration_su3.f90:1825-1972, 2269-2478) */
double  oc_norm2_momentum(const oc_lattice *L, int64_t site);
int64_t oc_gauge_coulomb_gaugefix(const oc_lattice *L, double *links, double tol, double alpha,
                                  int64_t max_iterations, double *deviations);
void    oc_gauge_transverse_correlators(const oc_lattice *L, const double *links, const double *efield,
                                        double *aa, double *ee, double *momenta);

int oc_num_threads(void);
void oc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
