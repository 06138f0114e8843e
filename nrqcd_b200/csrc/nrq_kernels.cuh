// Kernel declarations shared between the kernel translation units and the
// C-ABI translation unit.
#pragma once
#include <cuda.h>

#include "nrq_common.cuh"

namespace nrq {

// ---------------- gauge.cu
__global__ void k_links_f2soa(const double2 *__restrict__ f, double2 *__restrict__ U, int64_t V);
__global__ void k_links_soa2f(const double2 *__restrict__ U, double2 *__restrict__ f, int64_t V);
__global__ void k_efield_f2soa(const double *__restrict__ f, double *__restrict__ E, int64_t V);
__global__ void k_efield_soa2f(const double *__restrict__ E, double *__restrict__ f, int64_t V);
__global__ void k_cold(double2 *__restrict__ U, double *__restrict__ E, int64_t V);
__global__ void k_update_links(Lat L, double2 *__restrict__ U, const double *__restrict__ E, double dt);
__global__ void k_update_efield(Lat L, const double2 *__restrict__ U, double *__restrict__ E, double dt);
// precision form of the leapfrog: FP32 links, FP64 Ẽ (gauge.cu)
__global__ void k_update_links32(Lat L, float2 *__restrict__ U, const double *__restrict__ E, double dt);
__global__ void k_update_efield32(Lat L, const float2 *__restrict__ U, double *__restrict__ E, double dt);
__global__ void k_reunitarise(int64_t V, float2 *__restrict__ U32, double2 *__restrict__ U64);
__global__ void k_links_widen(int64_t n, const float2 *__restrict__ U32, double2 *__restrict__ U64);
__global__ void k_links_narrow(int64_t n, const double2 *__restrict__ U64, float2 *__restrict__ U32);
__global__ void k_unitarity(Lat L, const double2 *__restrict__ U, double *partials);
__global__ void k_energy(Lat L, const double2 *__restrict__ U, const double *__restrict__ E, double *partials);
__global__ void k_gauss(Lat L, const double2 *__restrict__ U, const double *__restrict__ E, double *partials);
__global__ void k_reduce_final(const double *__restrict__ partials, int64_t nblk, int nq, unsigned maxmask,
                               double *out);
__global__ void k_ic_pspace(Lat L, const double2 *__restrict__ R, const double *__restrict__ mtab,
                            double fwd_scale, double Q, double n0, double g, double2 *__restrict__ A,
                            double2 *__restrict__ Ef);
__global__ void k_ic_write(Lat L, const double2 *__restrict__ A, const double2 *__restrict__ Ef,
                           double inv_volume, int identity_links, double2 *__restrict__ U,
                           double *__restrict__ E);

// ---------------- gauss_proj.cu
// device state of a Gauss projection: convergence flag, sweeps taken, last
// deviation, and the block ticket of the deviation reduction (zero between
// launches)
struct GaussProjState {
  int done;
  unsigned ticket;
  long long sweeps;
  double dev;
};
__global__ void k_gauss_g(Lat L, const double2 *__restrict__ U, const double *__restrict__ E,
                          double2 *__restrict__ G, double *__restrict__ partials, GaussProjState *st, double tol,
                          int count);
__global__ void k_gauss_sweep(Lat L, const double2 *__restrict__ U, const double2 *__restrict__ G,
                              double *__restrict__ E, const GaussProjState *st, double kdt);

// ---------------- gluon.cu
__global__ void k_cg_divergence(Lat L, const double2 *__restrict__ U, double2 *__restrict__ D,
                                double *__restrict__ partials);
__global__ void k_cg_accelerate(Lat L, double2 *__restrict__ D, double pmax, double scale);
__global__ void k_cg_expah(int64_t V, double2 *__restrict__ D);
__global__ void k_cg_transform(Lat L, double2 *__restrict__ U, const double2 *__restrict__ G);
__global__ void k_gluon_fields(Lat L, const double2 *__restrict__ U, const double *__restrict__ E,
                               double2 *__restrict__ F);
__global__ void k_transverse_corr(Lat L, const double2 *__restrict__ F, double fwd, double volume,
                                  double *__restrict__ out);

// ---------------- cn.cu
// Per-species, per-term complex coefficients of the assembled CN operator:
//   out = in + sum_t alpha_t G_t in      (t = kinetic, magnetic, Darwin, spin-orbit)
struct CnCoef {
  cplx kin[2], mag[2], dar[2], so[2];
  double dkin;       // sum_i 1/a_i^2
  double inva2[3];   // 1/a_i^2
};

// FMA stencil only, the plain solve with the merged update and the shadow
// residual rh kept in FP32 (sh32; any fixed shadow vector serves BiCGStab,
// and every product with it uses the same rounded values):
//   MV_RES2: MV_RES writing rh = f32(r) to sh32 and reducing rh^H r (rho_0);
//   MV_V2:   MV_V with rh^H v from sh32;
//   MV_T2:   MV_T on a materialised s that also reduces rh^H t from sh32,
//            from which the merged update takes beta
enum MvMode { MV_PLAIN = 0, MV_RHS = 1, MV_RES = 2, MV_V = 3, MV_T = 4, MV_RESC = 5, MV_T2 = 6, MV_RES2 = 7,
              MV_V2 = 8 };

struct MvArgs {
  const double2 *in;  // operand (PLAIN/RHS: psi, RES: x, V: p, T: r)
  const double2 *in2; // T: v ; RHS: (unused)
  double2 *out;       // PLAIN: A in ; RHS: b ; RES: r ; V: v ; T: t
  double2 *out2;      // RHS: x0 = 2b - psi ; RES: rh
  double2 *out3;      // RES: p
  const double2 *bvec;// RES: b
  const double *scal; // per-column scalars
  double *partials;   // per block, per column, NQ doubles
  // MV_RESC (residual for the FP32 Chebyshev inner solve): r32 = f32(b - A^H x),
  // d32 = f32((b - A^H x) / theta_species)
  float2 *r32;
  float2 *d32;
  cplx inv_theta[2];
  float2 *sh32;       // RES2: FP32 shadow residual written; V2, T2: read
};

// per-species coefficients of one Chebyshev step: d' = c1 d + c2 r
struct ChebCoef {
  cplx c1[2], c2[2];
};

constexpr int CN_SITES_PER_BLOCK = 32;
constexpr int CN_COLS = 12;  // 2 species x 6 propagator columns
constexpr int SC_STRIDE = 16; // doubles per column in the scalar array
// scalar slots (per column)
enum {
  SC_RHO = 0,    // complex (2)
  SC_ALPHA = 2,  // complex
  SC_OMEGA = 4,  // complex
  SC_BETA = 6,   // complex
  SC_RR = 8,
  SC_BB = 9,
  SC_CONV = 10,  // 1.0 when converged
  SC_BREAK = 11, // 1.0 on breakdown (restart requested)
  SC_NONFIN = 12,
  SC_SS = 13,    // |s|^2 of the half step (when checked)
  SC_HALF = 14   // 1.0 when the half step s = r - alpha v met the tolerance
};

void launch_cn_prepare(Lat L, const double2 *U, const double *E, double2 *Dsum, double *Bsum, double2 *DE,
                       cudaStream_t st);
void launch_cn_mv(int mode, Lat L, const CnCoef &C, const double2 *U, const double2 *Dsum, const double *Bsum,
                  const double2 *DE, const MvArgs &a, cudaStream_t st);
void launch_vec_xr(Lat L, double2 *x, double2 *r, const double2 *p, const double2 *v, const double2 *t,
                   const double2 *rh, const double *scal, double *partials, cudaStream_t st);
void launch_vec_p(Lat L, double2 *p, const double2 *r, const double2 *v, const double *scal, cudaStream_t st);
void launch_vec_s(Lat L, double2 *s, const double2 *r, const double2 *v, const double *scal, cudaStream_t st,
                  double *partials = nullptr);
void launch_vec_xp(Lat L, double2 *x, const double2 *p, const double *scal, cudaStream_t st);
void launch_vec_xrp(Lat L, double2 *x, double2 *r, double2 *p, const double2 *s, const double2 *t,
                    const double2 *v, const double *scal, double *partials, cudaStream_t st);
void launch_vec_xr_s(Lat L, double2 *x, double2 *r, const double2 *p, const double2 *s, const double2 *t,
                     const double2 *rh, const double *scal, double *partials, cudaStream_t st);
// TMA-staged stencil (cn_mv3.cu); returns nonzero if the tensor maps cannot
// describe this lattice (then the caller uses launch_cn_mv).  For MV_T its
// input is the materialised s = r - alpha v.
int launch_cn_mv3(int mode, Lat L, const CnCoef &C, const double2 *U, const double2 *Dsum, const double *Bsum,
                  const double2 *DE, const MvArgs &a, int *err, int sm_count, cudaStream_t st);
// Tensor-core stencil (cn_mv4.cu): forward 6x6 blocks of every site,
// direction and species for coefficients C (216 complex per site), then the
// stencil over them; nb_sign = -1 applies the operator whose off-diagonal
// coefficients are those of C negated.  Needs imaginary off-diagonal
// coefficients.  Returns nonzero if the tensor maps cannot describe this
// lattice.  One partial row per CTA (cn_mv4_rows).
void launch_cn_blocks(Lat L, const CnCoef &C, const double2 *U, const double2 *DE, double2 *W, cudaStream_t st);
int64_t cn_mv4_units(int64_t V);
int64_t cn_mv4_rows(int64_t V, int sm_count);
int launch_cn_mv4(int mode, Lat L, const CnCoef &C, double nb_sign, const double2 *W, const double2 *Dsum,
                  const double *Bsum, const MvArgs &a, int *err, int sm_count, cudaStream_t st);
// FP64 FMA stencil (cn_mv5.cu) on the same forward blocks, stored as 216
// planes (direction, species, row, column; cn_mv5_block_entries complex in
// all); the same conditions as the tensor-core stencil.  wait_cycles bounds
// every pipeline wait; stall_load >= 0 stops the producer before that load
// (the test of the timeout path).  One partial row per CTA (cn_mv5_rows).
// launch_cn_blocks5 writes the blocks in FP64 (W), rounded to FP32 (Wf), or
// both in one pass; a null pointer skips that precision.
void launch_cn_blocks5(Lat L, const CnCoef &C, const double2 *U, const double2 *DE, double2 *W, float2 *Wf,
                       cudaStream_t st);
int64_t cn_mv5_units(int64_t V);
int64_t cn_mv5_rows(int64_t V, int sm_count);
int64_t cn_mv5_block_entries(int64_t V);
int launch_cn_mv5(int mode, Lat L, const CnCoef &C, double nb_sign, const double2 *W, const double2 *Dsum,
                  const double *Bsum, const MvArgs &a, int *err, int sm_count, cudaStream_t st,
                  long long wait_cycles, int stall_load);
// finalize stages: 0 = after RES (rr, bb), 1 = alpha (rh.v), 2 = omega (t.s, t.t), 3 = beta (rh.r, r.r)
void launch_cn_finalize(int stage, int64_t nblocks, const double *partials, double *scal, double tol,
                        cudaStream_t st);
// one field of a batched Crank-Nicolson step (device table entry)
constexpr int BATCH_MAX_CHEB = 32;
struct BatchField {
  CnCoef CA, CH;                 // operator A and A^H coefficients at this field's mass
  double2 *psi, *b, *x;          // FP64 propagator, right-hand side, iterate (72 planes)
  float2 *r32, *dA, *dB, *e32;   // FP32 Chebyshev vectors (72 planes)
  double *partials;              // residual (r.r, b.b) partials of this field
  double *scal;                  // per-column scalars of this field (CN_COLS x SC_STRIDE)
  const double *bounds;          // spectral enclosure of this field's mass (lo0, hi0, lo1, hi1)
  double tau;                    // dt a0 / 2 (signed)
  double mass;                   // heavy mass of this field
  int wblk;                      // the field's FP32 block set (its distinct mass)
  // learned initial guess: the field's history (v1 newest, v2 older; null
  // when absent) and the slot the new history goes to (null: no learned guess)
  const float2 *h1, *h2;
  float2 *hnew;
  // history start without the learned guess: the field's third and fourth
  // newest history vectors (null when absent; h1, h2 the newest two)
  const float2 *h3, *h4;
  cplx inv_theta[2];             // 1/theta per species (written on the device)
  ChebCoef cheb[BATCH_MAX_CHEB]; // Chebyshev steps (written on the device)
  // guaranteed gain |T_m(sigma)| of m Chebyshev steps per species (written
  // on the device)
  double gain[2][BATCH_MAX_CHEB + 1];
};
// every column of the field converged at its last residual check
__device__ __forceinline__ bool batch_field_done(const BatchField &f) {
  bool d = true;
#pragma unroll
  for (int k = 0; k < CN_COLS; ++k) d = d && f.scal[k * SC_STRIDE + SC_CONV] != 0.0;
  return d;
}
// skip_done: residual launches after the first of a step leave converged
// fields alone (their iterate did not change since their last check)
void launch_batch_mv(int mode, int order, Lat L, const double2 *U, const double2 *Dsum, const double *Bsum,
                     const double2 *DE, const BatchField *tab, int nfields, int skip_done, cudaStream_t st);
// The same two modes (MV_RHS, MV_RESC) on the FP64 FMA stencil's blocks
// (cn_batch_mv5.cu): W holds nblk block sets of 216 planes, one per distinct
// mass, built with that mass's A^H coefficients (the field's wblk); fmaps[f]
// the tensor maps of field f's psi and iterate x (written by
// batch_mv5_field_maps before every step; device memory).  The residual's
// partials are one row per (field, 32-site unit), the rows of
// launch_batch_finalize.  Returns nonzero where it does not apply (V even,
// at least 34 sites, V < 2^31).
struct CnBatchMaps {
  struct {
    CUtensorMap spin;   // 72 planes x 2V doubles, box {68, 36}
    CUtensorMap spin1;  // one site, box {2, 36}
  } in[2];              // 0: psi, 1: the iterate x
};
bool batch_mv5_applicable(const Lat &L);
bool batch_mv5_field_maps(CnBatchMaps *m, const Lat &L, const double2 *psi, const double2 *x);
int launch_batch_mv5(int mode, int order, Lat L, const double2 *W, int nblk, const double2 *Dsum, const double *Bsum,
                     const CnBatchMaps *fmaps, const BatchField *tab, int nfields, int skip_done, int *err,
                     int sm_count, cudaStream_t st, long long wait_cycles);
// Chebyshev kernel variants: 0 = one field per tile, 2 blocks/SM (168
// registers); 1 = one field per tile, 3 blocks/SM (113 registers); 2 = two
// fields of one mass per tile, 1 block/SM.  Returns nonzero for an
// unsupported variant (a two-field tile needs an even count per mass).
constexpr int BATCH_CHEB_VARIANTS = 4;
int launch_batch_cheb(int step, int variant, int order, Lat L, const float2 *U, const float2 *Dsum,
                      const float *Bsum, const float2 *DE, const BatchField *tab, int nfields, cudaStream_t st);
// Variant 3 of the batched Chebyshev step: the FP32 block step of
// launch_cheb5f over every field (work items (field, unit), field fastest
// for order 0), on the block sets Wf (nblk of 216 planes, one per distinct
// mass, built with that mass's A^H coefficients) and the fields' d vectors
// (dA_all / dB_all by the step's parity, 72 planes per field).  Returns
// nonzero where it does not apply.
int launch_batch_cheb5f(int step, int order, Lat L, const float2 *Wf, int nblk, const float2 *Dsum,
                        const float *Bsum, const float2 *dA_all, const float2 *dB_all, const BatchField *tab,
                        int nfields, int *err, int sm_count, cudaStream_t st, long long wait_cycles);
void launch_batch_add_e(int64_t n, const BatchField *tab, int nfields, cudaStream_t st);
// Chebyshev coefficients of every field from its mass's bounds; sets
// flags[f] = 1 for non-finite bounds
void launch_batch_coef(BatchField *tab, int nfields, int *flags, cudaStream_t st);
// stage-0 reduction of every field's residual partials (nrows rows per field)
// skip_done: the residual launch skipped the fields whose every column had
// converged (their scalars stay as they are)
void launch_batch_finalize(const BatchField *tab, int nfields, int64_t nrows, double tol, int skip_done,
                           cudaStream_t st);
// The prediction of the scheduled step's last pass (m Chebyshev steps):
// every unconverged column's residual before the pass over the pass's
// guaranteed gain.  pstate = {ratio, steps}: the largest true-to-predicted
// ratio measured so far (-1: none) and the scheduled steps taken.  Where
// prediction is on (a ratio measured and steps not a multiple of 16) and
// twice the prediction, scaled by max(1, ratio), meets tol, the column is
// marked converged on it (SC_HALF = 1, SC_RR the scaled prediction);
// otherwise it waits for the residual check (SC_HALF = 2, SC_SS the
// prediction).  launch_batch_calibrate, after that check, takes the ratio
// of the measured columns into pstate and counts the step.
void launch_batch_predict(const BatchField *tab, int nfields, int m, double tol, const double *pstate,
                          cudaStream_t st);
void launch_batch_calibrate(const BatchField *tab, int nfields, double *pstate, cudaStream_t st);
// The history start of every field (no learned guess): with the field's
// history vectors h1.. (d of them, the first null ends the list) x +=
// sum_k c_k h_k, c of the degree d - 1 extrapolation, and hnew = the same
// sum in FP32 (0 without history), to which every correction is added.
void launch_batch_hist_start(int64_t V, const BatchField *tab, int nfields, cudaStream_t st);
void launch_cn_to_f32(int64_t V, const double2 *U, const double2 *DE, const double2 *D, const double *B, float2 *U32,
                      float2 *DE32, float2 *D32, float *B32, cudaStream_t st);
void launch_cn_bounds(Lat L, const CnCoef &C, double tau, const double2 *U, const double2 *Dsum, const double *Bsum,
                      const double2 *DE, double *partials, double *out, cudaStream_t st);
void launch_cheb32(bool first, Lat L, const CnCoef &C, const float2 *U, const float2 *Dsum, const float *Bsum,
                   const float2 *DE, const float2 *D, float2 *Dn, float2 *R, float2 *E, const ChebCoef &K,
                   cudaStream_t st);
// The same Chebyshev step on the FP32 blocks of launch_cn_blocks5 (Wf, built
// with the coefficients C; nb_sign as for the FP64 FMA stencil), staged by
// TMA (cn_cheb5f.cu).  cheb5f_applicable: the lattices it describes (V a
// multiple of 4, at least 36 sites, nx even, V < 2^31).  Returns nonzero if
// the tensor maps cannot be made; wait_cycles bounds every pipeline wait.
bool cheb5f_applicable(const Lat &L);
int launch_cheb5f(bool first, Lat L, const CnCoef &C, double nb_sign, const float2 *Wf, const float2 *Dsum,
                  const float *Bsum, const float2 *D, float2 *Dn, float2 *R, float2 *E, const ChebCoef &K, int *err,
                  int sm_count, cudaStream_t st, long long wait_cycles);
void launch_add_e(int64_t n, double2 *X, const float2 *E, cudaStream_t st);
void launch_prop_f2soa(const double2 *f, double2 *P, int64_t V, cudaStream_t st);
void launch_prop_soa2f(const double2 *P, double2 *f, int64_t V, cudaStream_t st);
void launch_single_point(double2 *P, int64_t V, int64_t sq, int64_t sa, cudaStream_t st);
void launch_norms(const double2 *P, int64_t V, double *partials, int64_t &nblk, cudaStream_t st);
// x += sum_k c_k t_k over the d newest history vectors t[0..d-1] (d = 1..4),
// c the coefficients of the degree d - 1 extrapolation
void launch_hist_extrapolate(int64_t n, double2 *X, const float2 *const *t, int d, cudaStream_t st);
void launch_hist_store(int64_t n, const double2 *X, const double2 *B, const double2 *Psi, float2 *T, cudaStream_t st);
void launch_correlators(const double2 *P, int64_t V, double *partials, int64_t &nblk, cudaStream_t st,
                        bool gconjg = false);

}  // namespace nrq
