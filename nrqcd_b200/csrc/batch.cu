// Batching form of the Crank-Nicolson step (C ABI: nrq_cn_batch_*,
// nrq_ensemble_*).
//
// A batch advances n heavy fields (sources x masses) of one context through
// one CN step in one gauge field.  Every kernel covers all n fields: the
// FP64 right-hand-side and residual stencils take the field from the block
// index, and the FP32 Chebyshev stencil applies each gauge-derived weight to
// a tile of fields of the same mass.  Field pointers and mass-dependent
// coefficients live in a device table (nrq::BatchField); the Chebyshev
// coefficients are computed on the device from the per-mass spectral bounds,
// so once the per-pass inner step counts (the schedule) are known a whole step
// enqueues without host synchronisation and is captured as a CUDA graph.
//
// The batch keeps its own FP64 copy of the links, so its solve reads nothing
// that the leapfrog writes: an ensemble member's step (CN, then leapfrog, as
// src/main.f90:346-348) is one child graph, and a field that misses the
// tolerance after the scheduled passes can still be refined after the
// leapfrog has run.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/nrqcd_b200.h"
#include "nrq_internal.h"
#include "nrq_kernels.cuh"

using nrqh::check_launch;
using nrqh::set_device;

struct nrq_cn_batch {
  nrq_ctx *ctx = nullptr;
  int nf = 0;
  double tol = 1e-10;
  // table order: fields grouped by mass (stable); user[i] = user index of entry i
  std::vector<nrq_heavy *> fields;
  std::vector<int> user;
  std::vector<int> mass_of;       // entry -> distinct mass index
  std::vector<double> masses;     // distinct masses
  std::vector<int> group_size;    // fields per distinct mass
  std::vector<double2 *> xbuf;    // current iterate buffer of every entry
  // per-step gauge-derived data (owned copies)
  double2 *U64 = nullptr, *Dsum = nullptr, *DE = nullptr;
  double *Bsum = nullptr;
  float2 *U32 = nullptr, *DE32 = nullptr, *D32 = nullptr;
  float *B32 = nullptr;
  double *bpart = nullptr;   // bounds partial blocks
  double *bounds = nullptr;  // 4 per distinct mass
  // per-field vectors, contiguous over fields
  double2 *b_all = nullptr;
  float2 *r32_all = nullptr, *dA_all = nullptr, *dB_all = nullptr, *e32_all = nullptr;
  double *part_all = nullptr, *scal_all = nullptr;
  // the scheduled steps' predicted acceptance: {largest true-to-predicted
  // ratio measured (-1: none), scheduled steps taken} (device)
  double *pstate = nullptr;
  // without a learned guess every field starts from 2b - psi plus the
  // extrapolation of its last kBatchHistDepth corrections, as the
  // single-field solves do
  bool history = true;
  int *flags = nullptr;
  int64_t nsb = 0;  // 32-site blocks
  // device table and pinned mirrors
  nrq::BatchField *d_tab = nullptr, *h_tab = nullptr;
  double *h_scal = nullptr;
  int *h_flags = nullptr;
  double *h_bounds = nullptr;
  // calibration key, schedule and tuning
  bool have_key = false;
  double key_dt = 0.0, key_c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<int> schedule;
  bool tuned = false;
  int variant = 0, order = 0;  // Chebyshev kernel variant (nrq_kernels.cuh) and block order
  double cand_ms[2 * nrq::BATCH_CHEB_VARIANTS] = {-1, -1, -1, -1, -1, -1, -1, -1};
  // FP32 blocks of every distinct mass (Chebyshev variant 3; null where the
  // lattice does not allow it) and the bounded waits' error record
  float2 *W5f = nullptr;
  int *err = nullptr, *h_err = nullptr;
  // the FP64 stencil of the right-hand side and residuals: per-update FP64
  // blocks of every distinct mass and every field's tensor maps (null where
  // the lattice does not allow it); fp64 = 1 runs it, 0 the register-tiled
  // one (timed with the Chebyshev candidates)
  double2 *W5 = nullptr;
  nrq::CnBatchMaps *d_fmaps = nullptr, *h_fmaps = nullptr;
  int fp64 = 0;
  double fp64_ms[2] = {-1, -1};
  // generation: changes with every new schedule, tuning or key
  uint64_t gen = 0;
  // graph of one scheduled step (CN only), with the generation and gauge
  // field it was captured for
  cudaGraphExec_t exec = nullptr;
  uint64_t exec_gen = 0;
  const nrq_gauge *exec_g = nullptr;
  // learned initial guess (attached network, per-batch scratch) and the
  // history depth the schedule was calibrated for
  nrq_learn *learn = nullptr;
  float4 *lgf = nullptr, *lomega = nullptr;
  float *lfeat = nullptr;
  int key_depth = -1;
  // the guess's gate: -1 undecided, 1 on, 0 off (it cost more than the
  // Chebyshev steps and passes it saved, measured at the calibration with
  // the full two-step history); the last schedule calibrated without the
  // guess, the measured cost of the guess and the value of what it saved
  int learn_gate = -1;
  bool have_plain = false;
  double plain_dt = 0.0, plain_c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<int> plain_schedule;
  bool time_guess = false;
  double guess_ms = -1.0, guess_saving_ms = -1.0;
  // statistics of the last update
  int64_t last_inner = 0, last_passes = 0, last_matvecs = 0;
  double last_maxrel = 0.0, last_initial = 0.0;
  bool last_conv = false;
};

struct nrq_ensemble {
  std::vector<nrq_cn_batch *> batches;
  std::vector<nrq_gauge *> gauges;
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> exec_gen;  // member generations the graph was captured for
};

namespace {

constexpr int kMaxPasses = 8;
constexpr size_t kFieldScal = (size_t)nrq::CN_COLS * nrq::SC_STRIDE;

int64_t plane(const nrq_cn_batch *b) { return 72 * b->ctx->lat.V; }

void free_graph(cudaGraphExec_t &g) {
  if (g) cudaGraphExecDestroy(g);
  g = nullptr;
}

bool learned_on(const nrq_cn_batch *b) {
  return b->learn && nrqh::learned_ready(b->learn) && b->learn_gate != 0;
}

constexpr int kBatchHistDepth = 4;
bool hist_on(const nrq_cn_batch *b) { return b->history && !learned_on(b); }

// history depth of the start (every field's count, capped at 2 for the
// learned guess and at kBatchHistDepth for the extrapolation), -1 without one
int depth_of(const nrq_cn_batch *b) {
  if (!learned_on(b) && !hist_on(b)) return -1;
  int d = learned_on(b) ? 2 : kBatchHistDepth;
  for (const nrq_heavy *h : b->fields) d = std::min(d, h->hist_count);
  return d;
}

// every field's history ring holds the extrapolation's steps
int ensure_batch_hist(nrq_cn_batch *b) {
  if (!hist_on(b)) return NRQ_OK;
  for (nrq_heavy *h : b->fields) {
    const int rc = nrqh::ensure_hist(h, kBatchHistDepth);
    if (rc) return rc;
  }
  return NRQ_OK;
}

bool same_key(const nrq_cn_batch *b, const double c[8], double dt) {
  if (!b->have_key || b->key_dt != dt || b->key_depth != depth_of(b)) return false;
  for (int k = 0; k < 8; ++k)
    if (b->key_c[k] != c[k]) return false;
  return true;
}

// table mirror for the current field/iterate pointers and coefficients
void fill_table(nrq_cn_batch *b, const double c[8], double dt) {
  nrq_ctx *ctx = b->ctx;
  const int64_t P = plane(b);
  const int64_t nrows = b->nsb;
  for (int i = 0; i < b->nf; ++i) {
    nrq::BatchField &f = b->h_tab[i];
    std::memset((void *)&f, 0, sizeof(f));
    const double m = b->masses[b->mass_of[i]];
    f.CA = nrqh::make_coef(ctx, m, c, dt, false);
    f.CH = nrqh::make_coef(ctx, m, c, dt, true);
    f.psi = b->fields[i]->P;
    f.b = b->b_all + (int64_t)i * P;
    f.x = b->xbuf[i];
    f.r32 = b->r32_all + (int64_t)i * P;
    f.dA = b->dA_all + (int64_t)i * P;
    f.dB = b->dB_all + (int64_t)i * P;
    f.e32 = b->e32_all + (int64_t)i * P;
    f.partials = b->part_all + (int64_t)i * nrows * nrq::CN_COLS * 2;
    f.scal = b->scal_all + (int64_t)i * kFieldScal;
    f.bounds = b->bounds + 4 * b->mass_of[i];
    f.tau = dt * ctx->a[0] / 2.0;
    f.mass = m;
    f.wblk = b->mass_of[i];
    if (b->h_fmaps && !nrq::batch_mv5_field_maps(b->h_fmaps + i, ctx->lat, f.psi, f.x)) b->fp64 = 0;
    if (learned_on(b)) {
      nrq_heavy *h = b->fields[i];
      f.h1 = hist_v1(h);
      f.h2 = hist_v2(h);
      f.hnew = hist_next(h);
    } else if (hist_on(b)) {
      nrq_heavy *h = b->fields[i];
      f.h1 = hist_v(h, 1);
      f.h2 = hist_v(h, 2);
      f.h3 = hist_v(h, 3);
      f.h4 = hist_v(h, 4);
      f.hnew = hist_next(h);
    }
  }
}

int upload_table(nrq_cn_batch *b, cudaStream_t st) {
  NRQ_CUDA_TRY(b->ctx, cudaMemcpyAsync(b->d_tab, b->h_tab, sizeof(nrq::BatchField) * b->nf,
                                       cudaMemcpyHostToDevice, st));
  if (b->d_fmaps)
    NRQ_CUDA_TRY(b->ctx, cudaMemcpyAsync(b->d_fmaps, b->h_fmaps, sizeof(nrq::CnBatchMaps) * b->nf,
                                         cudaMemcpyHostToDevice, st));
  return NRQ_OK;
}

// ---- enqueue helpers (no host synchronisation) ----------------------------
// the FP64 stencil of every field: MV_RHS or MV_RESC, the FMA stencil on the
// blocks (fp64 = 1, where it applies) or the register-tiled one
void launch_fp64(nrq_cn_batch *b, int mode, int fp64, int skip_done, cudaStream_t st) {
  nrq_ctx *ctx = b->ctx;
  if (fp64 == 1 && b->W5 &&
      nrq::launch_batch_mv5(mode, b->order, ctx->lat, b->W5, (int)b->masses.size(), b->Dsum, b->Bsum, b->d_fmaps,
                            b->d_tab, b->nf, skip_done, b->err, ctx->sm_count, st, nrq_wait_cycles_default) == 0)
    return;
  nrq::launch_batch_mv(mode, b->order, ctx->lat, b->U64, b->Dsum, b->Bsum, b->DE, b->d_tab, b->nf, skip_done, st);
}

// gauge-derived data of this step: link copy, CN blocks, FP32 copies, the
// spectral enclosure of every mass and the Chebyshev coefficients of every
// field
int enq_prepare(nrq_cn_batch *b, const nrq_gauge *g, const double c[8], double dt, cudaStream_t st) {
  nrq_ctx *ctx = b->ctx;
  const nrq::Lat L = ctx->lat;
  const int64_t V = L.V;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(b->U64, g->U, sizeof(double2) * 27 * V, cudaMemcpyDeviceToDevice, st));
  {
    ProfScope ps(ctx, 3, (double)V * (432.0 + 192.0));
    nrq::launch_cn_prepare(L, b->U64, g->E, b->Dsum, b->Bsum, b->DE, st);
  }
  {
    ProfScope ps(ctx, 3, (double)V * (1080.0 + 540.0));
    nrq::launch_cn_to_f32(V, b->U64, b->DE, b->Dsum, b->Bsum, b->U32, b->DE32, b->D32, b->B32, st);
  }
  // per-update blocks of every mass: FP32 for Chebyshev variant 3, FP64 for
  // the FP64 FMA stencil (the tuner times both before it chooses)
  const bool want32 = b->W5f && (!b->tuned || b->variant == 3), want64 = b->W5 && (!b->tuned || b->fp64 == 1);
  if (want32 || want64)
    for (size_t k = 0; k < b->masses.size(); ++k) {
      ProfScope ps(ctx, 3, (double)V * (432.0 + 864.0 + (want32 ? 1728.0 : 0.0) + (want64 ? 3456.0 : 0.0)));
      const nrq::CnCoef CH = nrqh::make_coef(ctx, b->masses[k], c, dt, true);
      const int64_t off = (int64_t)k * nrq::cn_mv5_block_entries(V);
      nrq::launch_cn_blocks5(L, CH, b->U64, b->DE, want64 ? b->W5 + off : nullptr, want32 ? b->W5f + off : nullptr,
                             st);
    }
  const double tau = dt * ctx->a[0] / 2.0;
  for (size_t k = 0; k < b->masses.size(); ++k) {
    ProfScope ps(ctx, 3, (double)V * (432.0 + 864.0 + 216.0));
    const nrq::CnCoef CH = nrqh::make_coef(ctx, b->masses[k], c, dt, true);
    nrq::launch_cn_bounds(L, CH, tau, b->U64, b->Dsum, b->Bsum, b->DE, b->bpart, b->bounds + 4 * k, st);
  }
  nrq::launch_batch_coef(b->d_tab, b->nf, b->flags, st);
  return check_launch(ctx, "batch prepare");
}

// b = A psi and the start x (2b - psi, or the learned guess)
int enq_rhs(nrq_cn_batch *b, const nrq_gauge *g, cudaStream_t st) {
  nrq_ctx *ctx = b->ctx;
  {
    ProfScope ps(ctx, 0, (double)ctx->lat.V * (b->nf * 1152.0 * 3 + 432.0 + 192.0));
    launch_fp64(b, nrq::MV_RHS, b->fp64, 0, st);
  }
  int rc = check_launch(ctx, "batch rhs");
  if (!rc && hist_on(b)) {
    ProfScope ps(ctx, 1, (double)ctx->lat.V * b->nf * (1152.0 * 2 + 576.0 * (kBatchHistDepth + 1)));
    nrq::launch_batch_hist_start(ctx->lat.V, b->d_tab, b->nf, st);
    rc = check_launch(ctx, "batch history start");
  }
  if (!rc && learned_on(b)) {
    ProfScope ps(ctx, 3, (double)ctx->lat.V * b->nf * (1152.0 * 4 + 576.0 * 5 + 128.0));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (b->time_guess) {  // the gate's measurement of the guess's cost
      NRQ_CUDA_TRY(ctx, cudaEventCreate(&e0));
      NRQ_CUDA_TRY(ctx, cudaEventCreate(&e1));
      cudaEventRecord(e0, st);
    }
    rc = nrqh::learned_guess_batch(b->learn, ctx, b->d_tab, b->nf, b->U64, g->E, b->lgf, b->lfeat, b->lomega, st);
    if (b->time_guess) {
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      b->guess_ms = ms;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
  }
  return rc;
}

// r = b - A^H x (FP64) of every field, FP32 copies r32 and d = r/theta, and
// the per-column (r.r, b.b) reduction.  After the first check of a step
// (first = false) fields that already converged are skipped.
int enq_residual(nrq_cn_batch *b, cudaStream_t st, bool first) {
  nrq_ctx *ctx = b->ctx;
  {
    ProfScope ps(ctx, 0, (double)ctx->lat.V * (b->nf * (1152.0 * 2 + 576.0 * 2) + 432.0 + 192.0));
    launch_fp64(b, nrq::MV_RESC, b->fp64, first ? 0 : 1, st);
  }
  {
    ProfScope ps(ctx, 2, (double)b->nf * b->nsb * nrq::CN_COLS * 2 * 8);
    nrq::launch_batch_finalize(b->d_tab, b->nf, b->nsb, b->tol, first ? 0 : 1, st);
  }
  return check_launch(ctx, "batch residual");
}

// Chebyshev step `step` of every field with kernel variant / block order
// (nonzero: the variant does not apply)
int launch_cheb(nrq_cn_batch *b, int step, int variant, int order, cudaStream_t st) {
  nrq_ctx *ctx = b->ctx;
  if (variant == 3)
    return b->W5f ? nrq::launch_batch_cheb5f(step, order, ctx->lat, b->W5f, (int)b->masses.size(), b->D32, b->B32,
                                             b->dA_all, b->dB_all, b->d_tab, b->nf, b->err, ctx->sm_count, st,
                                             nrq_wait_cycles_default)
                  : 1;
  return nrq::launch_batch_cheb(step, variant, order, ctx->lat, b->U32, b->D32, b->B32, b->DE32, b->d_tab, b->nf,
                                st);
}

// m FP32 Chebyshev steps on A^H e = r, then x += e
int enq_inner(nrq_cn_batch *b, int m, cudaStream_t st) {
  nrq_ctx *ctx = b->ctx;
  const double V = (double)ctx->lat.V;
  for (int k = 0; k < m; ++k) {
    ProfScope ps(ctx, 0, V * (b->nf * 576.0 * 6 + 756.0));
    if (launch_cheb(b, k, b->variant, b->order, st)) {
      ctx->last_error = "batch: unsupported Chebyshev tile";
      return NRQ_ERR_BAD_ARG;
    }
  }
  {
    ProfScope ps(ctx, 1, V * b->nf * (1152.0 * 2 + 576.0));
    nrq::launch_batch_add_e(72 * ctx->lat.V, b->d_tab, b->nf, st);
  }
  return check_launch(ctx, "batch inner solve");
}

int enq_readback(nrq_cn_batch *b, cudaStream_t st) {
  NRQ_CUDA_TRY(b->ctx, cudaMemcpyAsync(b->h_scal, b->scal_all, sizeof(double) * kFieldScal * b->nf,
                                       cudaMemcpyDeviceToHost, st));
  NRQ_CUDA_TRY(b->ctx, cudaMemcpyAsync(b->h_flags, b->flags, sizeof(int) * b->nf, cudaMemcpyDeviceToHost, st));
  NRQ_CUDA_TRY(b->ctx, cudaMemcpyAsync(b->h_err, b->err, sizeof(int) * 16, cudaMemcpyDeviceToHost, st));
  return NRQ_OK;
}

// the scheduled step: prepare, RHS, the scheduled passes, the final residual
// check and its read-back.  After the last pass its Chebyshev prediction
// marks the columns it brings within the tolerance (with the measured
// margin) as converged, so that the final check skips the fields it
// predicts in full; the check's measured columns then calibrate the margin.
int enq_scheduled(nrq_cn_batch *b, const nrq_gauge *g, const double c[8], double dt, cudaStream_t st) {
  int rc = enq_prepare(b, g, c, dt, st);
  if (!rc) rc = enq_rhs(b, g, st);
  for (size_t p = 0; !rc && p < b->schedule.size(); ++p) {
    rc = enq_residual(b, st, p == 0);
    if (!rc) rc = enq_inner(b, b->schedule[p], st);
  }
  const bool predict = !b->schedule.empty();
  if (!rc && predict) nrq::launch_batch_predict(b->d_tab, b->nf, b->schedule.back(), b->tol, b->pstate, st);
  if (!rc) rc = enq_residual(b, st, b->schedule.empty());
  if (!rc && predict) {
    nrq::launch_batch_calibrate(b->d_tab, b->nf, b->pstate, st);
    rc = check_launch(b->ctx, "batch prediction");
  }
  if (!rc) rc = enq_readback(b, st);
  return rc;
}

// ---- host-side checks -------------------------------------------------------
struct Check {
  bool conv = true, nonfin = false, badbounds = false, timeout = false;
  double worst = 0.0;
};
Check check(const nrq_cn_batch *b) {
  Check r;
  r.timeout = b->h_err[0] != 0;
  for (int i = 0; i < b->nf; ++i) {
    if (b->h_flags[i]) r.badbounds = true;
    const double *s = b->h_scal + (size_t)i * kFieldScal;
    for (int k = 0; k < nrq::CN_COLS; ++k) {
      const double *sc = s + k * nrq::SC_STRIDE;
      r.conv = r.conv && sc[nrq::SC_CONV] != 0.0;
      r.nonfin = r.nonfin || sc[nrq::SC_NONFIN] != 0.0;
      if (sc[nrq::SC_BB] > 0) r.worst = std::max(r.worst, std::sqrt(sc[nrq::SC_RR] / sc[nrq::SC_BB]));
    }
  }
  return r;
}

// inner steps whose guaranteed Chebyshev gain reaches `gain` for every mass
// and species
int steps_for(const nrq_cn_batch *b, double dt, double gain) {
  gain = std::max(gain, 10.0);
  // FP32 arithmetic caps one pass at about 1e6; a pass that can finish the
  // solve may aim up to 3e7 (the FP64 check decides whether it did)
  if (gain > 3e7) gain = 1e6;
  const double tau = dt * b->ctx->a[0] / 2.0;
  int m = 1;
  for (; m < nrq::BATCH_MAX_CHEB; ++m) {
    double g = 1e300;
    for (size_t k = 0; k < b->masses.size(); ++k)
      for (int sp = 0; sp < 2; ++sp) {
        const double *bd = b->h_bounds + 4 * k + 2 * sp;
        g = std::min(g, nrqh::cheb_gain(nrqh::cheb_segment(tau, bd[0], bd[1]).sigma, m));
      }
    if (g >= gain) break;
  }
  return m;
}

// candidate kernels timed on the step's own buffers: every buffer a candidate
// writes (r32, e32, d of the second slot, the residual partials) is rewritten
// by the residual and first Chebyshev step of the solve before it is read.
int autotune(nrq_cn_batch *b, cudaStream_t st) {
  nrq_ctx *ctx = b->ctx;
  bool even = true;
  for (int n : b->group_size) even = even && (n % 2 == 0);
  cudaEvent_t e0, e1;
  NRQ_CUDA_TRY(ctx, cudaEventCreate(&e0));
  NRQ_CUDA_TRY(ctx, cudaEventCreate(&e1));
  double best = 1e300;
  int best_variant = 0, best_order = 0;
  const int reps = 3;
  // no field may count as converged while the candidates are timed (the
  // residual check of the solve rewrites these flags before they matter)
  NRQ_CUDA_TRY(ctx, cudaMemsetAsync(b->scal_all, 0, sizeof(double) * kFieldScal * b->nf, st));
  for (int variant = 0; variant < nrq::BATCH_CHEB_VARIANTS; ++variant)
    for (int order = 0; order < 2; ++order) {
      const int idx = variant * 2 + order;
      b->cand_ms[idx] = -1.0;
      if ((variant == 2 && !even) || (variant == 3 && !b->W5f)) continue;
      // warm-up launch, then timed repetitions
      int bad = launch_cheb(b, 0, variant, order, st);
      cudaEventRecord(e0, st);
      for (int r = 0; r < reps && !bad; ++r) bad = launch_cheb(b, 0, variant, order, st);
      cudaEventRecord(e1, st);
      if (bad) continue;
      int rc = check_launch(ctx, "batch autotune");
      if (rc) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
      }
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      b->cand_ms[idx] = ms / reps;
      if (ms / reps < best) {
        best = ms / reps;
        best_variant = variant;
        best_order = order;
      }
    }
  b->variant = best_variant;
  b->order = best_order;
  // the FP64 residual stencil (it writes r32, d of the first slot and the
  // partials, which the solve's first residual rewrites), in the chosen order
  b->fp64 = 0;
  for (int which = 0; which < 2; ++which) {
    b->fp64_ms[which] = -1.0;
    if (which == 1 && !b->W5) continue;
    launch_fp64(b, nrq::MV_RESC, which, 0, st);
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) launch_fp64(b, nrq::MV_RESC, which, 0, st);
    cudaEventRecord(e1, st);
    int rc = check_launch(ctx, "batch autotune");
    if (rc) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return rc;
    }
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    b->fp64_ms[which] = ms / reps;
  }
  if (b->fp64_ms[1] > 0.0 && b->fp64_ms[1] < b->fp64_ms[0]) b->fp64 = 1;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tuned = true;
  return NRQ_OK;
}

// Adaptive refinement after a residual check already read back: passes of
// m inner steps (m from the worst residual) until every field converges or
// `budget` passes ran.  Appends the step counts used to `used`.
int refine_adaptive(nrq_cn_batch *b, double dt, cudaStream_t st, int budget, std::vector<int> &used, Check &chk) {
  nrq_ctx *ctx = b->ctx;
  for (int p = 0; p < budget && !chk.conv && !chk.nonfin && !chk.badbounds && !chk.timeout; ++p) {
    const int m = steps_for(b, dt, chk.worst / (0.3 * b->tol));
    int rc = enq_inner(b, m, st);
    if (!rc) rc = enq_residual(b, st, false);
    if (!rc) rc = enq_readback(b, st);
    if (rc) return rc;
    NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    used.push_back(m);
    chk = check(b);
  }
  return NRQ_OK;
}

// calibration step: adaptive passes with host synchronisation; records the
int64_t sum(const std::vector<int> &v) {
  int64_t s = 0;
  for (int x : v) s += x;
  return s;
}

// schedule and tunes the kernels on the first call
int update_calibrate(nrq_cn_batch *b, const nrq_gauge *g, const double c[8], double dt, cudaStream_t st,
                     Check &chk) {
  nrq_ctx *ctx = b->ctx;
  int rc = enq_prepare(b, g, c, dt, st);
  if (rc) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(b->h_bounds, b->bounds, sizeof(double) * 4 * b->masses.size(),
                                    cudaMemcpyDeviceToHost, st));
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (!b->tuned && (rc = autotune(b, st))) return rc;
  const bool deciding = learned_on(b) && b->learn_gate < 0 && depth_of(b) == 2;
  b->time_guess = deciding;
  rc = enq_rhs(b, g, st);
  b->time_guess = false;
  if (rc || (rc = enq_residual(b, st, true)) || (rc = enq_readback(b, st))) return rc;
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  chk = check(b);
  b->last_initial = chk.worst;
  std::vector<int> used;
  if ((rc = refine_adaptive(b, dt, st, kMaxPasses, used, chk))) return rc;
  if (!learned_on(b)) {  // the plain schedule, for the gate of a later guess
    b->have_plain = true;
    b->plain_schedule = used;
    b->plain_dt = dt;
    std::memcpy(b->plain_c, c, sizeof(b->plain_c));
  } else if (deciding) {
    // the gate: the inner steps and passes the guess saved against the last
    // plain schedule of the same step width and coefficients, at the
    // measured time of a Chebyshev launch and of a residual launch, against
    // the guess's measured cost (and a quarter more for its history
    // updates); no plain schedule to compare with keeps the guess on
    bool same = b->have_plain && b->plain_dt == dt;
    for (int k = 0; k < 8 && same; ++k) same = b->plain_c[k] == c[k];
    b->learn_gate = 1;
    if (same && b->guess_ms >= 0.0) {
      const double cheb = b->cand_ms[2 * b->variant + b->order];
      const double resc = b->fp64_ms[b->fp64] > 0.0 ? b->fp64_ms[b->fp64] : cheb;
      const double steps = (double)(sum(b->plain_schedule) - sum(used));
      const double passes = (double)b->plain_schedule.size() - (double)used.size();
      b->guess_saving_ms = std::max(0.0, steps) * std::max(0.0, cheb) + std::max(0.0, passes) * resc;
      if (b->guess_saving_ms < 1.25 * b->guess_ms) b->learn_gate = 0;
    }
  }
  b->schedule = used;
  b->have_key = true;
  b->key_depth = depth_of(b);
  b->key_dt = dt;
  std::memcpy(b->key_c, c, sizeof(b->key_c));
  b->gen++;
  return NRQ_OK;
}

// after a scheduled step: verify, refine the fields that missed the tolerance
// (and lengthen the schedule), then hand the results to the fields
int finish_step(nrq_cn_batch *b, double dt, cudaStream_t st, Check &chk, bool *schedule_changed) {
  chk = check(b);
  *schedule_changed = false;
  if (!chk.conv && !chk.nonfin && !chk.badbounds && !chk.timeout) {
    NRQ_CUDA_TRY(b->ctx, cudaMemcpyAsync(b->h_bounds, b->bounds, sizeof(double) * 4 * b->masses.size(),
                                         cudaMemcpyDeviceToHost, st));
    NRQ_CUDA_TRY(b->ctx, cudaStreamSynchronize(st));
    std::vector<int> used;
    int rc = refine_adaptive(b, dt, st, kMaxPasses, used, chk);
    if (rc) return rc;
    if (!used.empty() && (int)(b->schedule.size() + 1) <= kMaxPasses) {
      b->schedule.push_back(*std::max_element(used.begin(), used.end()));
      b->gen++;
      *schedule_changed = true;
    }
  }
  return NRQ_OK;
}

int conclude(nrq_cn_batch *b, const Check &chk, int64_t inner, int64_t passes) {
  // results: the iterate becomes the field, the old field the next work
  // buffer; a learned step leaves the new history in the field
  const bool keep = (learned_on(b) || hist_on(b)) && chk.conv && !chk.nonfin && !chk.badbounds && !chk.timeout;
  for (int i = 0; i < b->nf; ++i) {
    std::swap(b->fields[i]->P, b->xbuf[i]);
    if (keep) hist_push(b->fields[i]);
    else b->fields[i]->hist_count = 0;
  }
  b->last_inner = inner;
  b->last_passes = passes;
  b->last_matvecs = 1 + (passes + 1) + inner;
  b->last_maxrel = chk.worst;
  b->last_conv = chk.conv;
  if (chk.timeout) {
    b->ctx->last_error = std::string("batch stencil: a bounded pipeline wait expired (") +
                         (b->h_err[1] / 16 == 7 ? "k_batch_mv5" : "k_cheb5f") + ", load " +
                         std::to_string(b->h_err[2]) + ", CTA " + std::to_string(b->h_err[3]) + ")";
    cudaMemsetAsync(b->err, 0, sizeof(int) * 16, b->ctx->stream);
    b->h_err[0] = 0;
    return NRQ_ERR_TIMEOUT;
  }
  if (chk.badbounds) {
    b->ctx->last_error = "batch: invalid spectral bounds";
    return NRQ_ERR_NONFINITE;
  }
  if (chk.nonfin) {
    b->ctx->last_error = "batch CN solve: non-finite residual";
    return NRQ_ERR_NONFINITE;
  }
  return chk.conv ? NRQ_OK : NRQ_ERR_NOT_CONVERGED;
}

void fill_stats(const nrq_cn_batch *b, nrq_cn_stats *s) {
  if (!s) return;
  s->iterations = b->last_inner;
  s->matvecs = b->last_matvecs;
  s->vector_streams = 1 + 3 * (b->last_passes + 1) + 3 * b->last_passes;
  s->max_rel_residual = b->last_maxrel;
  s->converged = b->last_conv ? 1 : 0;
  s->initial_rel_residual = b->last_initial;
}


int capture(nrq_ctx *ctx, cudaStream_t st, cudaGraph_t *graph, int (*body)(void *), void *arg) {
  const bool prof = ctx->prof;
  ctx->prof = false;  // no event records inside a capture
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    ctx->prof = prof;
    ctx->last_error = std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e);
    return NRQ_ERR_CUDA;
  }
  int rc = body(arg);
  e = cudaStreamEndCapture(st, graph);
  ctx->prof = prof;
  if (rc) {
    if (e == cudaSuccess && *graph) cudaGraphDestroy(*graph);
    return rc;
  }
  if (e != cudaSuccess) {
    ctx->last_error = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
    return NRQ_ERR_CUDA;
  }
  return NRQ_OK;
}

struct StepArgs {
  nrq_cn_batch *b;
  const nrq_gauge *g;
  const double *c;
  double dt;
  bool leapfrog;
};
int step_body(void *p) {
  StepArgs *a = (StepArgs *)p;
  int rc = enq_scheduled(a->b, a->g, a->c, a->dt, a->b->ctx->stream);
  if (!rc && a->leapfrog) rc = nrq_gauge_update((nrq_gauge *)a->g, a->dt);
  return rc;
}

}  // namespace

// ============================================================ batch C ABI
extern "C" int nrq_cn_batch_create(nrq_ctx *ctx, int nfields, nrq_heavy *const *fields, const double *masses,
                                   double tol, nrq_cn_batch **out) {
  if (!ctx || !fields || !masses || !out || nfields <= 0 || !(tol > 0.0)) return NRQ_ERR_BAD_ARG;
  // per-field grid dimension (<= 65535) and flattened (site block, field) grids (< 2^31)
  if (nfields > 65535 || ((ctx->lat.V + 31) / 32) * (int64_t)nfields >= (int64_t)1 << 31) {
    ctx->last_error = "batch: too many fields for this lattice";
    return NRQ_ERR_CAPACITY;
  }
  for (int i = 0; i < nfields; ++i) {
    if (!fields[i] || fields[i]->ctx != ctx || masses[i] == 0.0 || !std::isfinite(masses[i])) return NRQ_ERR_BAD_ARG;
    for (int j = 0; j < i; ++j)
      if (fields[j] == fields[i]) return NRQ_ERR_BAD_ARG;
  }
  int rc = set_device(ctx);
  if (rc) return rc;
  nrq_cn_batch *b = new (std::nothrow) nrq_cn_batch();
  if (!b) return NRQ_ERR_OOM;
  b->ctx = ctx;
  b->nf = nfields;
  b->tol = tol;
  // group by mass, first-appearance order of the masses
  for (int i = 0; i < nfields; ++i)
    if (std::find(b->masses.begin(), b->masses.end(), masses[i]) == b->masses.end()) b->masses.push_back(masses[i]);
  b->group_size.assign(b->masses.size(), 0);
  for (size_t k = 0; k < b->masses.size(); ++k)
    for (int i = 0; i < nfields; ++i)
      if (masses[i] == b->masses[k]) {
        b->fields.push_back(fields[i]);
        b->user.push_back(i);
        b->mass_of.push_back((int)k);
        b->group_size[k]++;
      }
  const int64_t V = ctx->lat.V;
  const int64_t P = 72 * V;
  b->nsb = (V + 31) / 32;
  const int64_t nbb = (V + 255) / 256;
  auto fail = [&](cudaError_t e) {
    ctx->last_error = std::string("batch allocation: ") + cudaGetErrorString(e);
    nrq_cn_batch_destroy(b);
    return e == cudaErrorMemoryAllocation ? NRQ_ERR_OOM : NRQ_ERR_CUDA;
  };
  cudaError_t e = cudaSuccess;
#define NRQ_B_ALLOC(ptr, bytes)                       \
  if ((e = cudaMalloc(&(ptr), (bytes))) != cudaSuccess) { \
    (ptr) = nullptr;                                  \
    return fail(e);                                   \
  }
  NRQ_B_ALLOC(b->U64, sizeof(double2) * 27 * V);
  NRQ_B_ALLOC(b->Dsum, sizeof(double2) * 9 * V);
  NRQ_B_ALLOC(b->Bsum, sizeof(double) * 9 * V);
  NRQ_B_ALLOC(b->DE, sizeof(double2) * 54 * V);
  NRQ_B_ALLOC(b->U32, sizeof(float2) * 27 * V);
  NRQ_B_ALLOC(b->DE32, sizeof(float2) * 54 * V);
  NRQ_B_ALLOC(b->D32, sizeof(float2) * 9 * V);
  NRQ_B_ALLOC(b->B32, sizeof(float) * 9 * V);
  NRQ_B_ALLOC(b->bpart, sizeof(double) * 4 * nbb);
  NRQ_B_ALLOC(b->bounds, sizeof(double) * 4 * b->masses.size());
  NRQ_B_ALLOC(b->b_all, sizeof(double2) * P * nfields);
  NRQ_B_ALLOC(b->r32_all, sizeof(float2) * P * nfields);
  NRQ_B_ALLOC(b->dA_all, sizeof(float2) * P * nfields);
  NRQ_B_ALLOC(b->dB_all, sizeof(float2) * P * nfields);
  NRQ_B_ALLOC(b->e32_all, sizeof(float2) * P * nfields);
  NRQ_B_ALLOC(b->part_all, sizeof(double) * b->nsb * nrq::CN_COLS * 2 * nfields);
  NRQ_B_ALLOC(b->scal_all, sizeof(double) * kFieldScal * nfields);
  NRQ_B_ALLOC(b->pstate, sizeof(double) * 2);
  NRQ_B_ALLOC(b->flags, sizeof(int) * nfields);
  NRQ_B_ALLOC(b->d_tab, sizeof(nrq::BatchField) * nfields);
  NRQ_B_ALLOC(b->err, sizeof(int) * 16);
  if (nrq::cheb5f_applicable(ctx->lat))
    NRQ_B_ALLOC(b->W5f, sizeof(float2) * nrq::cn_mv5_block_entries(V) * b->masses.size());
  if (nrq::batch_mv5_applicable(ctx->lat)) {
    NRQ_B_ALLOC(b->W5, sizeof(double2) * nrq::cn_mv5_block_entries(V) * b->masses.size());
    NRQ_B_ALLOC(b->d_fmaps, sizeof(nrq::CnBatchMaps) * nfields);
  }
  b->xbuf.assign(nfields, nullptr);
  for (int i = 0; i < nfields; ++i) NRQ_B_ALLOC(b->xbuf[i], sizeof(double2) * P);
#undef NRQ_B_ALLOC
  if ((e = cudaMallocHost(&b->h_tab, sizeof(nrq::BatchField) * nfields)) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&b->h_scal, sizeof(double) * kFieldScal * nfields)) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&b->h_flags, sizeof(int) * nfields)) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&b->h_bounds, sizeof(double) * 4 * b->masses.size())) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&b->h_err, sizeof(int) * 16)) != cudaSuccess) return fail(e);
  if (b->d_fmaps && (e = cudaMallocHost(&b->h_fmaps, sizeof(nrq::CnBatchMaps) * nfields)) != cudaSuccess)
    return fail(e);
  std::memset(b->h_err, 0, sizeof(int) * 16);
  if ((e = cudaMemsetAsync(b->err, 0, sizeof(int) * 16, ctx->stream)) != cudaSuccess) return fail(e);
  // defined contents for the FP32 vectors and flags the tuner's first launches read
  for (float2 *p : {b->r32_all, b->dA_all, b->dB_all, b->e32_all})
    if ((e = cudaMemsetAsync(p, 0, sizeof(float2) * P * nfields, ctx->stream)) != cudaSuccess) return fail(e);
  if ((e = cudaMemsetAsync(b->scal_all, 0, sizeof(double) * kFieldScal * nfields, ctx->stream)) != cudaSuccess)
    return fail(e);
  {
    const double p0[2] = {-1.0, 0.0};  // no ratio measured, no scheduled step taken
    if ((e = cudaMemcpy(b->pstate, p0, sizeof(p0), cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
  }
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(e);
  *out = b;
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_destroy(nrq_cn_batch *b) {
  if (!b) return NRQ_ERR_NOT_INITIALISED;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  free_graph(b->exec);
  for (void *p : {(void *)b->U64, (void *)b->Dsum, (void *)b->Bsum, (void *)b->DE, (void *)b->U32, (void *)b->DE32,
                  (void *)b->D32, (void *)b->B32, (void *)b->bpart, (void *)b->bounds, (void *)b->b_all,
                  (void *)b->r32_all, (void *)b->dA_all, (void *)b->dB_all, (void *)b->e32_all, (void *)b->part_all,
                  (void *)b->scal_all, (void *)b->flags, (void *)b->d_tab, (void *)b->lgf, (void *)b->lfeat,
                  (void *)b->lomega, (void *)b->W5f, (void *)b->err, (void *)b->W5, (void *)b->d_fmaps,
                  (void *)b->pstate})
    if (p) cudaFree(p);
  for (double2 *p : b->xbuf)
    if (p) cudaFree(p);
  for (void *p : {(void *)b->h_tab, (void *)b->h_scal, (void *)b->h_flags, (void *)b->h_bounds, (void *)b->h_err,
                  (void *)b->h_fmaps})
    if (p) cudaFreeHost(p);
  delete b;
  return NRQ_OK;
}

namespace {
int check_inputs(nrq_cn_batch *b, const nrq_gauge *g, const double c[8]) {
  if (!b || !g || !c) return NRQ_ERR_BAD_ARG;
  if (g->ctx != b->ctx) return NRQ_ERR_BAD_ARG;
  if (c[1] != 0.0 || c[3] != 0.0 || c[5] != 0.0 || c[7] != 0.0) {
    b->ctx->last_error = "batch: Wilson coefficients must be real";
    return NRQ_ERR_BAD_ARG;
  }
  for (int i = 0; i < b->nf; ++i)
    if (b->fields[i]->ctx != b->ctx || !b->fields[i]->P) return NRQ_ERR_BAD_ARG;
  return NRQ_OK;
}
// ensemble members step inside one graph: their leapfrog must be the FP64 one
int check_member_gauge(nrq_cn_batch *b, const nrq_gauge *g) {
  if (g->prec != 0) {
    b->ctx->last_error = "ensemble: gauge fields in the FP32-link precision form are not supported";
    return NRQ_ERR_BAD_ARG;
  }
  return NRQ_OK;
}

// one batch update (CN only), eager or as the batch's own graph
int batch_update(nrq_cn_batch *b, const nrq_gauge *g, const double c[8], double dt, bool use_graph) {
  nrq_ctx *ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  int rc = ensure_batch_hist(b);
  if (rc) return rc;
  fill_table(b, c, dt);
  rc = upload_table(b, st);
  if (rc) return rc;
  Check chk;
  if (!same_key(b, c, dt)) {
    if ((rc = update_calibrate(b, g, c, dt, st, chk))) return rc;
    return conclude(b, chk, sum(b->schedule), (int64_t)b->schedule.size());
  }
  if (use_graph) {
    if (b->exec && (b->exec_gen != b->gen || b->exec_g != g)) free_graph(b->exec);
    if (!b->exec) {
      cudaGraph_t graph = nullptr;
      StepArgs a{b, g, c, dt, false};
      if ((rc = capture(ctx, st, &graph, step_body, &a))) return rc;
      cudaError_t e = cudaGraphInstantiate(&b->exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        b->exec = nullptr;
        ctx->last_error = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
        return NRQ_ERR_CUDA;
      }
      b->exec_gen = b->gen;
      b->exec_g = g;
    }
    NRQ_CUDA_TRY(ctx, cudaGraphLaunch(b->exec, st));
  } else {
    if ((rc = enq_scheduled(b, g, c, dt, st))) return rc;
  }
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (learned_on(b) && (rc = nrqh::learned_check(b->learn))) return rc;
  b->last_initial = 0.0;  // not read back by scheduled steps
  const int64_t planned = sum(b->schedule), planned_passes = (int64_t)b->schedule.size();
  bool changed = false;
  if ((rc = finish_step(b, dt, st, chk, &changed))) return rc;
  int64_t inner = planned, passes = planned_passes;
  if (changed) {  // the refinement ran one extra pass per appended step count (at least)
    inner = sum(b->schedule);
    passes = (int64_t)b->schedule.size();
  }
  return conclude(b, chk, inner, passes);
}
}  // namespace

extern "C" int nrq_cn_batch_update(nrq_cn_batch *b, const nrq_gauge *g, const double c[8], double dt, int use_graph,
                                   nrq_cn_stats *stats) {
  int rc = check_inputs(b, g, c);
  if (rc) return rc;
  if ((rc = set_device(b->ctx)) || (rc = nrqh::gauge_sync64(g))) return rc;
  rc = batch_update(b, g, c, dt, use_graph != 0);
  fill_stats(b, stats);
  return rc;
}

extern "C" int nrq_cn_batch_attach_learned(nrq_cn_batch *b, nrq_learn *net) {
  if (!b || (net && nrqh::learned_ctx(net) != b->ctx)) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = b->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  if (net) {
    const int64_t V = ctx->lat.V, ns = 2 * V * b->nf;
    if (!b->lgf) NRQ_CUDA_TRY(ctx, cudaMalloc(&b->lgf, sizeof(float4) * V));
    if (!b->lfeat) NRQ_CUDA_TRY(ctx, cudaMalloc(&b->lfeat, sizeof(float) * 16 * ns));
    if (!b->lomega) NRQ_CUDA_TRY(ctx, cudaMalloc(&b->lomega, sizeof(float4) * 2 * ns));
    for (nrq_heavy *h : b->fields)
      if ((rc = nrqh::ensure_hist(h))) return rc;
  }
  b->learn = net;
  b->learn_gate = -1;
  b->guess_ms = b->guess_saving_ms = -1.0;
  b->have_key = false;  // recalibrate (and recapture) with or without the guess
  b->gen++;
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_residuals(const nrq_cn_batch *b, double *rel) {
  if (!b || !rel) return NRQ_ERR_BAD_ARG;
  for (int i = 0; i < b->nf; ++i) {
    const double *s = b->h_scal + (size_t)i * kFieldScal;
    double w = 0.0;
    for (int k = 0; k < nrq::CN_COLS; ++k) {
      const double *sc = s + k * nrq::SC_STRIDE;
      if (sc[nrq::SC_BB] > 0) w = std::max(w, std::sqrt(sc[nrq::SC_RR] / sc[nrq::SC_BB]));
    }
    rel[b->user[i]] = w;
  }
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_info(const nrq_cn_batch *b, int *variant, int *order, double candidate_ms[8],
                                 int *npasses, int steps[16]) {
  if (!b) return NRQ_ERR_BAD_ARG;
  if (variant) *variant = b->variant;
  if (order) *order = b->order;
  if (candidate_ms)
    for (int k = 0; k < 2 * nrq::BATCH_CHEB_VARIANTS; ++k) candidate_ms[k] = b->cand_ms[k];
  if (npasses) *npasses = (int)b->schedule.size();
  if (steps)
    for (int k = 0; k < 16; ++k) steps[k] = k < (int)b->schedule.size() ? b->schedule[k] : 0;
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_learned_info(const nrq_cn_batch *b, int *gate, double *guess_ms, double *saving_ms) {
  if (!b) return NRQ_ERR_BAD_ARG;
  if (gate) *gate = b->learn ? b->learn_gate : -2;
  if (guess_ms) *guess_ms = b->guess_ms;
  if (saving_ms) *saving_ms = b->guess_saving_ms;
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_set_history(nrq_cn_batch *b, int on) {
  if (!b || on < 0 || on > 1) return NRQ_ERR_BAD_ARG;
  if (b->history != (on != 0)) {
    b->history = on != 0;
    b->have_key = false;  // recalibrate (and recapture) with the other start
    b->gen++;
  }
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_prediction_info(const nrq_cn_batch *b, double *ratio, int64_t *steps) {
  if (!b) return NRQ_ERR_BAD_ARG;
  int rc = set_device(b->ctx);
  if (rc) return rc;
  double p[2] = {-1.0, 0.0};
  NRQ_CUDA_TRY(b->ctx, cudaMemcpyAsync(p, b->pstate, sizeof(p), cudaMemcpyDeviceToHost, b->ctx->stream));
  NRQ_CUDA_TRY(b->ctx, cudaStreamSynchronize(b->ctx->stream));
  if (ratio) *ratio = p[0];
  if (steps) *steps = (int64_t)p[1];
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_fp64_info(const nrq_cn_batch *b, int *which, double ms[2]) {
  if (!b) return NRQ_ERR_BAD_ARG;
  if (which) *which = b->fp64;
  if (ms)
    for (int k = 0; k < 2; ++k) ms[k] = b->fp64_ms[k];
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_set_fp64(nrq_cn_batch *b, int which) {
  if (!b || which < 0 || which > 1) return NRQ_ERR_BAD_ARG;
  if (which == 1 && !b->W5) {
    b->ctx->last_error = "batch: the FP64 block stencil needs an even V of at least 34 sites";
    return NRQ_ERR_BAD_ARG;
  }
  b->fp64 = which;
  b->have_key = false;
  b->gen++;
  return NRQ_OK;
}

extern "C" int nrq_cn_batch_set_variant(nrq_cn_batch *b, int variant, int order) {
  if (!b || variant < -1 || variant >= nrq::BATCH_CHEB_VARIANTS || order < 0 || order > 1) return NRQ_ERR_BAD_ARG;
  if (variant == 2) {
    for (int n : b->group_size)
      if (n % 2) {
        b->ctx->last_error = "batch: two-field tiles need an even number of fields per mass";
        return NRQ_ERR_BAD_ARG;
      }
  }
  if (variant == 3 && !b->W5f) {
    b->ctx->last_error = "batch: the FP32 block step needs V a multiple of 4, V >= 36, nx even";
    return NRQ_ERR_BAD_ARG;
  }
  if (variant < 0) {
    b->tuned = false;
  } else {
    b->variant = variant;
    b->order = order;
    if (b->fp64 < 0 || !b->tuned) b->fp64 = b->W5 ? 1 : 0;  // untimed: the FMA stencil where it applies
    b->tuned = true;
  }
  b->have_key = false;  // recalibrate the schedule with the new kernel
  b->gen++;
  return NRQ_OK;
}

// ============================================================ ensemble C ABI
extern "C" int nrq_ensemble_create(int n, nrq_cn_batch *const *batches, nrq_gauge *const *gauges,
                                   nrq_ensemble **out) {
  if (n <= 0 || !batches || !gauges || !out) return NRQ_ERR_BAD_ARG;
  for (int i = 0; i < n; ++i) {
    if (!batches[i] || !gauges[i] || gauges[i]->ctx != batches[i]->ctx) return NRQ_ERR_BAD_ARG;
    if (batches[i]->ctx->device != batches[0]->ctx->device) return NRQ_ERR_BAD_ARG;
    for (int j = 0; j < i; ++j)
      if (batches[j] == batches[i] || gauges[j] == gauges[i]) return NRQ_ERR_BAD_ARG;
  }
  nrq_ensemble *e = new (std::nothrow) nrq_ensemble();
  if (!e) return NRQ_ERR_OOM;
  e->batches.assign(batches, batches + n);
  e->gauges.assign(gauges, gauges + n);
  *out = e;
  return NRQ_OK;
}

extern "C" int nrq_ensemble_destroy(nrq_ensemble *e) {
  // touches no member: an executable graph still in flight is released by
  // the driver when it completes (and every step synchronises before return)
  if (!e) return NRQ_ERR_NOT_INITIALISED;
  free_graph(e->exec);
  delete e;
  return NRQ_OK;
}

extern "C" int nrq_ensemble_step(nrq_ensemble *e, const double c[8], double dt, int use_graph,
                                 nrq_cn_stats *stats) {
  if (!e || !c) return NRQ_ERR_BAD_ARG;
  const int n = (int)e->batches.size();
  for (int i = 0; i < n; ++i) {
    int rc = check_inputs(e->batches[i], e->gauges[i], c);
    if (!rc) rc = check_member_gauge(e->batches[i], e->gauges[i]);
    if (rc) return rc;
  }
  nrq_ctx *ctx0 = e->batches[0]->ctx;
  int rc = set_device(ctx0);
  if (rc) return rc;
  bool calibrated = true;
  for (nrq_cn_batch *b : e->batches) calibrated = calibrated && same_key(b, c, dt);
  int status = NRQ_OK;
  auto note = [&](int r) {
    if (r == NRQ_ERR_NOT_CONVERGED) {
      if (status == NRQ_OK) status = r;
    } else if (r) {
      status = r;
    }
  };
  if (!calibrated || !use_graph) {
    // member by member, eager (calibrating where needed), then the leapfrog
    for (int i = 0; i < n && (status == NRQ_OK || status == NRQ_ERR_NOT_CONVERGED); ++i) {
      note(batch_update(e->batches[i], e->gauges[i], c, dt, false));
      if (status == NRQ_OK || status == NRQ_ERR_NOT_CONVERGED) note(nrq_gauge_update(e->gauges[i], dt));
    }
  } else {
    cudaStream_t st0 = ctx0->stream;
    for (nrq_cn_batch *b : e->batches) {
      if ((rc = ensure_batch_hist(b))) return rc;
      fill_table(b, c, dt);
      if ((rc = upload_table(b, st0))) return rc;
    }
    bool stale = !e->exec || e->exec_gen.size() != (size_t)n;
    for (int i = 0; !stale && i < n; ++i) stale = e->exec_gen[i] != e->batches[i]->gen;
    if (stale) free_graph(e->exec);
    if (!e->exec) {
      cudaGraph_t master = nullptr;
      NRQ_CUDA_TRY(ctx0, cudaGraphCreate(&master, 0));
      // members run as concurrent branches, except where a member uses the
      // persistent block stencils: those size their grids to every SM and
      // hold most of an SM's shared memory, so concurrent members only
      // fragment the GPU, and the members' steps are chained instead
      bool chain = false;
      for (nrq_cn_batch *b : e->batches) chain = chain || b->variant == 3 || b->fp64 == 1;
      cudaGraphNode_t prev = nullptr;
      for (int i = 0; i < n; ++i) {
        cudaGraph_t child = nullptr;
        StepArgs a{e->batches[i], e->gauges[i], c, dt, true};
        if ((rc = capture(e->batches[i]->ctx, e->batches[i]->ctx->stream, &child, step_body, &a))) {
          cudaGraphDestroy(master);
          if (e->batches[i]->ctx != ctx0) ctx0->last_error = e->batches[i]->ctx->last_error;
          return rc;
        }
        cudaGraphNode_t node;
        cudaError_t er = cudaGraphAddChildGraphNode(&node, master, chain && prev ? &prev : nullptr,
                                                    chain && prev ? 1 : 0, child);
        cudaGraphDestroy(child);
        prev = node;
        if (er != cudaSuccess) {
          cudaGraphDestroy(master);
          ctx0->last_error = std::string("cudaGraphAddChildGraphNode: ") + cudaGetErrorString(er);
          return NRQ_ERR_CUDA;
        }
      }
      cudaError_t er = cudaGraphInstantiate(&e->exec, master, 0);
      cudaGraphDestroy(master);
      if (er != cudaSuccess) {
        e->exec = nullptr;
        ctx0->last_error = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(er);
        return NRQ_ERR_CUDA;
      }
      e->exec_gen.clear();
      for (nrq_cn_batch *b : e->batches) e->exec_gen.push_back(b->gen);
    }
    NRQ_CUDA_TRY(ctx0, cudaGraphLaunch(e->exec, st0));
    NRQ_CUDA_TRY(ctx0, cudaStreamSynchronize(st0));
    for (nrq_cn_batch *b : e->batches)
      if (learned_on(b) && (rc = nrqh::learned_check(b->learn))) return rc;
    for (nrq_cn_batch *b : e->batches) {
      Check chk;
      bool changed = false;
      const int64_t inner = sum(b->schedule), passes = (int64_t)b->schedule.size();
      rc = finish_step(b, dt, b->ctx->stream, chk, &changed);
      if (rc) return rc;
      note(conclude(b, chk, changed ? sum(b->schedule) : inner, changed ? (int64_t)b->schedule.size() : passes));
    }
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->converged = 1;
    for (nrq_cn_batch *b : e->batches) {
      stats->iterations = std::max<int64_t>(stats->iterations, b->last_inner);
      stats->matvecs += b->last_matvecs * b->nf;
      stats->vector_streams += (1 + 3 * (b->last_passes + 1) + 3 * b->last_passes) * b->nf;
      stats->max_rel_residual = std::max(stats->max_rel_residual, b->last_maxrel);
      stats->initial_rel_residual = std::max(stats->initial_rel_residual, b->last_initial);
      stats->converged = stats->converged && b->last_conv;
    }
  }
  return status;
}
