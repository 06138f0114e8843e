// Host-side handle definitions behind the C ABI (include/nrqcd_b200.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <complex>
#include <string>
#include <vector>

#include "nrq_kernels.cuh"

struct nrq_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  nrq::Lat lat{};
  int64_t n[3] = {0, 0, 0};
  double a[4] = {0, 0, 0, 0};
  // reduction scratch (device + pinned host mirror)
  double *d_red = nullptr;     // partial sums, red_cap doubles
  int64_t red_cap = 0;
  double *d_res = nullptr;     // final results, 64 doubles
  double *h_res = nullptr;     // pinned, 64 doubles
  // staging buffer for layout transposes (device), grown on demand
  void *d_stage = nullptr;
  size_t stage_bytes = 0;
  // state of a Gauss projection (nrq::GaussProjState), allocated on first use
  void *d_proj = nullptr;
  // gluon observables: cuFFT plans over 9 and 48 complex planes and their
  // device buffer, created on first use and kept (as the reference keeps its
  // FFT descriptor, src/xpfft.f90:129-139); cufftHandle is an int
  int fft9 = 0, fft48 = 0;
  bool fft9_ok = false, fft48_ok = false;
  void *d_gluon = nullptr;
  size_t gluon_bytes = 0;
  std::string last_error;
  int sm_count = 148;
  // opt-in per-class kernel timing (events recorded on `stream`)
  bool prof = false;
  struct ProfRec {
    int cls;
    double bytes;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof_recs;
  std::vector<cudaEvent_t> prof_pool;
};

// RAII helper: records a start event on construction and an end event plus
// the algorithmic byte count on destruction when profiling is on.
struct ProfScope {
  nrq_ctx *ctx;
  int cls;
  double bytes;
  cudaEvent_t a = nullptr;
  ProfScope(nrq_ctx *c, int k, double by) : ctx(c), cls(k), bytes(by) {
    if (!ctx->prof) return;
    a = take();
    cudaEventRecord(a, ctx->stream);
  }
  ~ProfScope() {
    if (!ctx->prof || !a) return;
    cudaEvent_t b = take();
    cudaEventRecord(b, ctx->stream);
    ctx->prof_recs.push_back({cls, bytes, a, b});
  }
  cudaEvent_t take() {
    if (!ctx->prof_pool.empty()) {
      cudaEvent_t e = ctx->prof_pool.back();
      ctx->prof_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
};

struct nrq_gauge {
  nrq_ctx *ctx = nullptr;
  double2 *U = nullptr;  // 27 planes of V complex: (dir*9 + row*3 + col)
  double *E = nullptr;   // 24 planes of V reals  : (dir*8 + a)
  // precision form of the leapfrog (prec 1): the links evolve in U32 (FP32,
  // same planes); U is their FP64 view, refreshed on demand (stale64) and
  // replaced by the FP64 reunitarised links every reunit_every steps
  float2 *U32 = nullptr;
  int prec = 0;
  int reunit_every = 10;
  int since_reunit = 0;
  bool stale64 = false;
};

struct nrq_heavy {
  nrq_ctx *ctx = nullptr;
  // 72 planes of V complex: (species*36 + col*6 + row); species 0 quark, 1 antiquark
  double2 *P = nullptr;
  // history of the field's steps (FP32, 72 planes each): what the start
  // 2 RHS - psi missed, t = x - (2 RHS - psi), in the last steps, for the
  // plain solve's extrapolated start and the learned guess.  A ring of
  // hist_cap slots (2, grown to the plain solve's history depth on demand);
  // hist_count vectors are valid, the newest in slot hist_head.
  static constexpr int kMaxHist = 4;
  float2 *hist[kMaxHist] = {nullptr, nullptr, nullptr, nullptr};
  int hist_cap = 2;
  int hist_count = 0;
  int hist_head = 0;
};

// the k-th newest history vector (k = 1, 2, ...), null where not valid
inline const float2 *hist_v(const nrq_heavy *h, int k) {
  return h->hist_count >= k ? h->hist[(h->hist_head - (k - 1) + h->hist_cap) % h->hist_cap] : nullptr;
}
inline const float2 *hist_v1(const nrq_heavy *h) { return hist_v(h, 1); }
inline const float2 *hist_v2(const nrq_heavy *h) { return hist_v(h, 2); }
// slot the next history vector goes to (the oldest one)
inline float2 *hist_next(nrq_heavy *h) { return h->hist[(h->hist_head + 1) % h->hist_cap]; }
inline void hist_push(nrq_heavy *h) {
  h->hist_head = (h->hist_head + 1) % h->hist_cap;
  h->hist_count = h->hist_count < h->hist_cap ? h->hist_count + 1 : h->hist_cap;
}

struct nrq_learn;

struct nrq_cn_stats_internal;
// about two seconds at 2 GHz: the default bound of a pipeline wait
constexpr long long nrq_wait_cycles_default = 4000000000LL;

struct nrq_cn {
  nrq_ctx *ctx = nullptr;
  double mass = 1.0;
  double c[8] = {1, 0, 1, 0, 1, 0, 1, 0};
  double stepwidth = 1.0;
  double tol = 1e-12;
  int64_t maxits = 10000;
  int form = 0;
  nrq_learn *learn = nullptr;  // learned initial guess (form 2)
  // per-step derived gauge data
  double2 *Dsum = nullptr;  // 9 planes
  double *Bsum = nullptr;   // 9 planes
  double2 *DE = nullptr;    // 54 planes: ((i*2 + perm)*9 + r*3 + c)
  // Krylov vectors, 72 planes each
  double2 *b = nullptr, *x = nullptr, *r = nullptr, *rh = nullptr, *p = nullptr, *v = nullptr,
          *t = nullptr, *s = nullptr;
  // FP64 stencil (NRQ_STENCIL_*): register-tiled, TMA-staged, tensor-core
  // or FMA on cached blocks.
  // Chosen by timing the applicable ones on the first update (tune_ms, per
  // launch) unless forced; tma_ok: tensor maps can describe the lattice.
  // last_stencil: the stencil of the latest launch (its partial-row count).
  int stencil = 0;
  int forced_stencil = -1;
  int last_stencil = 0;
  bool tma_ok = false;
  bool stencil_tuned = false;
  double tune_ms[4] = {-1.0, -1.0, -1.0, -1.0};
  // plain form: start from 2b - psi + 2 t1 - t2 with the field's history of
  // corrections (FP32); on by default
  bool history_guess = true;
  int history_depth = 4;  // history vectors the start extrapolates from (1-4)
  // plain form: confirm every converged solve with the true residual (a
  // residual pass), or (false, the default) accept the recursive residual
  // where it meets the tolerance with a margin of four times the largest
  // recursive-to-true gap measured on this solver's confirmed solves (gap_rel,
  // relative to ||b||; -1 before the first), confirming again after
  // kReconfirm unconfirmed solves; last_true: the last update's reported
  // residual is the true one
  static constexpr int kReconfirm = 16;
  bool confirm_always = false;
  bool last_true = true;
  double gap_rel = -1.0;
  int since_confirm = 0;
  // precision forms: the largest ratio of the true residual to the
  // Chebyshev prediction (previous residual / the pass's guaranteed gain)
  // measured on confirmed passes (-1 before the first), and the updates
  // accepted on the prediction since the last confirmation
  double cheb_ratio = -1.0;
  int cheb_unconfirmed = 0;
  // plain form on the FMA stencil: the x, r and p updates of an iteration in
  // one pass, beta from the rh.t the t = A^H s launch reduces (false: the
  // x, r update and the p update as two passes)
  bool merged_update = true;
  // tensor-core stencil: forward 6x6 blocks (6 per site: direction x
  // species, 36 complex each) built for the coefficients w_coef from the
  // current gauge field (w_valid cleared by every preparation)
  double2 *Wblk = nullptr;
  bool w_valid = false;
  nrq::CnCoef w_coef{};
  // FP64 FMA stencil: the same blocks as 216 planes
  double2 *Wblk5 = nullptr;
  bool w5_valid = false;
  nrq::CnCoef w5_coef{};
  // the FP32 Chebyshev step of the precision forms: the same blocks rounded
  // to FP32, and which step kernel runs (-1: k_cheb5f where it applies, else
  // k_cheb32; NRQ_CHEB_* forces one); last_cheb: the one the last update ran
  float2 *Wblk5f = nullptr;
  bool w5f_valid = false;
  nrq::CnCoef w5f_coef{};
  int cheb_stencil = -1;
  int last_cheb = -1;
  // the timed choice between the two steps (per-launch ms; -1 not timed)
  bool cheb_tuned = false;
  int cheb_choice = -1;
  double cheb_ms[2] = {-1.0, -1.0};
  // bound of the FMA stencil's pipeline waits (clock cycles) and, for the
  // test of the timeout path, the load its producer stops before (-1: none)
  long long wait_cycles = nrq_wait_cycles_default;
  int stall_load = -1;
  // precision form (form 1): FP32 copies of the per-step matrices and the
  // FP32 Chebyshev vectors; spectral bounds of the hermitian part
  float2 *U32 = nullptr, *DE32 = nullptr, *D32 = nullptr;
  float *B32 = nullptr;
  float2 *r32 = nullptr, *dA32 = nullptr, *dB32 = nullptr, *e32 = nullptr;
  double *bounds = nullptr;    // partial blocks, then 4 final values
  double *h_bounds = nullptr;  // pinned
  int64_t last_inner = 0;      // FP32 Chebyshev steps of the last update
  int64_t last_outer = 0;      // FP64 refinement passes of the last update
  double last_lo[2] = {0, 0}, last_hi[2] = {0, 0};
  double *scal = nullptr;     // device scalars per column
  double *h_scal = nullptr;   // pinned mirror
  int *d_flags = nullptr;
  int64_t nblocks = 0;
  double *partials = nullptr;  // nblocks * 12 * 4
  unsigned int *counter = nullptr;
  // statistics of the last update
  int64_t last_iterations = 0;
  int64_t last_matvecs = 0;
  int64_t last_vecstreams = 0;
};

// error helpers
#define NRQ_CUDA_TRY(ctx, expr)                                              \
  do {                                                                       \
    cudaError_t _e = (expr);                                                 \
    if (_e != cudaSuccess) {                                                 \
      if (ctx) (ctx)->last_error = std::string(#expr) + ": " + cudaGetErrorString(_e); \
      return NRQ_ERR_CUDA;                                                   \
    }                                                                        \
  } while (0)

// host helpers shared by the C-ABI translation units (capi.cu, batch.cu)
namespace nrqh {
int set_device(nrq_ctx *ctx);
// NRQ_ERR_CUDA with ctx->last_error set when the last launch failed
int check_launch(nrq_ctx *ctx, const char *what);
// per-species, per-term coefficients of A (herm = false) or A^H (herm = true)
nrq::CnCoef make_coef(const nrq_ctx *ctx, double mass, const double c[8], double dt, bool herm);
// Chebyshev segment of A^H = 1 + i tau H for spec(H) in [lo, hi]
struct ChebSeg {
  std::complex<double> theta, delta, sigma;
};
ChebSeg cheb_segment(double tau, double lo, double hi);
// |T_m(sigma)|: error reduction guaranteed by m Chebyshev steps
double cheb_gain(std::complex<double> sigma, int m);
// FP64 view of the links of g current (precision form: widen the FP32 links)
int gauge_sync64(const nrq_gauge *g);
// learned initial guess (learned.cu)
bool learned_ready(const nrq_learn *net);
// x = 2b - psi + w0 u + w1 v1 + w2 v2, hnew = the learned part (v1, v2 may be
// null; hnew may alias v2)
int learned_guess(nrq_learn *net, const nrq_ctx *ctx, const double2 *psi, const double2 *b, const float2 *v1,
                  const float2 *v2, float2 *hnew, const double2 *U, const double *E, double mass, double dt,
                  double2 *x, cudaStream_t st);
void add_e_hist(int64_t n, double2 *x, const float2 *e, float2 *hist, cudaStream_t st);
int learned_check(nrq_learn *net);
const nrq_ctx *learned_ctx(const nrq_learn *net);
int learn_record(nrq_learn *net, const nrq_ctx *ctx, const double2 *psi, const double2 *b, const double2 *x,
                 const float2 *v1, const float2 *v2, float2 *hnew, const double2 *U, const double *E, double mass,
                 double dt);
// at least `depth` history slots of h allocated (2 by default); growing the
// ring drops the history it held
int ensure_hist(nrq_heavy *h, int depth = 2);
// learned guess of every field of a batch table (learned.cu)
int learned_guess_batch(nrq_learn *net, const nrq_ctx *ctx, const nrq::BatchField *tab, int nfields,
                        const double2 *U, const double *E, float4 *gf, float *fbuf, float4 *omega,
                        cudaStream_t st);
}  // namespace nrqh
