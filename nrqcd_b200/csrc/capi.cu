// C ABI (include/nrqcd_b200.h): handles, host<->device transfers, the
// leapfrog sequencing, the Krylov driver of the Crank-Nicolson step, and the
// initial-condition pipeline (host ranlxd stream, cuFFT, device kernels).
#include <cufft.h>

#include <cfloat>
#include <cmath>
#include <complex>
#include <cstring>
#include <new>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/nrqcd_b200.h"
#include "nrq_internal.h"
#include "nrq_kernels.cuh"
#include "ranlxd_host.h"
#include "ranlxd_dev.cuh"

using nrq::cplx;
using nrqh::check_launch;
using nrqh::make_coef;
using nrqh::set_device;

namespace {
using nrqh::Ranlxd;

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// per-column Krylov scalars followed by one int error flag written by the
// stencil kernels (NRQ_ERR_TIMEOUT when a bounded wait expired)
constexpr size_t kScalDoubles = (size_t)nrq::CN_COLS * nrq::SC_STRIDE;
// after the scalars: 16 ints of the stencils' error record (the flag, and
// where a bounded wait expired)
constexpr size_t kScalBytes = sizeof(double) * (kScalDoubles + 8);
inline int *scal_err(double *scal) { return (int *)(scal + kScalDoubles); }
// the stencils' record of an expired pipeline wait (4 ints after the
// scalars): the message of the update that reports it, and a reset
std::string timeout_message(const double *h_scal) {
  const int *e = (const int *)(h_scal + kScalDoubles);
  static const char *roles[] = {"a consumer's wait for a load", "a consumer's wait for the diagonal matrices",
                                "the loader's wait for a released buffer", "the loader's wait for a landed load",
                                "the loader's final drain"};
  const int stencil = e[1] / 16, role = e[1] % 16;
  std::string m = "CN stencil: a bounded pipeline wait expired";
  if (e[1] != 0) {
    m += std::string(" (") + (stencil == 6 ? "k_cheb5f" : "k_cn_mv" + std::to_string(stencil)) + ", " +
         (role >= 0 && role < 5 ? roles[role] : "?") +
         ", load " + std::to_string(e[2]) + ", CTA " + std::to_string(e[3]);
    if (e[4] != 0) {  // the FMA stencil's detail: the loader's progress and the barrier's word
      char buf[96];
      snprintf(buf, sizeof buf, ", loads issued %d, barrier %08x%08x, parity %d", e[4] - 1, (unsigned)e[6],
               (unsigned)e[5], e[7]);
      m += buf;
    }
    m += ")";
  }
  return m;
}

int ensure_stage(nrq_ctx *ctx, size_t bytes) {
  if (ctx->stage_bytes >= bytes) return NRQ_OK;
  if (ctx->d_stage) cudaFree(ctx->d_stage);
  ctx->d_stage = nullptr;
  ctx->stage_bytes = 0;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&ctx->d_stage, bytes));
  ctx->stage_bytes = bytes;
  return NRQ_OK;
}

int ensure_red(nrq_ctx *ctx, int64_t doubles) {
  if (ctx->red_cap >= doubles) return NRQ_OK;
  if (ctx->d_red) cudaFree(ctx->d_red);
  ctx->d_red = nullptr;
  ctx->red_cap = 0;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&ctx->d_red, sizeof(double) * doubles));
  ctx->red_cap = doubles;
  return NRQ_OK;
}

// final reduction of nq values over nb partial blocks into h_res[0..nq)
int reduce_to_host(nrq_ctx *ctx, int64_t nb, int nq, unsigned maxmask) {
  nrq::k_reduce_final<<<1, 256, 0, ctx->stream>>>(ctx->d_red, nb, nq, maxmask, ctx->d_res);
  int rc = check_launch(ctx, "k_reduce_final");
  if (rc) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_res, ctx->d_res, sizeof(double) * nq, cudaMemcpyDeviceToHost,
                                    ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return NRQ_OK;
}

}  // namespace

namespace nrqh {
// Chebyshev parameters for A^H = 1 + i tau H with spec(H) in [lo, hi]:
// theta (centre), delta (half-length), sigma = theta/delta
ChebSeg cheb_segment(double tau, double lo, double hi) {
  ChebSeg s;
  s.theta = std::complex<double>(1.0, tau * 0.5 * (lo + hi));
  double half = std::fabs(tau) * 0.5 * (hi - lo);
  if (half < 1e-14) half = 1e-14;
  s.delta = std::complex<double>(0.0, half);
  s.sigma = s.theta / s.delta;
  return s;
}
// |T_m(sigma)| via the recurrence T_{k+1} = 2 sigma T_k - T_{k-1}
double cheb_gain(std::complex<double> sigma, int m) {
  std::complex<double> t0(1.0, 0.0), t1 = sigma;
  if (m == 0) return 1.0;
  for (int k = 1; k < m; ++k) {
    std::complex<double> t2 = 2.0 * sigma * t1 - t0;
    t0 = t1;
    t1 = t2;
  }
  return std::abs(t1);
}

int set_device(nrq_ctx *ctx) {
  NRQ_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  return NRQ_OK;
}

int check_launch(nrq_ctx *ctx, const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return NRQ_ERR_CUDA;
  }
  return NRQ_OK;
}

// per-species, per-term coefficients; herm selects A^H
nrq::CnCoef make_coef(const nrq_ctx *ctx, double mass, const double c_[8], double dt, bool herm) {
  nrq::CnCoef C{};
  const cplx kappa = {0.0, -dt / 2 * ctx->a[0]};
  for (int sp = 0; sp < 2; ++sp) {
    const double M = sp == 0 ? mass : -mass;
    cplx c[4];
    for (int k = 0; k < 4; ++k) c[k] = {c_[2 * k], sp == 0 ? c_[2 * k + 1] : -c_[2 * k + 1]};
    cplx kin = (1.0 / M) * (kappa * c[0]);
    cplx mag = (-1.0 / (2.0 * M)) * (kappa * c[1]);
    cplx dar = (-1.0 / (8.0 * M * M)) * (kappa * c[2]);
    cplx so = (-1.0 / (8.0 * M * M)) * (kappa * c[3]);
    if (herm) {
      kin = nrq::conj(kin);
      mag = nrq::conj(mag);
      dar = nrq::conj(dar);
      so = nrq::conj(so);
    }
    C.kin[sp] = kin;
    C.mag[sp] = mag;
    C.dar[sp] = dar;
    C.so[sp] = so;
  }
  C.dkin = 0.0;
  for (int i = 0; i < 3; ++i) {
    C.inva2[i] = 1.0 / (ctx->a[i + 1] * ctx->a[i + 1]);
    C.dkin += C.inva2[i];
  }
  return C;
}

int gauge_sync64(const nrq_gauge *gc) {
  nrq_gauge *g = const_cast<nrq_gauge *>(gc);
  if (g->prec != 1 || !g->stale64) return NRQ_OK;
  const int64_t n = 27 * g->ctx->lat.V;
  nrq::k_links_widen<<<(unsigned)((n + 255) / 256), 256, 0, g->ctx->stream>>>(n, g->U32, g->U);
  int rc = check_launch(g->ctx, "k_links_widen");
  if (!rc) g->stale64 = false;
  return rc;
}
}  // namespace nrqh

namespace {
// after the FP64 links were written: refresh the FP32 links of the precision form
int gauge_written64(nrq_gauge *g) {
  if (g->prec != 1) return NRQ_OK;
  const int64_t n = 27 * g->ctx->lat.V;
  nrq::k_links_narrow<<<(unsigned)((n + 255) / 256), 256, 0, g->ctx->stream>>>(n, g->U, g->U32);
  g->stale64 = false;
  g->since_reunit = 0;
  return check_launch(g->ctx, "k_links_narrow");
}
}  // namespace
using nrqh::gauge_sync64;

// ====================================================================== context
extern "C" const char *nrq_status_string(int s) {
  switch (s) {
    case NRQ_OK: return "ok";
    case NRQ_ERR_NOT_INITIALISED: return "not initialised";
    case NRQ_ERR_ALREADY_INITIALISED: return "already initialised";
    case NRQ_ERR_BAD_ARG: return "bad argument";
    case NRQ_ERR_CUDA: return "CUDA error";
    case NRQ_ERR_NOT_CONVERGED: return "Krylov solve did not converge";
    case NRQ_ERR_TIMEOUT: return "timeout";
    case NRQ_ERR_NONFINITE: return "non-finite value";
    case NRQ_ERR_NO_DEVICE: return "no CUDA device";
    case NRQ_ERR_OOM: return "out of memory";
    case NRQ_ERR_CAPACITY: return "lattice exceeds the fixed scratch capacity of a no-allocation entry point";
    default: return "unknown status";
  }
}

extern "C" const char *nrq_last_error(const nrq_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

extern "C" int nrq_init(const int64_t ext[3], const double a[4], int device, nrq_ctx **out) {
  if (!ext || !a || !out) return NRQ_ERR_BAD_ARG;
  *out = nullptr;
  for (int k = 0; k < 3; ++k)
    if (ext[k] < 1) return NRQ_ERR_BAD_ARG;
  for (int k = 0; k < 4; ++k)
    if (!(a[k] > 0.0)) return NRQ_ERR_BAD_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return NRQ_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = new (std::nothrow) nrq_ctx();
  if (!ctx) return NRQ_ERR_OOM;
  ctx->device = device;
  for (int k = 0; k < 3; ++k) ctx->n[k] = ext[k];
  for (int k = 0; k < 4; ++k) ctx->a[k] = a[k];
  ctx->lat.nx = ext[0];
  ctx->lat.ny = ext[1];
  ctx->lat.nz = ext[2];
  ctx->lat.V = ext[0] * ext[1] * ext[2];
  ctx->lat.a0 = a[0];
  for (int k = 0; k < 3; ++k) ctx->lat.a[k] = a[k + 1];
  int rc = set_device(ctx);
  if (rc == NRQ_OK) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) ctx->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_res, sizeof(double) * 64) != cudaSuccess ||
        cudaMallocHost(&ctx->h_res, sizeof(double) * 64) != cudaSuccess)
      rc = NRQ_ERR_CUDA;
  }
  if (rc == NRQ_OK) rc = ensure_red(ctx, ((ctx->lat.V + 127) / 128) * 8 + 1024);
  if (rc != NRQ_OK) {
    nrq_finalize(ctx);
    return rc;
  }
  *out = ctx;
  return NRQ_OK;
}

extern "C" int nrq_finalize(nrq_ctx *ctx) {
  if (!ctx) return NRQ_ERR_NOT_INITIALISED;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->d_red) cudaFree(ctx->d_red);
  if (ctx->d_res) cudaFree(ctx->d_res);
  if (ctx->h_res) cudaFreeHost(ctx->h_res);
  if (ctx->d_stage) cudaFree(ctx->d_stage);
  if (ctx->d_proj) cudaFree(ctx->d_proj);
  if (ctx->fft9_ok) cufftDestroy((cufftHandle)ctx->fft9);
  if (ctx->fft48_ok) cufftDestroy((cufftHandle)ctx->fft48);
  if (ctx->d_gluon) cudaFree(ctx->d_gluon);
  for (auto &r : ctx->prof_recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : ctx->prof_pool) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return NRQ_OK;
}

extern "C" int nrq_synchronize(nrq_ctx *ctx) {
  if (!ctx) return NRQ_ERR_NOT_INITIALISED;
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return NRQ_OK;
}

extern "C" void *nrq_cuda_stream(nrq_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" int nrq_profile_enable(nrq_ctx *ctx, int enable) {
  if (!ctx) return NRQ_ERR_NOT_INITIALISED;
  ctx->prof = enable != 0;
  return NRQ_OK;
}

extern "C" int nrq_profile_read(nrq_ctx *ctx, int64_t launches[6], double ms[6], double bytes[6]) {
  if (!ctx || !launches || !ms || !bytes) return NRQ_ERR_BAD_ARG;
  int rc = set_device(ctx);
  if (rc) return rc;
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < NRQ_PROF_CLASSES; ++k) {
    launches[k] = 0;
    ms[k] = 0.0;
    bytes[k] = 0.0;
  }
  for (auto &r : ctx->prof_recs) {
    float t = 0.f;
    cudaEventElapsedTime(&t, r.a, r.b);
    if (r.cls >= 0 && r.cls < NRQ_PROF_CLASSES) {
      launches[r.cls] += 1;
      ms[r.cls] += t;
      bytes[r.cls] += r.bytes;
    }
    ctx->prof_pool.push_back(r.a);
    ctx->prof_pool.push_back(r.b);
  }
  ctx->prof_recs.clear();
  return NRQ_OK;
}

// ====================================================================== gauge
extern "C" int nrq_gauge_create(nrq_ctx *ctx, nrq_gauge **out) {
  if (!ctx || !out) return NRQ_ERR_BAD_ARG;
  *out = nullptr;
  int rc = set_device(ctx);
  if (rc) return rc;
  nrq_gauge *g = new (std::nothrow) nrq_gauge();
  if (!g) return NRQ_ERR_OOM;
  g->ctx = ctx;
  const int64_t V = ctx->lat.V;
  if (cudaMalloc(&g->U, sizeof(double2) * 27 * V) != cudaSuccess ||
      cudaMalloc(&g->E, sizeof(double) * 24 * V) != cudaSuccess) {
    cudaGetLastError();
    if (g->U) cudaFree(g->U);
    if (g->E) cudaFree(g->E);
    delete g;
    ctx->last_error = "nrq_gauge_create: device allocation failed";
    return NRQ_ERR_OOM;
  }
  nrq::k_cold<<<nblk(V, 256), 256, 0, ctx->stream>>>(g->U, g->E, V);
  rc = check_launch(ctx, "k_cold");
  if (rc) {
    nrq_gauge_destroy(g);
    return rc;
  }
  *out = g;
  return NRQ_OK;
}

extern "C" int nrq_gauge_destroy(nrq_gauge *g) {
  if (!g) return NRQ_ERR_BAD_ARG;
  cudaSetDevice(g->ctx->device);
  cudaStreamSynchronize(g->ctx->stream);
  if (g->U) cudaFree(g->U);
  if (g->E) cudaFree(g->E);
  if (g->U32) cudaFree(g->U32);
  delete g;
  return NRQ_OK;
}

extern "C" int nrq_gauge_upload(nrq_gauge *g, const double *links, const double *efield) {
  if (!g || !links || !efield) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  const int64_t V = ctx->lat.V;
  int rc = set_device(ctx);
  if (!rc) rc = ensure_stage(ctx, sizeof(double2) * 27 * V);
  if (rc) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_stage, links, sizeof(double2) * 27 * V, cudaMemcpyHostToDevice,
                                    ctx->stream));
  nrq::k_links_f2soa<<<nblk(V, 128), 128, 0, ctx->stream>>>((const double2 *)ctx->d_stage, g->U, V);
  if ((rc = check_launch(ctx, "k_links_f2soa"))) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_stage, efield, sizeof(double) * 24 * V, cudaMemcpyHostToDevice,
                                    ctx->stream));
  nrq::k_efield_f2soa<<<nblk(V, 128), 128, 0, ctx->stream>>>((const double *)ctx->d_stage, g->E, V);
  if ((rc = check_launch(ctx, "k_efield_f2soa"))) return rc;
  return gauge_written64(g);
}

extern "C" int nrq_gauge_download(const nrq_gauge *g, double *links, double *efield) {
  if (!g || !links || !efield) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  const int64_t V = ctx->lat.V;
  int rc = set_device(ctx);
  if (!rc) rc = ensure_stage(ctx, sizeof(double2) * 27 * V);
  if (!rc) rc = gauge_sync64(g);
  if (rc) return rc;
  nrq::k_links_soa2f<<<nblk(V, 128), 128, 0, ctx->stream>>>(g->U, (double2 *)ctx->d_stage, V);
  if ((rc = check_launch(ctx, "k_links_soa2f"))) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(links, ctx->d_stage, sizeof(double2) * 27 * V, cudaMemcpyDeviceToHost,
                                    ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  nrq::k_efield_soa2f<<<nblk(V, 128), 128, 0, ctx->stream>>>(g->E, (double *)ctx->d_stage, V);
  if ((rc = check_launch(ctx, "k_efield_soa2f"))) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(efield, ctx->d_stage, sizeof(double) * 24 * V, cudaMemcpyDeviceToHost,
                                    ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return NRQ_OK;
}

extern "C" int nrq_gauge_copy(nrq_gauge *dst, const nrq_gauge *src) {
  if (!dst || !src || dst->ctx != src->ctx) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = dst->ctx;
  const int64_t V = ctx->lat.V;
  int rc = set_device(ctx);
  if (!rc) rc = gauge_sync64(src);
  if (rc) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(dst->U, src->U, sizeof(double2) * 27 * V, cudaMemcpyDeviceToDevice, ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(dst->E, src->E, sizeof(double) * 24 * V, cudaMemcpyDeviceToDevice, ctx->stream));
  return gauge_written64(dst);
}

extern "C" int nrq_gauge_cold_init(nrq_gauge *g) {
  if (!g) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  nrq::k_cold<<<nblk(ctx->lat.V, 256), 256, 0, ctx->stream>>>(g->U, g->E, ctx->lat.V);
  if ((rc = check_launch(ctx, "k_cold"))) return rc;
  return gauge_written64(g);
}

extern "C" int nrq_gauge_transverse_box_init(nrq_gauge *g, double Q, double n0, double coupling, int64_t seed,
                                             int identity_links) {
  if (!g) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  const nrq::Lat L = ctx->lat;
  const int64_t V = L.V;
  int rc = set_device(ctx);
  if (rc) return rc;
  Ranlxd rng;
  if (!rng.init(2, seed)) {
    ctx->last_error = "transverse_box_init: seed must lie in [1, 2^31-1]";
    return NRQ_ERR_BAD_ARG;
  }
  // backward-derivative momentum per direction and coordinate (lattice:963-979):
  // component (re, im) and modulus, in the host's arithmetic
  std::vector<double> mtab;
  {
    const double pi = std::acos(-1.0);
    for (int i = 0; i < 3; ++i)
      for (int64_t n = 0; n < ctx->n[i]; ++n) {
        const double ang = pi * (double)n / (double)ctx->n[i];
        const double mag = 2.0 * std::sin(ang) / ctx->a[i + 1];
        const double re = mag * std::cos(-ang), im = mag * std::sin(-ang);
        mtab.push_back(re);
        mtab.push_back(im);
        mtab.push_back(std::hypot(re, im));
      }
  }
  double2 *dR = nullptr, *dA = nullptr, *dEf = nullptr;
  double *dM = nullptr;
  cufftHandle plan16 = 0, plan24 = 0;
  bool p16 = false, p24 = false;
  auto cleanup = [&]() {
    if (p16) cufftDestroy(plan16);
    if (p24) cufftDestroy(plan24);
    if (dR) cudaFree(dR);
    if (dA) cudaFree(dA);
    if (dEf) cudaFree(dEf);
    if (dM) cudaFree(dM);
  };
  if (cudaMalloc(&dR, sizeof(double2) * 16 * V) != cudaSuccess ||
      cudaMalloc(&dA, sizeof(double2) * 24 * V) != cudaSuccess ||
      cudaMalloc(&dEf, sizeof(double2) * 24 * V) != cudaSuccess ||
      cudaMalloc(&dM, sizeof(double) * mtab.size()) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    ctx->last_error = "transverse_box_init: device allocation failed";
    return NRQ_ERR_OOM;
  }
  int dims[3] = {(int)L.nz, (int)L.ny, (int)L.nx};
  if (cufftPlanMany(&plan16, 3, dims, nullptr, 1, (int)V, nullptr, 1, (int)V, CUFFT_Z2Z, 16) != CUFFT_SUCCESS) {
    cleanup();
    ctx->last_error = "transverse_box_init: cufftPlanMany failed";
    return NRQ_ERR_CUDA;
  }
  p16 = true;
  if (cufftPlanMany(&plan24, 3, dims, nullptr, 1, (int)V, nullptr, 1, (int)V, CUFFT_Z2Z, 24) != CUFFT_SUCCESS) {
    cleanup();
    ctx->last_error = "transverse_box_init: cufftPlanMany failed";
    return NRQ_ERR_CUDA;
  }
  p24 = true;
  cufftSetStream(plan16, ctx->stream);
  cufftSetStream(plan24, ctx->stream);
  // real parts of complex Box-Muller normals, per site, per polarisation
  // (gauge:1334-1340, random.f90:238-255): plane (pol*8 + a), pair
  // e = 16 s + 8 pol + a of the stream, drawn on the device
  if ((rc = nrq::device_draw_pairs(ctx, 2, seed, 0, 16 * V, nrq::BoxPairs{dR, V}))) {
    cleanup();
    return rc;
  }
  if (cudaMemcpyAsync(dM, mtab.data(), sizeof(double) * mtab.size(), cudaMemcpyHostToDevice, ctx->stream) !=
      cudaSuccess) {
    cleanup();
    return NRQ_ERR_CUDA;
  }
  bool ok = cufftExecZ2Z(plan16, (cufftDoubleComplex *)dR, (cufftDoubleComplex *)dR, CUFFT_FORWARD) == CUFFT_SUCCESS;
  const double fwd_scale = ctx->a[1] * ctx->a[2] * ctx->a[3];
  const double volume = (double)V * fwd_scale;
  if (ok) {
    nrq::k_ic_pspace<<<nblk(V, 128), 128, 0, ctx->stream>>>(L, dR, dM, fwd_scale, Q, n0, coupling, dA, dEf);
    ok = cudaGetLastError() == cudaSuccess;
  }
  ok = ok && cufftExecZ2Z(plan24, (cufftDoubleComplex *)dA, (cufftDoubleComplex *)dA, CUFFT_INVERSE) == CUFFT_SUCCESS;
  ok = ok && cufftExecZ2Z(plan24, (cufftDoubleComplex *)dEf, (cufftDoubleComplex *)dEf, CUFFT_INVERSE) == CUFFT_SUCCESS;
  if (ok) {
    nrq::k_ic_write<<<nblk(V, 128), 128, 0, ctx->stream>>>(L, dA, dEf, 1.0 / volume, identity_links, g->U, g->E);
    ok = cudaGetLastError() == cudaSuccess;
  }
  ok = ok && cudaStreamSynchronize(ctx->stream) == cudaSuccess;
  cleanup();
  if (!ok) {
    ctx->last_error = "transverse_box_init: FFT or kernel failure";
    return NRQ_ERR_CUDA;
  }
  return gauge_written64(g);
}

extern "C" int nrq_gauge_update(nrq_gauge *g, double dt) {
  if (!g) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  const unsigned nb_ = nblk(ctx->lat.V, 128);
  const double V = (double)ctx->lat.V;
  const bool p32 = g->prec == 1;
  auto links = [&]() {
    if (p32) {
      ProfScope ps(ctx, 4, V * (192.0 + 216.0 + 216.0));
      nrq::k_update_links32<<<nb_, 128, 0, ctx->stream>>>(ctx->lat, g->U32, g->E, dt);
    } else {
      ProfScope ps(ctx, 4, V * (192.0 + 432.0 + 432.0));
      nrq::k_update_links<<<nb_, 128, 0, ctx->stream>>>(ctx->lat, g->U, g->E, dt);
    }
  };
  auto efield = [&]() {
    if (p32) {
      ProfScope ps(ctx, 5, V * (216.0 + 192.0 + 192.0));
      nrq::k_update_efield32<<<nb_, 128, 0, ctx->stream>>>(ctx->lat, g->U32, g->E, dt);
    } else {
      ProfScope ps(ctx, 5, V * (432.0 + 192.0 + 192.0));
      nrq::k_update_efield<<<3 * nb_, 128, 0, ctx->stream>>>(ctx->lat, g->U, g->E, dt);
    }
  };
  // Update_Leapfrog ordering (gauge:2100-2110)
  if (dt > 0) {
    links();
    efield();
  } else {
    efield();
    links();
  }
  if ((rc = check_launch(ctx, "leapfrog"))) return rc;
  if (p32) {
    g->stale64 = true;
    if (++g->since_reunit >= g->reunit_every) {  // FP64 reunitarisation
      ProfScope ps(ctx, 4, V * (216.0 + 432.0 + 216.0));
      nrq::k_reunitarise<<<nblk(ctx->lat.V, 128), 128, 0, ctx->stream>>>(ctx->lat.V, g->U32, g->U);
      g->since_reunit = 0;
      g->stale64 = false;
      rc = check_launch(ctx, "k_reunitarise");
    }
  }
  return rc;
}

extern "C" int nrq_gauge_set_precision(nrq_gauge *g, int prec, int reunit_every) {
  if (!g || prec < 0 || prec > 1 || (prec == 1 && reunit_every < 1)) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  if (prec == g->prec) {
    if (prec == 1) g->reunit_every = reunit_every;
    return NRQ_OK;
  }
  if (prec == 1) {
    if (!g->U32) NRQ_CUDA_TRY(ctx, cudaMalloc(&g->U32, sizeof(float2) * 27 * ctx->lat.V));
    g->prec = 1;
    g->reunit_every = reunit_every;
    return gauge_written64(g);
  }
  if ((rc = gauge_sync64(g))) return rc;  // back to FP64: the FP64 view becomes the state
  g->prec = 0;
  g->stale64 = false;
  return NRQ_OK;
}

extern "C" int nrq_gauge_unitarity(nrq_gauge *g, double *max_dev, double *max_det_dev) {
  if (!g) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  int rc = set_device(ctx);
  if (!rc) rc = gauge_sync64(g);
  if (rc) return rc;
  const int64_t nb_ = nblk(ctx->lat.V, 256);
  if ((rc = ensure_red(ctx, nb_ * 2))) return rc;
  nrq::k_unitarity<<<(unsigned)nb_, 256, 0, ctx->stream>>>(ctx->lat, g->U, ctx->d_red);
  if ((rc = check_launch(ctx, "k_unitarity"))) return rc;
  if ((rc = reduce_to_host(ctx, nb_, 2, 3u))) return rc;
  if (max_dev) *max_dev = ctx->h_res[0];
  if (max_det_dev) *max_det_dev = ctx->h_res[1];
  return NRQ_OK;
}

extern "C" int nrq_gauge_energy(nrq_gauge *g, double *energy) {
  if (!g || !energy) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  const int64_t nb_ = nblk(ctx->lat.V, 256);
  if ((rc = ensure_red(ctx, nb_ * 2))) return rc;
  if ((rc = gauge_sync64(g))) return rc;
  nrq::k_energy<<<(unsigned)nb_, 256, 0, ctx->stream>>>(ctx->lat, g->U, g->E, ctx->d_red);
  if ((rc = check_launch(ctx, "k_energy"))) return rc;
  if ((rc = reduce_to_host(ctx, nb_, 1, 0u))) return rc;
  *energy = ctx->h_res[0];
  return NRQ_OK;
}

extern "C" int nrq_gauge_gauss(nrq_gauge *g, double *ref_measure, double *max_norm) {
  if (!g) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  const int64_t nb_ = nblk(ctx->lat.V, 256);
  if ((rc = ensure_red(ctx, nb_ * 2))) return rc;
  if ((rc = gauge_sync64(g))) return rc;
  nrq::k_gauss<<<(unsigned)nb_, 256, 0, ctx->stream>>>(ctx->lat, g->U, g->E, ctx->d_red);
  if ((rc = check_launch(ctx, "k_gauss"))) return rc;
  if ((rc = reduce_to_host(ctx, nb_, 2, 2u))) return rc;
  if (ref_measure) *ref_measure = ctx->h_res[0];
  if (max_norm) *max_norm = ctx->h_res[1];
  return NRQ_OK;
}

// ---------------------------------------------------------------- thermal initial condition
namespace {
constexpr int64_t kProjUnbounded = INT64_MAX;

// Gauss projection sweeps of EquilibriumInit (gauge:455-500) on g's FP64
// field.  Sweeps are queued in growing batches; the kernels themselves stop
// at the first sweep whose deviation is at most tol, so the count is exact.
int gauss_project(nrq_gauge *g, double tol, int64_t max_sweeps, int64_t *sweeps, double *deviation) {
  nrq_ctx *ctx = g->ctx;
  const nrq::Lat L = ctx->lat;
  const int64_t V = L.V;
  const unsigned nbg = (unsigned)nblk(V, 128), nbs = (unsigned)nblk(V, 128);
  int rc = gauge_sync64(g);
  if (!rc) rc = ensure_stage(ctx, sizeof(double2) * 9 * V);
  if (!rc) rc = ensure_red(ctx, nbg);
  if (rc) return rc;
  if (!ctx->d_proj) NRQ_CUDA_TRY(ctx, cudaMalloc(&ctx->d_proj, sizeof(nrq::GaussProjState)));
  nrq::GaussProjState *st = (nrq::GaussProjState *)ctx->d_proj;
  double2 *G = (double2 *)ctx->d_stage;
  const double kdt = 0.01 * ctx->a[0];  // kappa a0, kappa = 0.01 (gauge:408)
  NRQ_CUDA_TRY(ctx, cudaMemsetAsync(st, 0, sizeof(nrq::GaussProjState), ctx->stream));
  nrq::k_gauss_g<<<nbg, 128, 0, ctx->stream>>>(L, g->U, g->E, G, ctx->d_red, st, tol, 0);
  if ((rc = check_launch(ctx, "k_gauss_g"))) return rc;
  const int64_t limit = max_sweeps > 0 ? max_sweeps : kProjUnbounded;
  int64_t queued = 0, batch = 16;
  nrq::GaussProjState h{};
  for (;;) {
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h.done || queued >= limit) break;
    const int64_t n = std::min(batch, limit - queued);
    for (int64_t k = 0; k < n; ++k) {
      nrq::k_gauss_sweep<<<nbs, 128, 0, ctx->stream>>>(L, g->U, G, g->E, st, kdt);
      nrq::k_gauss_g<<<nbg, 128, 0, ctx->stream>>>(L, g->U, g->E, G, ctx->d_red, st, tol, 1);
    }
    if ((rc = check_launch(ctx, "Gauss projection sweep"))) return rc;
    queued += n;
    batch = std::min<int64_t>(batch * 2, 512);
  }
  if (sweeps) *sweeps = h.sweeps;
  if (deviation) *deviation = h.dev;
  if (!h.done) {
    ctx->last_error = "Gauss projection: deviation above tolerance after max_sweeps sweeps";
    return NRQ_ERR_NOT_CONVERGED;
  }
  return NRQ_OK;
}
}  // namespace

extern "C" int nrq_gauge_gauss_project(nrq_gauge *g, double tol, int64_t max_sweeps, int64_t *sweeps,
                                       double *deviation) {
  if (!g || !(tol >= 0.0) || g->ctx->lat.V > INT32_MAX) return NRQ_ERR_BAD_ARG;
  int rc = set_device(g->ctx);
  if (rc) return rc;
  return gauss_project(g, tol, max_sweeps, sweeps, deviation);
}

extern "C" int nrq_gauge_equilibrium_init(nrq_gauge *g, double beta, int64_t nefieldinit, int64_t nequilibrium,
                                          double tol, int64_t seed, int64_t max_sweeps, int64_t *sweeps,
                                          double *energies, double *deviations) {
  if (!g || !(beta > 0.0) || nefieldinit < 0 || nequilibrium < 0 || !(tol >= 0.0) || g->ctx->lat.V > INT32_MAX)
    return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  const int64_t V = ctx->lat.V;
  int rc = set_device(ctx);
  if (rc) return rc;
  Ranlxd rng;
  if (!rng.init(2, seed)) {
    ctx->last_error = "equilibrium_init: seed must lie in [1, 2^31-1]";
    return NRQ_ERR_BAD_ARG;
  }
  nrq::k_cold<<<nblk(V, 256), 256, 0, ctx->stream>>>(g->U, g->E, V);
  if ((rc = check_launch(ctx, "k_cold"))) return rc;
  if ((rc = gauge_written64(g))) return rc;
  const double sigma = std::sqrt(4.0 / beta), a0 = ctx->a[0];
  for (int64_t r = 0; r < nefieldinit; ++r) {
    // Box-Muller pairs in the reference's order: site, direction, generator
    // (random.f90:238-255); the real part, times sigma, times a0.  Round r
    // starts at number 48 V r of the stream; drawn on the device, straight
    // into the field's planes.
    if ((rc = nrq::device_draw_pairs(ctx, 2, seed, (uint64_t)r * 48 * (uint64_t)V, 24 * V,
                                     nrq::ThermalPairs{g->E, V, sigma, a0})))
      return rc;
    int64_t it = 0;
    rc = gauss_project(g, tol, max_sweeps, &it, nullptr);
    if (sweeps) sweeps[r] = it;
    if (rc) return rc;
    for (int64_t t = 0; t < nequilibrium; ++t)
      if ((rc = nrq_gauge_update(g, 1.0))) return rc;
    if (energies && (rc = nrq_gauge_energy(g, &energies[r]))) return rc;
    if (deviations && (rc = nrq_gauge_gauss(g, nullptr, &deviations[r]))) return rc;
  }
  return NRQ_OK;
}

extern "C" int nrq_ranlxd_draw(nrq_ctx *ctx, int level, int64_t seed, uint64_t first, int64_t count, int normals,
                               double *out) {
  if (!ctx || !out || count < 0 || (first & 1) || (!normals && (count & 1)) || (level != 1 && level != 2) ||
      seed < 1 || seed > 2147483647LL)
    return NRQ_ERR_BAD_ARG;
  int rc = set_device(ctx);
  if (rc || count == 0) return rc;
  double *d = nullptr;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&d, sizeof(double) * count));
  rc = normals ? nrq::device_draw_pairs(ctx, level, seed, first, count, nrq::NormalPairs{d})
               : nrq::device_draw_pairs(ctx, level, seed, first, count / 2, nrq::UniformPairs{d});
  if (!rc && cudaMemcpy(out, d, sizeof(double) * count, cudaMemcpyDeviceToHost) != cudaSuccess) rc = NRQ_ERR_CUDA;
  cudaFree(d);
  return rc;
}

// ---------------------------------------------------------------- gluon distribution
namespace {
// cuFFT Z2Z plan over `batch` (9 or 48) complex planes of the lattice (x
// fastest), created once per context
bool lattice_fft_plan(nrq_ctx *ctx, int batch, cufftHandle *plan) {
  int *h = batch == 9 ? &ctx->fft9 : &ctx->fft48;
  bool *ok = batch == 9 ? &ctx->fft9_ok : &ctx->fft48_ok;
  if (!*ok) {
    const nrq::Lat L = ctx->lat;
    int dims[3] = {(int)L.nz, (int)L.ny, (int)L.nx};
    cufftHandle p = 0;
    if (cufftPlanMany(&p, 3, dims, nullptr, 1, (int)L.V, nullptr, 1, (int)L.V, CUFFT_Z2Z, batch) != CUFFT_SUCCESS)
      return false;
    *h = (int)p;
    *ok = true;
  }
  *plan = (cufftHandle)*h;
  cufftSetStream(*plan, ctx->stream);
  return true;
}

// the gluon observables' device buffer (grown on demand, kept)
int ensure_gluon(nrq_ctx *ctx, size_t bytes) {
  if (ctx->gluon_bytes >= bytes) return NRQ_OK;
  if (ctx->d_gluon) cudaFree(ctx->d_gluon);
  ctx->d_gluon = nullptr;
  ctx->gluon_bytes = 0;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&ctx->d_gluon, bytes));
  ctx->gluon_bytes = bytes;
  return NRQ_OK;
}

// FindMaxNorm2Momentum (lattice:422-465): |p|^2 is a sum over directions of
// (2 sin(pi n_i / N_i) / a_i)^2, so its maximum is the sum of the maxima
double max_norm2_momentum(const nrq_ctx *ctx) {
  const double pi = std::acos(-1.0);
  double s = 0.0;
  for (int i = 0; i < 3; ++i) {
    double m = 0.0;
    for (int64_t n = 0; n < ctx->n[i]; ++n) {
      const double v = 2.0 * std::sin(pi * (double)n / (double)ctx->n[i]) / ctx->a[i + 1];
      m = std::max(m, v * v);
    }
    s += m;
  }
  return std::sqrt(s);
}
}  // namespace

extern "C" int nrq_gauge_coulomb_gaugefix(nrq_gauge *g, double tol, double alpha, int64_t max_iterations,
                                          int64_t *iterations, double *deviations) {
  if (!g || max_iterations < 0) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  const nrq::Lat L = ctx->lat;
  const int64_t V = L.V;
  int rc = set_device(ctx);
  if (!rc) rc = gauge_sync64(g);
  if (rc) return rc;
  const unsigned nb_ = (unsigned)nblk(V, 128);
  if ((rc = ensure_red(ctx, nb_))) return rc;
  if ((rc = ensure_gluon(ctx, sizeof(double2) * 9 * V))) return rc;
  double2 *D = (double2 *)ctx->d_gluon;
  cufftHandle plan = 0;
  if (!lattice_fft_plan(ctx, 9, &plan)) {
    ctx->last_error = "CoulombGaugefixing: cufftPlanMany failed";
    return NRQ_ERR_CUDA;
  }
  const double pmax = max_norm2_momentum(ctx);
  // x2p scale a1 a2 a3 times p2x scale 1/Volume is 1/V; alpha folded in
  const double scale = alpha / (double)V;
  int64_t it;
  for (it = 1; it <= max_iterations; ++it) {
    nrq::k_cg_divergence<<<nb_, 128, 0, ctx->stream>>>(L, g->U, D, ctx->d_red);
    if ((rc = check_launch(ctx, "k_cg_divergence")) || (rc = reduce_to_host(ctx, nb_, 1, 1u))) break;
    const double dev = ctx->h_res[0];
    if (deviations) deviations[it - 1] = dev;
    if (!(dev > tol)) break;
    bool ok = cufftExecZ2Z(plan, (cufftDoubleComplex *)D, (cufftDoubleComplex *)D, CUFFT_FORWARD) == CUFFT_SUCCESS;
    if (ok) nrq::k_cg_accelerate<<<nb_, 128, 0, ctx->stream>>>(L, D, pmax, scale);
    ok = ok && cufftExecZ2Z(plan, (cufftDoubleComplex *)D, (cufftDoubleComplex *)D, CUFFT_INVERSE) == CUFFT_SUCCESS;
    if (!ok) {
      ctx->last_error = "CoulombGaugefixing: cuFFT failure";
      rc = NRQ_ERR_CUDA;
      break;
    }
    nrq::k_cg_expah<<<nb_, 128, 0, ctx->stream>>>(V, D);
    nrq::k_cg_transform<<<nb_, 128, 0, ctx->stream>>>(L, g->U, D);
    if ((rc = check_launch(ctx, "Coulomb gauge transformation"))) break;
  }
  if (iterations) *iterations = it;
  if (rc) return rc;
  return gauge_written64(g);
}

extern "C" int nrq_gauge_transverse_correlators(nrq_gauge *g, double *aa, double *ee, double *momenta) {
  if (!g) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = g->ctx;
  const nrq::Lat L = ctx->lat;
  const int64_t V = L.V;
  int rc = set_device(ctx);
  if (!rc) rc = gauge_sync64(g);
  if (rc) return rc;
  if ((rc = ensure_gluon(ctx, sizeof(double2) * 48 * V + sizeof(double) * 3 * V))) return rc;
  double2 *F = (double2 *)ctx->d_gluon;
  double *out = (double *)(F + 48 * V);
  cufftHandle plan = 0;
  if (!lattice_fft_plan(ctx, 48, &plan)) {
    ctx->last_error = "transverse correlators: cufftPlanMany failed";
    return NRQ_ERR_CUDA;
  }
  const unsigned nb_ = (unsigned)nblk(V, 128);
  const double fwd = ctx->a[1] * ctx->a[2] * ctx->a[3];
  nrq::k_gluon_fields<<<nb_, 128, 0, ctx->stream>>>(L, g->U, g->E, F);
  bool ok = cudaGetLastError() == cudaSuccess &&
            cufftExecZ2Z(plan, (cufftDoubleComplex *)F, (cufftDoubleComplex *)F, CUFFT_FORWARD) == CUFFT_SUCCESS;
  if (ok) {
    nrq::k_transverse_corr<<<nb_, 128, 0, ctx->stream>>>(L, F, fwd, (double)V * fwd, out);
    ok = cudaGetLastError() == cudaSuccess;
  }
  double *dst[3] = {aa, ee, momenta};
  for (int k = 0; k < 3 && ok; ++k)
    if (dst[k])
      ok = cudaMemcpyAsync(dst[k], out + (int64_t)k * V, sizeof(double) * V, cudaMemcpyDeviceToHost, ctx->stream) ==
           cudaSuccess;
  ok = ok && cudaStreamSynchronize(ctx->stream) == cudaSuccess;
  if (!ok) {
    ctx->last_error = "transverse correlators: kernel, cuFFT or copy failure";
    return NRQ_ERR_CUDA;
  }
  return NRQ_OK;
}

// ====================================================================== heavy field
extern "C" int nrq_heavy_create(nrq_ctx *ctx, nrq_heavy **out) {
  if (!ctx || !out) return NRQ_ERR_BAD_ARG;
  *out = nullptr;
  int rc = set_device(ctx);
  if (rc) return rc;
  nrq_heavy *h = new (std::nothrow) nrq_heavy();
  if (!h) return NRQ_ERR_OOM;
  h->ctx = ctx;
  if (cudaMalloc(&h->P, sizeof(double2) * 72 * ctx->lat.V) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    ctx->last_error = "nrq_heavy_create: device allocation failed";
    return NRQ_ERR_OOM;
  }
  NRQ_CUDA_TRY(ctx, cudaMemsetAsync(h->P, 0, sizeof(double2) * 72 * ctx->lat.V, ctx->stream));
  *out = h;
  return NRQ_OK;
}

extern "C" int nrq_heavy_destroy(nrq_heavy *h) {
  if (!h) return NRQ_ERR_BAD_ARG;
  cudaSetDevice(h->ctx->device);
  cudaStreamSynchronize(h->ctx->stream);
  if (h->P) cudaFree(h->P);
  for (float2 *q : h->hist)
    if (q) cudaFree(q);
  delete h;
  return NRQ_OK;
}

extern "C" int nrq_heavy_upload(nrq_heavy *h, const double *q, const double *a) {
  if (!h || !q || !a) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = h->ctx;
  const int64_t V = ctx->lat.V;
  int rc = set_device(ctx);
  if (!rc) rc = ensure_stage(ctx, sizeof(double2) * 72 * V);
  if (rc) return rc;
  double2 *stg = (double2 *)ctx->d_stage;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(stg, q, sizeof(double2) * 36 * V, cudaMemcpyHostToDevice, ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(stg + 36 * V, a, sizeof(double2) * 36 * V, cudaMemcpyHostToDevice, ctx->stream));
  nrq::launch_prop_f2soa(stg, h->P, V, ctx->stream);
  h->hist_count = 0;
  return check_launch(ctx, "k_prop_f2soa");
}

extern "C" int nrq_heavy_download(const nrq_heavy *h, double *q, double *a) {
  if (!h || !q || !a) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = h->ctx;
  const int64_t V = ctx->lat.V;
  int rc = set_device(ctx);
  if (!rc) rc = ensure_stage(ctx, sizeof(double2) * 72 * V);
  if (rc) return rc;
  double2 *stg = (double2 *)ctx->d_stage;
  nrq::launch_prop_soa2f(h->P, stg, V, ctx->stream);
  if ((rc = check_launch(ctx, "k_prop_soa2f"))) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(q, stg, sizeof(double2) * 36 * V, cudaMemcpyDeviceToHost, ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(a, stg + 36 * V, sizeof(double2) * 36 * V, cudaMemcpyDeviceToHost, ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return NRQ_OK;
}

extern "C" int nrq_heavy_copy(nrq_heavy *dst, const nrq_heavy *src) {
  if (!dst || !src || dst->ctx != src->ctx) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = dst->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(dst->P, src->P, sizeof(double2) * 72 * ctx->lat.V, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
  dst->hist_count = 0;
  return NRQ_OK;
}

extern "C" int nrq_heavy_init_single_point(nrq_heavy *h, int64_t lq, int64_t la) {
  if (!h) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = h->ctx;
  const int64_t V = ctx->lat.V;
  if (lq < 1 || lq > V || la < 1 || la > V) {
    ctx->last_error = "InitSinglePoint: lattice index out of range";
    return NRQ_ERR_BAD_ARG;
  }
  int rc = set_device(ctx);
  if (rc) return rc;
  nrq::launch_single_point(h->P, V, lq - 1, la - 1, ctx->stream);
  h->hist_count = 0;
  return check_launch(ctx, "k_single_point");
}

extern "C" int nrq_heavy_norms(nrq_heavy *h, double *nq, double *na) {
  if (!h) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = h->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  int64_t nb_ = nblk(ctx->lat.V, 256);
  if ((rc = ensure_red(ctx, nb_ * 2))) return rc;
  nrq::launch_norms(h->P, ctx->lat.V, ctx->d_red, nb_, ctx->stream);
  if ((rc = check_launch(ctx, "k_norms"))) return rc;
  if ((rc = reduce_to_host(ctx, nb_, 2, 0u))) return rc;
  if (nq) *nq = std::sqrt(ctx->h_res[0]);
  if (na) *na = std::sqrt(ctx->h_res[1]);
  return NRQ_OK;
}

namespace {
int heavy_correlators(nrq_heavy *h, double out[8], bool gconjg) {
  if (!h || !out) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = h->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  int64_t nb_ = nblk(ctx->lat.V, 128);
  if ((rc = ensure_red(ctx, nb_ * 8))) return rc;
  nrq::launch_correlators(h->P, ctx->lat.V, ctx->d_red, nb_, ctx->stream, gconjg);
  if ((rc = check_launch(ctx, "k_correlators"))) return rc;
  if ((rc = reduce_to_host(ctx, nb_, 8, 0u))) return rc;
  for (int k = 0; k < 8; ++k) out[k] = ctx->h_res[k];
  return NRQ_OK;
}
}  // namespace

extern "C" int nrq_heavy_correlators(nrq_heavy *h, double out[8]) { return heavy_correlators(h, out, false); }

extern "C" int nrq_heavy_correlators_gconjg(nrq_heavy *h, double out[8]) { return heavy_correlators(h, out, true); }

// ====================================================================== CN solver
extern "C" int nrq_cn_init(nrq_ctx *ctx, double mass, const double c[8], double stepwidth, double tol,
                           int64_t maxits, int form, nrq_cn **out) {
  if (!ctx || !c || !out) return NRQ_ERR_BAD_ARG;
  *out = nullptr;
  if (mass == 0.0 || !(tol > 0.0) || maxits < 1 || form < 0 || form > 2) {
    ctx->last_error = "nrq_cn_init: invalid mass, tolerance, maxits or form";
    return NRQ_ERR_BAD_ARG;
  }
  if (form >= 1 && (c[1] != 0.0 || c[3] != 0.0 || c[5] != 0.0 || c[7] != 0.0)) {
    ctx->last_error = "nrq_cn_init: the precision form needs real Wilson coefficients";
    return NRQ_ERR_BAD_ARG;
  }
  int rc = set_device(ctx);
  if (rc) return rc;
  nrq_cn *cn = new (std::nothrow) nrq_cn();
  if (!cn) return NRQ_ERR_OOM;
  cn->ctx = ctx;
  cn->mass = mass;
  for (int k = 0; k < 8; ++k) cn->c[k] = c[k];
  cn->stepwidth = stepwidth;
  cn->tol = tol;
  cn->maxits = maxits;
  cn->form = form;
  const int64_t V = ctx->lat.V;
  cn->nblocks = (V + nrq::CN_SITES_PER_BLOCK - 1) / nrq::CN_SITES_PER_BLOCK;
  bool ok = true;
  auto alloc = [&](void **p, size_t bytes) {
    if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
  };
  alloc((void **)&cn->Dsum, sizeof(double2) * 9 * V);
  alloc((void **)&cn->Bsum, sizeof(double) * 9 * V);
  alloc((void **)&cn->DE, sizeof(double2) * 54 * V);
  for (double2 **pp : {&cn->b, &cn->x, &cn->r, &cn->rh, &cn->p, &cn->v, &cn->t, &cn->s})
    alloc((void **)pp, sizeof(double2) * 72 * V);
  alloc((void **)&cn->scal, kScalBytes);
  alloc((void **)&cn->partials, sizeof(double) * 3 * cn->nblocks * nrq::CN_COLS * 3);
  if (ok && cudaMallocHost((void **)&cn->h_scal, kScalBytes) != cudaSuccess) ok = false;
  if (form >= 1) {
    alloc((void **)&cn->U32, sizeof(float2) * 27 * V);
    alloc((void **)&cn->DE32, sizeof(float2) * 54 * V);
    alloc((void **)&cn->D32, sizeof(float2) * 9 * V);
    alloc((void **)&cn->B32, sizeof(float) * 9 * V);
    for (float2 **pp : {&cn->r32, &cn->dA32, &cn->dB32, &cn->e32}) alloc((void **)pp, sizeof(float2) * 72 * V);
    alloc((void **)&cn->bounds, sizeof(double) * (4 * ((V + 255) / 256) + 8));
    if (ok && cudaMallocHost((void **)&cn->h_bounds, sizeof(double) * 8) != cudaSuccess) ok = false;
  }
  // the TMA-staged stencil needs 16-byte plane strides for the real-valued
  // magnetic planes (V even) and tiles no wider than the lattice
  cn->tma_ok = (V % 2 == 0) && V >= 64;
  cn->stencil = cn->tma_ok ? NRQ_STENCIL_TMA : NRQ_STENCIL_REGISTER;
  if (!ok) {
    cudaGetLastError();
    nrq_cn_finalize(cn);
    ctx->last_error = "nrq_cn_init: device allocation failed";
    return NRQ_ERR_OOM;
  }
  NRQ_CUDA_TRY(ctx, cudaMemsetAsync(cn->scal, 0, kScalBytes, ctx->stream));
  for (double2 *p : {cn->r, cn->v, cn->s})
    NRQ_CUDA_TRY(ctx, cudaMemsetAsync(p, 0, sizeof(double2) * 72 * V, ctx->stream));
  *out = cn;
  return NRQ_OK;
}

extern "C" int nrq_cn_stencil_info(const nrq_cn *cn, int *stencil, double ms[4]) {
  if (!cn) return NRQ_ERR_BAD_ARG;
  if (stencil) *stencil = cn->stencil;
  if (ms)
    for (int k = 0; k < 4; ++k) ms[k] = cn->tune_ms[k];
  return NRQ_OK;
}

extern "C" int nrq_cn_set_wait_test(nrq_cn *cn, int64_t wait_cycles, int stall_load) {
  if (!cn || wait_cycles < 0 || stall_load < -1) return NRQ_ERR_BAD_ARG;
  cn->wait_cycles = wait_cycles > 0 ? (long long)wait_cycles : nrq_wait_cycles_default;
  cn->stall_load = stall_load;
  return NRQ_OK;
}

extern "C" int nrq_cn_set_stencil(nrq_cn *cn, int stencil) {
  if (!cn || stencil < -1 || stencil > NRQ_STENCIL_FMA) return NRQ_ERR_BAD_ARG;
  if (stencil > NRQ_STENCIL_REGISTER && !cn->tma_ok) {
    cn->ctx->last_error = "nrq_cn_set_stencil: tensor maps cannot describe this lattice";
    return NRQ_ERR_BAD_ARG;
  }
  cn->forced_stencil = stencil;
  cn->stencil_tuned = false;
  cn->stencil = stencil >= 0 ? stencil : (cn->tma_ok ? NRQ_STENCIL_TMA : NRQ_STENCIL_REGISTER);
  return NRQ_OK;
}

extern "C" int nrq_cn_set_cheb_stencil(nrq_cn *cn, int which) {
  if (!cn || which < -1 || which > NRQ_CHEB_BLOCKS) return NRQ_ERR_BAD_ARG;
  if (which == NRQ_CHEB_BLOCKS && !nrq::cheb5f_applicable(cn->ctx->lat)) {
    cn->ctx->last_error = "nrq_cn_set_cheb_stencil: the FP32 block step needs V a multiple of 4, V >= 36, nx even";
    return NRQ_ERR_BAD_ARG;
  }
  cn->cheb_stencil = which;
  cn->cheb_tuned = false;
  return NRQ_OK;
}

extern "C" int nrq_cn_cheb_info(const nrq_cn *cn, int *last, double ms[2]) {
  if (!cn) return NRQ_ERR_BAD_ARG;
  if (last) *last = cn->last_cheb;
  if (ms)
    for (int k = 0; k < 2; ++k) ms[k] = cn->cheb_ms[k];
  return NRQ_OK;
}

extern "C" int nrq_cn_set_merged_update(nrq_cn *cn, int on) {
  if (!cn || on < 0 || on > 1) return NRQ_ERR_BAD_ARG;
  cn->merged_update = on != 0;
  return NRQ_OK;
}

extern "C" int nrq_cn_set_true_residual(nrq_cn *cn, int always) {
  if (!cn || always < 0 || always > 1) return NRQ_ERR_BAD_ARG;
  cn->confirm_always = always != 0;
  return NRQ_OK;
}

extern "C" int nrq_cn_true_residual_info(const nrq_cn *cn, int *last_true) {
  if (!cn || !last_true) return NRQ_ERR_BAD_ARG;
  *last_true = cn->last_true ? 1 : 0;
  return NRQ_OK;
}

extern "C" int nrq_cn_set_history_depth(nrq_cn *cn, int depth) {
  if (!cn || depth < 1 || depth > nrq_heavy::kMaxHist) return NRQ_ERR_BAD_ARG;
  cn->history_depth = depth;
  return NRQ_OK;
}

extern "C" int nrq_cn_set_history_guess(nrq_cn *cn, int on) {
  if (!cn || on < 0 || on > 1) return NRQ_ERR_BAD_ARG;
  cn->history_guess = on != 0;
  return NRQ_OK;
}

extern "C" int nrq_cn_finalize(nrq_cn *cn) {
  if (!cn) return NRQ_ERR_NOT_INITIALISED;
  cudaSetDevice(cn->ctx->device);
  cudaStreamSynchronize(cn->ctx->stream);
  for (void *p : {(void *)cn->Dsum, (void *)cn->Bsum, (void *)cn->DE, (void *)cn->b, (void *)cn->x, (void *)cn->r,
                  (void *)cn->rh, (void *)cn->p, (void *)cn->v, (void *)cn->t, (void *)cn->s, (void *)cn->scal,
                  (void *)cn->partials, (void *)cn->U32, (void *)cn->DE32, (void *)cn->D32, (void *)cn->B32,
                  (void *)cn->r32, (void *)cn->dA32, (void *)cn->dB32, (void *)cn->e32, (void *)cn->bounds,
                  (void *)cn->Wblk, (void *)cn->Wblk5, (void *)cn->Wblk5f})
    if (p) cudaFree(p);
  if (cn->h_scal) cudaFreeHost(cn->h_scal);
  if (cn->h_bounds) cudaFreeHost(cn->h_bounds);
  delete cn;
  return NRQ_OK;
}

namespace {
// algorithmic bytes of one 12-column stencil launch, whichever stencil runs:
// vector streams of 12 x 6 complex per site plus the gauge inputs U (432 B)
// and E (192 B) once per species, from which the operator's blocks are
// formed.  Derived data a stencil reads instead (the tensor-core stencil's
// cached blocks) is extra traffic and is not counted.
double mv_bytes(const nrq_ctx *ctx, int mode) {
  // PLAIN, RHS, RES, V, T, RESC, T2, RES2, V2 (the FP32 shadow residual half a stream)
  const double streams[9] = {2, 3, 5, 3, 2, 3, 2.5, 4.5, 2.5};
  return (double)ctx->lat.V * (1152.0 * streams[mode] + 2.0 * (432.0 + 192.0));
}
// the tensor-core stencil's backward blocks are -W^H of the forward ones,
// which holds when every off-diagonal coefficient is imaginary (real
// Wilson coefficients)
bool offdiag_imaginary(const nrq::CnCoef &C) {
  for (int sp = 0; sp < 2; ++sp)
    if (C.kin[sp].re != 0.0 || C.so[sp].re != 0.0) return false;
  return true;
}
// +1 / -1 when the current blocks were built for C / for the coefficients
// whose off-diagonal terms are those of C negated (A vs A^H), 0 otherwise
double blocks_sign(bool valid, const nrq::CnCoef &w, const nrq::CnCoef &C) {
  if (!valid) return 0.0;
  bool same = true, neg = true;
  for (int sp = 0; sp < 2; ++sp) {
    same = same && C.kin[sp].im == w.kin[sp].im && C.so[sp].im == w.so[sp].im;
    neg = neg && C.kin[sp].im == -w.kin[sp].im && C.so[sp].im == -w.so[sp].im;
  }
  return same ? 1.0 : (neg ? -1.0 : 0.0);
}
int ensure_blocks(nrq_cn *cn, const nrq::CnCoef &C, const nrq_gauge *g, double *sign) {
  nrq_ctx *ctx = cn->ctx;
  *sign = blocks_sign(cn->w_valid, cn->w_coef, C);
  if (*sign != 0.0) return NRQ_OK;
  const int64_t V = ctx->lat.V;
  if (!cn->Wblk) NRQ_CUDA_TRY(ctx, cudaMalloc((void **)&cn->Wblk, sizeof(double2) * 216 * V));
  {
    ProfScope ps(ctx, 3, (double)V * (432.0 + 864.0 + 3456.0));
    nrq::launch_cn_blocks(ctx->lat, C, g->U, cn->DE, cn->Wblk, ctx->stream);
  }
  cn->w_coef = C;
  cn->w_valid = true;
  *sign = 1.0;
  return check_launch(ctx, "k_cn_blocks");
}
// whether the precision form's inner steps run on the FP32 blocks: forced,
// or the faster of the two on the first update (before it, the blocks are
// built so that the timing can run)
bool use_cheb5f(const nrq_cn *cn) {
  if (cn->form < 1 || cn->cheb_stencil == NRQ_CHEB_REGISTER || !nrq::cheb5f_applicable(cn->ctx->lat)) return false;
  return cn->cheb_stencil == NRQ_CHEB_BLOCKS || !cn->cheb_tuned || cn->cheb_choice == NRQ_CHEB_BLOCKS;
}
// The FMA stencil's blocks (FP64, f32 = false) or the FP32 Chebyshev step's
// (f32 = true), with the coefficients C.  Where the other precision is
// missing for the same coefficients and the update will need it too, one
// pass writes both.
int ensure_blocks5(nrq_cn *cn, const nrq::CnCoef &C, const nrq_gauge *g, double *sign, bool f32 = false) {
  nrq_ctx *ctx = cn->ctx;
  *sign = f32 ? blocks_sign(cn->w5f_valid, cn->w5f_coef, C) : blocks_sign(cn->w5_valid, cn->w5_coef, C);
  if (*sign != 0.0) return NRQ_OK;
  const int64_t V = ctx->lat.V;
  const bool want64 = !f32 || (cn->stencil == NRQ_STENCIL_FMA && blocks_sign(cn->w5_valid, cn->w5_coef, C) == 0.0);
  const bool want32 = f32 || (use_cheb5f(cn) && blocks_sign(cn->w5f_valid, cn->w5f_coef, C) == 0.0);
  if (want64 && !cn->Wblk5)
    NRQ_CUDA_TRY(ctx, cudaMalloc((void **)&cn->Wblk5, sizeof(double2) * nrq::cn_mv5_block_entries(V)));
  if (want32 && !cn->Wblk5f)
    NRQ_CUDA_TRY(ctx, cudaMalloc((void **)&cn->Wblk5f, sizeof(float2) * nrq::cn_mv5_block_entries(V)));
  {
    ProfScope ps(ctx, 3, (double)V * (432.0 + 864.0 + (want64 ? 3456.0 : 0.0) + (want32 ? 1728.0 : 0.0)));
    nrq::launch_cn_blocks5(ctx->lat, C, g->U, cn->DE, want64 ? cn->Wblk5 : nullptr, want32 ? cn->Wblk5f : nullptr,
                           ctx->stream);
  }
  if (want64) {
    cn->w5_coef = C;
    cn->w5_valid = true;
  }
  if (want32) {
    cn->w5f_coef = C;
    cn->w5f_valid = true;
  }
  *sign = 1.0;
  return check_launch(ctx, "k_cn_blocks5");
}
// The stencil launch of one 12-column application.  The tensor-core stencil
// needs imaginary off-diagonal coefficients and tensor maps; otherwise the
// TMA-staged stencil runs, and without tensor maps the register-tiled one.
// cn->last_stencil records which ran (the partial rows it left).
int mv(nrq_cn *cn, int mode, const nrq::CnCoef &C, const nrq_gauge *g, const nrq::MvArgs &a) {
  nrq_ctx *ctx = cn->ctx;
  if (cn->stencil == NRQ_STENCIL_FMA && offdiag_imaginary(C)) {
    double sign = 0.0;
    int rc = ensure_blocks5(cn, C, g, &sign);
    if (rc) return rc;
    ProfScope ps(ctx, 0, mv_bytes(ctx, mode));
    if (nrq::launch_cn_mv5(mode, ctx->lat, C, sign, cn->Wblk5, cn->Dsum, cn->Bsum, a, scal_err(cn->scal),
                           ctx->sm_count, ctx->stream, cn->wait_cycles, cn->stall_load) == 0) {
      cn->last_stencil = NRQ_STENCIL_FMA;
      return NRQ_OK;
    }
  }
  if (mode == nrq::MV_T2 || mode == nrq::MV_RES2 || mode == nrq::MV_V2) {  // asked for only after an FMA launch
    ctx->last_error = "cn stencil: the merged update needs the FMA stencil";
    return NRQ_ERR_BAD_ARG;
  }
  if (cn->stencil == NRQ_STENCIL_TENSOR && offdiag_imaginary(C)) {
    double sign = 0.0;
    int rc = ensure_blocks(cn, C, g, &sign);
    if (rc) return rc;
    ProfScope ps(ctx, 0, mv_bytes(ctx, mode));
    if (nrq::launch_cn_mv4(mode, ctx->lat, C, sign, cn->Wblk, cn->Dsum, cn->Bsum, a, scal_err(cn->scal),
                           ctx->sm_count, ctx->stream) == 0) {
      cn->last_stencil = NRQ_STENCIL_TENSOR;
      return NRQ_OK;
    }
  }
  ProfScope ps(ctx, 0, mv_bytes(ctx, mode));
  if (cn->tma_ok && cn->stencil != NRQ_STENCIL_REGISTER &&
      nrq::launch_cn_mv3(mode, ctx->lat, C, g->U, cn->Dsum, cn->Bsum, cn->DE, a, scal_err(cn->scal),
                         ctx->sm_count, ctx->stream) == 0) {
    cn->last_stencil = NRQ_STENCIL_TMA;
    return NRQ_OK;
  }
  if (cn->stencil != NRQ_STENCIL_REGISTER) {  // tensor maps unavailable
    cn->tma_ok = false;
    cn->stencil = NRQ_STENCIL_REGISTER;
  }
  nrq::launch_cn_mv(mode, ctx->lat, C, g->U, cn->Dsum, cn->Bsum, cn->DE, a, ctx->stream);
  cn->last_stencil = NRQ_STENCIL_REGISTER;
  return NRQ_OK;
}
// the MV_T input: the register-tiled stencil forms s = r - alpha v on the
// fly, the staged ones read a materialised s
bool mv_t_needs_s(const nrq_cn *cn, const nrq::CnCoef &CH) {
  if ((cn->stencil == NRQ_STENCIL_TENSOR || cn->stencil == NRQ_STENCIL_FMA) && offdiag_imaginary(CH)) return true;
  return cn->tma_ok && cn->stencil != NRQ_STENCIL_REGISTER;
}
void fin(nrq_cn *cn, int stage) {
  nrq_ctx *ctx = cn->ctx;
  // partial rows: one per 32-site block (register-tiled), per (unit, colour
  // warp) (TMA-staged), per CTA (tensor-core)
  int64_t rows = cn->nblocks;
  if (stage <= 2 && cn->last_stencil == NRQ_STENCIL_TMA) rows = 3 * cn->nblocks;
  if (stage <= 2 && cn->last_stencil == NRQ_STENCIL_TENSOR) rows = nrq::cn_mv4_rows(ctx->lat.V, ctx->sm_count);
  if ((stage <= 2 || stage == 5 || stage == 7) && cn->last_stencil == NRQ_STENCIL_FMA)
    rows = nrq::cn_mv5_rows(ctx->lat.V, ctx->sm_count);
  ProfScope ps(ctx, 2, (double)rows * 12 * 3 * 8);
  nrq::launch_cn_finalize(stage, rows, cn->partials, cn->scal, cn->tol, ctx->stream);
}
// Choose the stencil by timing, on this lattice and field, the work each
// does in the solve: for the plain form t = A^H (r - alpha v) (the
// register-tiled stencil forms s on the fly, the staged ones need s
// materialised first); for the precision forms the FP64 refinement
// residual.  Every buffer written here (s, t, the partials, r32, d32) is
// rewritten by the solve before it is read.  The choice minimises the time
// of an update's stencil work (launches per update x time per launch, plus
// the per-update block build of the tensor-core stencil).  A forced stencil
// skips this.
int tune_stencil(nrq_cn *cn, const nrq::CnCoef &CH, const nrq_gauge *g) {
  nrq_ctx *ctx = cn->ctx;
  cn->stencil_tuned = true;
  if (cn->forced_stencil >= 0) {
    cn->stencil = cn->forced_stencil;
    return NRQ_OK;
  }
  if (!cn->tma_ok) return NRQ_OK;  // only the register-tiled stencil applies
  cudaStream_t st = ctx->stream;
  const bool prof = ctx->prof;
  ctx->prof = false;
  const int reps = 3;
  const bool tensor = offdiag_imaginary(CH);
  cudaEvent_t e0, e1;
  NRQ_CUDA_TRY(ctx, cudaEventCreate(&e0));
  NRQ_CUDA_TRY(ctx, cudaEventCreate(&e1));
  int rc = NRQ_OK;
  for (int which = 0; which < 4 && !rc; ++which) {
    cn->tune_ms[which] = -1.0;
    if ((which == NRQ_STENCIL_TENSOR || which == NRQ_STENCIL_FMA) && !tensor) continue;
    cn->stencil = which;
    for (int r = 0; r < reps + 1 && !rc; ++r) {
      if (r == 1) cudaEventRecord(e0, st);
      nrq::MvArgs a{};
      a.partials = cn->partials;
      a.scal = cn->scal;
      if (cn->form == 0) {
        a.out = cn->t;
        if (mv_t_needs_s(cn, CH)) {
          nrq::launch_vec_s(ctx->lat, cn->s, cn->r, cn->v, cn->scal, st);
          a.in = cn->s;
        } else {
          a.in = cn->r;
          a.in2 = cn->v;
        }
        rc = mv(cn, nrq::MV_T, CH, g, a);
      } else {
        a.in = cn->x;
        a.bvec = cn->b;
        a.r32 = cn->r32;
        a.d32 = cn->dA32;
        rc = mv(cn, nrq::MV_RESC, CH, g, a);
      }
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (cn->last_stencil == which) cn->tune_ms[which] = ms / reps;
  }
  // the block stencils also build their blocks once per update: charge that
  // against the launches an update makes (about 10 for the plain BiCGStab
  // solve, 3 for the precision forms: right-hand side and refinement
  // residuals)
  double build_ms[4] = {0.0, 0.0, 0.0, 0.0};
  for (int which : {NRQ_STENCIL_TENSOR, NRQ_STENCIL_FMA}) {
    if (rc || cn->tune_ms[which] <= 0.0) continue;
    double sign = 0.0;
    // a first, untimed build allocates the block sets (once per solver);
    // the timed one is the rebuild every update makes
    rc = which == NRQ_STENCIL_TENSOR ? ensure_blocks(cn, CH, g, &sign) : ensure_blocks5(cn, CH, g, &sign);
    if (rc) continue;
    cudaEventRecord(e0, st);
    if (which == NRQ_STENCIL_TENSOR) {
      cn->w_valid = false;
      rc = ensure_blocks(cn, CH, g, &sign);
    } else {
      cn->w5_valid = false;
      cn->w5f_valid = false;
      rc = ensure_blocks5(cn, CH, g, &sign);
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    build_ms[which] = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->prof = prof;
  if (rc) return rc;
  if ((rc = check_launch(ctx, "stencil tuning"))) return rc;
  const double per_update = cn->form == 0 ? 10.0 : 3.0;
  auto cost = [&](int which) { return per_update * cn->tune_ms[which] + build_ms[which]; };
  int best = NRQ_STENCIL_REGISTER;
  for (int which = 1; which < 4; ++which)
    if (cn->tune_ms[which] > 0.0 && cost(which) < cost(best)) best = which;
  cn->stencil = best;
  return NRQ_OK;
}
int cn_prepare(nrq_cn *cn, const nrq_gauge *g) {
  nrq_ctx *ctx = cn->ctx;
  int rc = gauge_sync64(g);
  if (rc) return rc;
  ProfScope ps(ctx, 3, (double)ctx->lat.V * (432.0 + 192.0));
  nrq::launch_cn_prepare(ctx->lat, g->U, g->E, cn->Dsum, cn->Bsum, cn->DE, ctx->stream);
  cn->w_valid = false;  // the cached blocks follow the new gauge field on demand
  cn->w5_valid = false;
  cn->w5f_valid = false;
  return check_launch(ctx, "k_cn_prepare");
}
}  // namespace

extern "C" int nrq_cn_apply(nrq_cn *cn, const nrq_gauge *g, double mass, const double c[8], double dt, int herm,
                            const nrq_heavy *in, nrq_heavy *out) {
  if (!cn || !g || !c || !in || !out || in == out) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = cn->ctx;
  if (g->ctx != ctx || in->ctx != ctx || out->ctx != ctx || mass == 0.0) return NRQ_ERR_BAD_ARG;
  int rc = set_device(ctx);
  if (!rc) rc = cn_prepare(cn, g);
  if (rc) return rc;
  nrq::CnCoef C = make_coef(ctx, mass, c, dt, herm != 0);
  nrq::MvArgs a{};
  a.in = in->P;
  a.out = out->P;
  if ((rc = mv(cn, nrq::MV_PLAIN, C, g, a))) return rc;
  return check_launch(ctx, "k_cn_mv");
}


using nrqh::ChebSeg;
using nrqh::cheb_gain;
using nrqh::cheb_segment;
namespace {
// The first update's choice between the two FP32 Chebyshev steps: one warm-up
// and three timed launches of each as a first step, reading d = dA32 and
// writing only e32 and dB32 (the r operand pointed at e32 as well), which the
// solve's real first step rewrites before it reads them.
int tune_cheb(nrq_cn *cn, const nrq::CnCoef &CH, const nrq::ChebCoef &K, double wsign) {
  nrq_ctx *ctx = cn->ctx;
  cn->cheb_tuned = true;
  cn->cheb_choice = NRQ_CHEB_REGISTER;
  if (!nrq::cheb5f_applicable(ctx->lat)) return NRQ_OK;
  cudaStream_t st = ctx->stream;
  const bool prof = ctx->prof;
  ctx->prof = false;
  cudaEvent_t e0, e1;
  NRQ_CUDA_TRY(ctx, cudaEventCreate(&e0));
  NRQ_CUDA_TRY(ctx, cudaEventCreate(&e1));
  const int reps = 3;
  for (int which = 0; which < 2; ++which) {
    cn->cheb_ms[which] = -1.0;
    bool ok = true;
    for (int r = 0; r < reps + 1 && ok; ++r) {
      if (r == 1) cudaEventRecord(e0, st);
      if (which == NRQ_CHEB_BLOCKS)
        ok = nrq::launch_cheb5f(true, ctx->lat, CH, wsign, cn->Wblk5f, cn->D32, cn->B32, cn->dA32, cn->dB32, cn->e32,
                                cn->e32, K, scal_err(cn->scal), ctx->sm_count, st, cn->wait_cycles) == 0;
      else
        nrq::launch_cheb32(true, ctx->lat, CH, cn->U32, cn->D32, cn->B32, cn->DE32, cn->dA32, cn->dB32, cn->e32,
                           cn->e32, K, st);
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ok) cn->cheb_ms[which] = ms / reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->prof = prof;
  int rc = check_launch(ctx, "Chebyshev step timing");
  if (rc) return rc;
  if (cn->cheb_ms[NRQ_CHEB_BLOCKS] > 0.0 && cn->cheb_ms[NRQ_CHEB_BLOCKS] < cn->cheb_ms[NRQ_CHEB_REGISTER])
    cn->cheb_choice = NRQ_CHEB_BLOCKS;
  return NRQ_OK;
}

// Precision form: FP64 refinement around FP32 Chebyshev inner solves.
int cn_update_precision(nrq_cn *cn, nrq_heavy *h, const nrq_gauge *g, double mass, const double c[8], double dt,
                        nrq_cn_stats *stats) {
  nrq_ctx *ctx = cn->ctx;
  cudaStream_t st = ctx->stream;
  const nrq::Lat L = ctx->lat;
  const int64_t V = L.V;
  if (c[1] != 0.0 || c[3] != 0.0 || c[5] != 0.0 || c[7] != 0.0) {
    ctx->last_error = "precision form: Wilson coefficients must be real";
    return NRQ_ERR_BAD_ARG;
  }
  const nrq::CnCoef CA = make_coef(ctx, mass, c, dt, false);
  const nrq::CnCoef CH = make_coef(ctx, mass, c, dt, true);
  const double tau = std::fabs(dt) * ctx->a[0] / 2.0;
  int rc = cn_prepare(cn, g);
  if (rc) return rc;
  {
    ProfScope ps(ctx, 3, (double)V * (1080.0 + 540.0));
    nrq::launch_cn_to_f32(V, g->U, cn->DE, cn->Dsum, cn->Bsum, cn->U32, cn->DE32, cn->D32, cn->B32, st);
  }
  // spectral enclosure of H per species
  {
    ProfScope ps(ctx, 3, (double)V * (432.0 + 864.0 + 216.0));
    const int64_t nblk = (V + 255) / 256;
    nrq::launch_cn_bounds(L, CH, dt > 0 ? tau : -tau, g->U, cn->Dsum, cn->Bsum, cn->DE, cn->bounds,
                          cn->bounds + 4 * nblk, st);
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(cn->h_bounds, cn->bounds + 4 * nblk, sizeof(double) * 4,
                                      cudaMemcpyDeviceToHost, st));
  }
  int64_t matvecs = 0, vstreams = 0;
  {  // RHS = A psi ; x0 = 2 RHS - psi
    nrq::MvArgs a{};
    a.in = h->P;
    a.out = cn->b;
    a.out2 = cn->x;
    if ((rc = mv(cn, nrq::MV_RHS, CA, g, a))) return rc;
    matvecs += 1;
    vstreams += 1;
  }
  // learned form: x = 2 RHS - psi + w1 u + w2 v (network), history restarted
  // with the network's part; every refinement correction is added to it
  const bool learned = cn->form == 2 && nrqh::learned_ready(cn->learn);
  // otherwise the plain solve's extrapolated start from the field's history
  const bool hist = !learned && cn->history_guess;
  if (hist && h->hist_count >= 1) {
    const int d = std::min(cn->history_depth, h->hist_count);
    const float2 *t[4] = {hist_v(h, 1), hist_v(h, 2), hist_v(h, 3), hist_v(h, 4)};
    ProfScope ps(ctx, 1, (double)V * (1152.0 * 2 + 576.0 * d));
    nrq::launch_hist_extrapolate(72 * V, cn->x, t, d, st);
    vstreams += 2;
  }
  if (learned) {
    if ((rc = nrqh::ensure_hist(h))) return rc;
    ProfScope ps(ctx, 3, (double)V * (1152.0 * 4 + 576.0 * 6 + 432.0 * 3 + 128.0));
    if ((rc = nrqh::learned_guess(cn->learn, ctx, h->P, cn->b, hist_v1(h), hist_v2(h), hist_next(h), g->U, g->E,
                                  mass, dt, cn->x, st)))
      return rc;
  }
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (learned && (rc = nrqh::learned_check(cn->learn))) return rc;
  if (!cn->stencil_tuned && (rc = tune_stencil(cn, CH, g))) return rc;
  ChebSeg seg[2];
  for (int sp = 0; sp < 2; ++sp) {
    double lo = cn->h_bounds[2 * sp], hi = cn->h_bounds[2 * sp + 1];
    if (!std::isfinite(lo) || !std::isfinite(hi) || hi < lo) {
      ctx->last_error = "precision form: invalid spectral bounds";
      return NRQ_ERR_NONFINITE;
    }
    cn->last_lo[sp] = lo;
    cn->last_hi[sp] = hi;
    // A^H = 1 + i (dt a0/2) H: the sign of dt enters through tau
    seg[sp] = cheb_segment(dt > 0 ? tau : -tau, lo, hi);
  }
  // Chebyshev coefficients along the enclosing segments (the sequence does
  // not depend on how many steps an inner solve takes)
  const int kMaxInner = 40;
  std::vector<nrq::ChebCoef> coef(kMaxInner);
  {
    std::complex<double> rho[2];
    for (int sp = 0; sp < 2; ++sp) rho[sp] = 1.0 / seg[sp].sigma;
    for (int k = 0; k < kMaxInner; ++k)
      for (int sp = 0; sp < 2; ++sp) {
        std::complex<double> rn = 1.0 / (2.0 * seg[sp].sigma - rho[sp]);
        std::complex<double> c1 = rn * rho[sp], c2 = 2.0 * rn / seg[sp].delta;
        coef[k].c1[sp] = {c1.real(), c1.imag()};
        coef[k].c2[sp] = {c2.real(), c2.imag()};
        rho[sp] = rn;
      }
  }
  // smallest inner step count whose guaranteed gain reaches `gain` on both
  // species.  FP32 arithmetic caps one pass at about 1e6; a pass that can
  // finish the solve may aim up to 3e7 (the FP64 check decides whether it did)
  auto inner_steps = [&](double gain) {
    gain = std::max(gain, 10.0);
    if (gain > 3e7) gain = 1e6;
    int m = 1;
    while (m < kMaxInner && std::min(cheb_gain(seg[0].sigma, m), cheb_gain(seg[1].sigma, m)) < gain) ++m;
    return m;
  };
  int status = NRQ_OK;
  double *hs = cn->h_scal;
  int64_t outer = 0, inner = 0;
  bool conv = false;
  double initial = 0.0;
  // the Chebyshev prediction of each column's residual after the last pass
  // (pending: the next residual pass measures it against the true one)
  double pred[nrq::CN_COLS];
  bool pending = false, on_prediction = false;
  cn->last_true = true;
  for (outer = 0; outer < 8; ++outer) {
    nrq::MvArgs a{};
    a.in = cn->x;
    a.bvec = cn->b;
    a.r32 = cn->r32;
    a.d32 = cn->dA32;
    a.partials = cn->partials;
    for (int sp = 0; sp < 2; ++sp) {
      std::complex<double> it = 1.0 / seg[sp].theta;
      a.inv_theta[sp] = {it.real(), it.imag()};
    }
    if ((rc = mv(cn, nrq::MV_RESC, CH, g, a))) return rc;
    fin(cn, 0);
    matvecs += 1;
    vstreams += 3;
    if ((rc = check_launch(ctx, "cn residual"))) return rc;
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(hs, cn->scal, kScalBytes, cudaMemcpyDeviceToHost, st));
    NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (*scal_err(hs) != 0) {
      NRQ_CUDA_TRY(ctx, cudaMemsetAsync(scal_err(cn->scal), 0, 16 * sizeof(int), st));
      ctx->last_error = timeout_message(hs);
      return NRQ_ERR_TIMEOUT;
    }
    bool all = true, nonfin = false;
    for (int k = 0; k < nrq::CN_COLS; ++k) {
      all = all && hs[k * nrq::SC_STRIDE + nrq::SC_CONV] != 0.0;
      nonfin = nonfin || hs[k * nrq::SC_STRIDE + nrq::SC_NONFIN] != 0.0;
      const double *sc = hs + k * nrq::SC_STRIDE;
      if (outer == 0 && sc[nrq::SC_BB] > 0) initial = std::max(initial, std::sqrt(sc[nrq::SC_RR] / sc[nrq::SC_BB]));
    }
    if (nonfin) {
      ctx->last_error = "CN solve: non-finite residual";
      status = NRQ_ERR_NONFINITE;
      break;
    }
    double rel[nrq::CN_COLS];
    for (int kk = 0; kk < nrq::CN_COLS; ++kk) {
      const double *s = hs + kk * nrq::SC_STRIDE;
      rel[kk] = s[nrq::SC_BB] > 0 ? std::sqrt(s[nrq::SC_RR] / s[nrq::SC_BB]) : 0.0;
    }
    if (pending) {  // the true residual beside the prediction of the last pass
      double ratio = 0.0;
      for (int kk = 0; kk < nrq::CN_COLS; ++kk)
        if (pred[kk] > 0.0) ratio = std::max(ratio, rel[kk] / pred[kk]);
      cn->cheb_ratio = std::max(cn->cheb_ratio, ratio);
      cn->cheb_unconfirmed = 0;
      pending = false;
    }
    if (all) {
      conv = true;
      break;
    }
    if (outer == 7) break;
    // gain needed to bring the worst column to 0.3 tol in this pass
    double worst = 0.0;
    for (int kk = 0; kk < nrq::CN_COLS; ++kk) worst = std::max(worst, rel[kk]);
    // maxits bounds the FP32 inner steps of the whole update
    int m = inner_steps(worst / (0.3 * cn->tol));
    if (inner + m > cn->maxits) m = (int)(cn->maxits - inner);
    if (m <= 0) break;
    // FP32 inner Chebyshev solve of A^H e = r, then x += e
    float2 *dcur = cn->dA32, *dnext = cn->dB32;
    double wsign = 0.0;
    if (use_cheb5f(cn) && (rc = ensure_blocks5(cn, CH, g, &wsign, true))) return rc;
    if (cn->cheb_stencil < 0 && !cn->cheb_tuned && (rc = tune_cheb(cn, CH, coef[0], wsign))) return rc;
    const bool blk = use_cheb5f(cn);
    for (int k = 0; k < m; ++k) {
      ProfScope ps(ctx, 0, (double)V * (576.0 * 6 + 756.0));
      if (blk)
        rc = nrq::launch_cheb5f(k == 0, L, CH, wsign, cn->Wblk5f, cn->D32, cn->B32, dcur, dnext, cn->r32, cn->e32,
                                coef[k], scal_err(cn->scal), ctx->sm_count, st, cn->wait_cycles);
      if (!blk || rc) {
        rc = NRQ_OK;
        nrq::launch_cheb32(k == 0, L, CH, cn->U32, cn->D32, cn->B32, cn->DE32, dcur, dnext, cn->r32, cn->e32,
                           coef[k], st);
        cn->last_cheb = NRQ_CHEB_REGISTER;
      } else {
        cn->last_cheb = NRQ_CHEB_BLOCKS;
      }
      std::swap(dcur, dnext);
    }
    inner += m;
    if (learned) {
      ProfScope ps(ctx, 1, (double)V * (1152.0 * 2 + 576.0 * 3));
      nrqh::add_e_hist(72 * V, cn->x, cn->e32, hist_next(h), st);
    } else {
      ProfScope ps(ctx, 1, (double)V * (1152.0 * 2 + 576.0));
      nrq::launch_add_e(72 * V, cn->x, cn->e32, st);
    }
    matvecs += m;
    vstreams += 3;
    // the pass's guaranteed gain per species (quark columns 0-5, antiquark
    // 6-11) predicts each column's residual; where the prediction, scaled by
    // the largest true-to-predicted ratio measured on this solver's
    // confirmed passes and a factor 2, meets the tolerance, the update ends
    // without the confirming residual pass (every 16th such update and the
    // first confirm, and measure the ratio)
    const double g0 = cheb_gain(seg[0].sigma, m), g1 = cheb_gain(seg[1].sigma, m);
    bool predicted = !cn->confirm_always && cn->cheb_ratio >= 0.0 && cn->cheb_unconfirmed < nrq_cn::kReconfirm;
    const double scale = 2.0 * std::max(1.0, cn->cheb_ratio);
    for (int kk = 0; kk < nrq::CN_COLS; ++kk) {
      pred[kk] = rel[kk] / (kk < 6 ? g0 : g1);
      predicted = predicted && pred[kk] * scale <= cn->tol;
    }
    pending = true;
    if (predicted) {
      for (int kk = 0; kk < nrq::CN_COLS; ++kk) pred[kk] *= std::max(1.0, cn->cheb_ratio);
      ++cn->cheb_unconfirmed;
      cn->last_true = false;
      on_prediction = true;
      conv = true;
      ++outer;
      break;
    }
  }
  if (status == NRQ_OK && !conv) status = NRQ_ERR_NOT_CONVERGED;
  bool keep = learned && status == NRQ_OK;
  if (hist && status == NRQ_OK) {  // t = x - (2 RHS - psi) into the history
    if ((rc = nrqh::ensure_hist(h, cn->history_depth))) return rc;
    ProfScope ps(ctx, 1, (double)V * (1152.0 * 3 + 576.0));
    nrq::launch_hist_store(72 * V, cn->x, cn->b, h->P, hist_next(h), st);
    if ((rc = check_launch(ctx, "k_hist_store"))) return rc;
    keep = true;
  }
  std::swap(h->P, cn->x);
  if (keep) hist_push(h);
  else h->hist_count = 0;
  double maxrel = 0.0;
  for (int k = 0; k < nrq::CN_COLS; ++k) {
    const double *s = hs + k * nrq::SC_STRIDE;
    double rel = s[nrq::SC_BB] > 0 ? std::sqrt(s[nrq::SC_RR] / s[nrq::SC_BB]) : 0.0;
    maxrel = std::max(maxrel, on_prediction ? pred[k] : rel);
  }
  cn->last_iterations = inner;
  cn->last_inner = inner;
  cn->last_outer = outer;
  cn->last_matvecs = matvecs;
  cn->last_vecstreams = vstreams;
  if (stats) {
    stats->iterations = inner;
    stats->matvecs = matvecs;
    stats->vector_streams = vstreams;
    stats->max_rel_residual = maxrel;
    stats->converged = conv ? 1 : 0;
    stats->initial_rel_residual = initial;
  }
  return status;
}
}  // namespace

// The per-column recursive relative residuals at a convergence, from the
// scalars read back from the device; half: at the half-step exit, where the
// columns that met the tolerance there have |s| and the others (converged
// before) their last r.
static void recursive_rel(const double *hs, bool half, double rel[nrq::CN_COLS]) {
  for (int k = 0; k < nrq::CN_COLS; ++k) {
    const double *sc = hs + k * nrq::SC_STRIDE;
    const double q = (half && sc[nrq::SC_CONV] == 0.0) ? sc[nrq::SC_SS] : sc[nrq::SC_RR];
    rel[k] = sc[nrq::SC_BB] > 0.0 ? std::sqrt(q / sc[nrq::SC_BB]) : 0.0;
  }
}
// Whether a converged solve may end on its recursive residual: every column's
// plus four times the largest recursive-to-true gap that this solver's
// confirmed solves showed (at least 4 eps of ||b||) meets the tolerance.  The
// gap comes from rounding in the x and r updates (x carries about eps ||A||
// ||x|| per iteration that r does not); it is measured, not assumed.
static bool accept_recursive(const nrq_cn *cn, const double rel[nrq::CN_COLS]) {
  if (cn->confirm_always || cn->gap_rel < 0.0 || cn->since_confirm >= nrq_cn::kReconfirm) return false;
  const double margin = 4.0 * std::max(cn->gap_rel, 4.0 * DBL_EPSILON);
  for (int k = 0; k < nrq::CN_COLS; ++k)
    if (!(rel[k] + margin <= cn->tol)) return false;
  return true;
}

extern "C" int nrq_heavy_update_cn(nrq_cn *cn, nrq_heavy *h, const nrq_gauge *g, double mass, const double c[8],
                                   double dt, nrq_cn_stats *stats) {
  if (!cn || !h || !g || !c) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = cn->ctx;
  if (g->ctx != ctx || h->ctx != ctx || mass == 0.0) return NRQ_ERR_BAD_ARG;
  int rc = set_device(ctx);
  if (rc) return rc;
  if (cn->form >= 1) return cn_update_precision(cn, h, g, mass, c, dt, stats);
  cudaStream_t st = ctx->stream;
  const nrq::Lat L = ctx->lat;
  const nrq::CnCoef CA = make_coef(ctx, mass, c, dt, false);
  const nrq::CnCoef CH = make_coef(ctx, mass, c, dt, true);
  if ((rc = cn_prepare(cn, g))) return rc;
  if (!cn->stencil_tuned && (rc = tune_stencil(cn, CH, g))) return rc;
  int64_t matvecs = 0, vstreams = 0;
  // RHS = A psi ; extrapolated start x0 = 2 RHS - psi
  {
    nrq::MvArgs a{};
    a.in = h->P;
    a.out = cn->b;
    a.out2 = cn->x;
    if ((rc = mv(cn, nrq::MV_RHS, CA, g, a))) return rc;
    matvecs += 1;
    vstreams += 1;  // extra write of x0
  }
  if (cn->history_guess && h->hist_count >= 1) {  // x0 += the extrapolated t of the last steps
    const int d = std::min(cn->history_depth, h->hist_count);
    const float2 *t[4] = {hist_v(h, 1), hist_v(h, 2), hist_v(h, 3), hist_v(h, 4)};
    ProfScope ps(ctx, 1, (double)L.V * (1152.0 * 2 + 576.0 * d));
    nrq::launch_hist_extrapolate(72 * L.V, cn->x, t, d, st);
    vstreams += 2;
  }
  // the merged update on the FMA stencil (the right-hand side ran on it)
  // keeps the shadow residual rh in FP32, in the first half of the rh
  // buffer: any fixed shadow vector serves BiCGStab, and every product
  // with it (rho_0 included) uses the same rounded values
  const bool merged = cn->merged_update && cn->last_stencil == NRQ_STENCIL_FMA;
  float2 *const sh32 = merged ? reinterpret_cast<float2 *>(cn->rh) : nullptr;
  bool restart = true, just_restarted = false;
  bool half_accept = false;  // ended at a half step on the recursive |s|
  // a restart pass confirming a convergence measures the recursive-to-true
  // gap against the recursive residuals of that convergence
  bool gap_pending = false;
  double rec[nrq::CN_COLS];
  int64_t its = 0;
  int status = NRQ_OK;
  double *hs = cn->h_scal;
  double initial = -1.0;  // relative residual of the start, read after the first restart
  // largest relative residual of the unconverged columns at the last read
  // and the reduction of the last iteration; the half-step check runs when
  // the predicted |s| is within kHalfWindow of the tolerance
  double last_rel = 1.0, last_factor = 1e-2;
  constexpr double kHalfWindow = 3.0;
  for (;;) {
    if (restart) {
      nrq::MvArgs a{};
      a.in = cn->x;
      a.bvec = cn->b;
      a.out = cn->r;
      a.out2 = cn->rh;
      a.out3 = cn->p;
      a.sh32 = sh32;
      a.partials = cn->partials;
      if ((rc = mv(cn, merged ? nrq::MV_RES2 : nrq::MV_RES, CH, g, a))) return rc;
      fin(cn, merged ? 7 : 0);
      matvecs += 1;
      vstreams += 3;  // b read, rh and p writes
      restart = false;
      just_restarted = true;
    } else {
      just_restarted = false;
      if (its >= cn->maxits) {
        status = NRQ_ERR_NOT_CONVERGED;
        break;
      }
      nrq::MvArgs a{};
      a.in = cn->p;
      a.in2 = cn->rh;
      a.sh32 = sh32;
      a.out = cn->v;
      a.partials = cn->partials;
      a.scal = cn->scal;
      if ((rc = mv(cn, merged ? nrq::MV_V2 : nrq::MV_V, CH, g, a))) return rc;
      fin(cn, 1);
      const bool tma = mv_t_needs_s(cn, CH);
      // half-step exit: close to the tolerance, |s| = |r - alpha v| is
      // checked before t = A^H s; when every column meets the tolerance
      // there, x += alpha p ends the iteration and the restart pass confirms
      // (predicted |s|: the last residual times the square root of the last
      // pass's reduction, a half step being about half an iteration)
      const bool check_half = tma && last_rel * std::sqrt(last_factor) < kHalfWindow * cn->tol;
      nrq::MvArgs b{};
      if (tma) {  // s = r - alpha v materialised, then t = A^H s
        {
          ProfScope ps(ctx, 1, (double)L.V * 1152.0 * 3);
          nrq::launch_vec_s(L, cn->s, cn->r, cn->v, cn->scal, st, check_half ? cn->partials : nullptr);
        }
        b.in = cn->s;
        vstreams += 3;
        if (check_half) {
          fin(cn, 4);
          if ((rc = check_launch(ctx, "cn half step"))) return rc;
          NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(hs, cn->scal, kScalBytes, cudaMemcpyDeviceToHost, st));
          NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
          bool half = true;
          for (int k = 0; k < nrq::CN_COLS; ++k) {
            const double *sc = hs + k * nrq::SC_STRIDE;
            half = half && (sc[nrq::SC_CONV] != 0.0 || sc[nrq::SC_HALF] != 0.0);
          }
          if (half && *scal_err(hs) == 0) {
            {
              ProfScope ps(ctx, 1, (double)L.V * 1152.0 * 3);
              nrq::launch_vec_xp(L, cn->x, cn->p, cn->scal, st);
            }
            matvecs += 1;
            vstreams += 3;
            ++its;
            // the same acceptance as below, on |s| for the columns that met
            // the tolerance here
            recursive_rel(hs, true, rec);
            if (accept_recursive(cn, rec)) {
              half_accept = true;
              cn->last_true = false;
              ++cn->since_confirm;
              if ((rc = check_launch(ctx, "cn half step"))) return rc;
              break;
            }
            gap_pending = true;
            restart = true;
            continue;
          }
        }
      } else {    // s formed on the fly inside the stencil
        b.in = cn->r;
        b.in2 = cn->v;
      }
      b.out = cn->t;
      b.partials = cn->partials;
      b.scal = cn->scal;
      // the merged update: the t launch also reduces rh.t, which gives beta
      // before r is formed, so that x, r and p are updated in one pass
      b.sh32 = sh32;
      if ((rc = mv(cn, merged ? nrq::MV_T2 : nrq::MV_T, CH, g, b))) return rc;
      if (merged) {
        fin(cn, 5);
        {
          ProfScope ps(ctx, 1, (double)L.V * 1152.0 * 8);
          nrq::launch_vec_xrp(L, cn->x, cn->r, cn->p, cn->s, cn->t, cn->v, cn->scal, cn->partials, st);
        }
        fin(cn, 6);
        vstreams += 1 + 1 + 8;  // rh read by the v and t launches, the merged pass
      } else {
        fin(cn, 2);
        if (tma) {
          ProfScope ps(ctx, 1, (double)L.V * 1152.0 * 7);
          nrq::launch_vec_xr_s(L, cn->x, cn->r, cn->p, cn->s, cn->t, cn->rh, cn->scal, cn->partials, st);
          vstreams -= 1;
        } else {
          ProfScope ps(ctx, 1, (double)L.V * 1152.0 * 8);
          nrq::launch_vec_xr(L, cn->x, cn->r, cn->p, cn->v, cn->t, cn->rh, cn->scal, cn->partials, st);
        }
        fin(cn, 3);
        {
          ProfScope ps(ctx, 1, (double)L.V * 1152.0 * 4);
          nrq::launch_vec_p(L, cn->p, cn->r, cn->v, cn->scal, st);
        }
        vstreams += 1 + 1 + 8 + 4;
      }
      matvecs += 2;
      ++its;
    }
    if ((rc = check_launch(ctx, "cn iteration"))) return rc;
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(hs, cn->scal, kScalBytes, cudaMemcpyDeviceToHost, st));
    NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (*scal_err(hs) != 0) {
      status = NRQ_ERR_TIMEOUT;
      ctx->last_error = timeout_message(hs);
      NRQ_CUDA_TRY(ctx, cudaMemsetAsync(scal_err(cn->scal), 0, 16 * sizeof(int), st));
      break;
    }
    {
      double rel = 0.0;
      for (int k = 0; k < nrq::CN_COLS; ++k) {
        const double *s = hs + k * nrq::SC_STRIDE;
        if (s[nrq::SC_BB] > 0 && s[nrq::SC_CONV] == 0.0)
          rel = std::max(rel, std::sqrt(s[nrq::SC_RR] / s[nrq::SC_BB]));
      }
      // reduction of the last full iteration (a restart keeps the previous one)
      if (!just_restarted && last_rel > 0.0 && rel > 0.0) last_factor = std::min(1.0, rel / last_rel);
      last_rel = rel;
    }
    if (initial < 0.0) {
      initial = 0.0;
      for (int k = 0; k < nrq::CN_COLS; ++k) {
        const double *s = hs + k * nrq::SC_STRIDE;
        if (s[nrq::SC_BB] > 0) initial = std::max(initial, std::sqrt(s[nrq::SC_RR] / s[nrq::SC_BB]));
      }
    }
    bool all = true, brk = false, nonfin = false;
    for (int k = 0; k < nrq::CN_COLS; ++k) {
      const double *s = hs + k * nrq::SC_STRIDE;
      all = all && s[nrq::SC_CONV] != 0.0;
      brk = brk || s[nrq::SC_BREAK] != 0.0;
      nonfin = nonfin || s[nrq::SC_NONFIN] != 0.0;
    }
    if (nonfin) {
      status = NRQ_ERR_NONFINITE;
      ctx->last_error = "CN solve: non-finite residual";
      break;
    }
    if (just_restarted && gap_pending) {  // the true residual beside the recursive one
      double gap = 0.0;
      for (int k = 0; k < nrq::CN_COLS; ++k) {
        const double *sc = hs + k * nrq::SC_STRIDE;
        if (sc[nrq::SC_BB] > 0.0) gap = std::max(gap, std::fabs(std::sqrt(sc[nrq::SC_RR] / sc[nrq::SC_BB]) - rec[k]));
      }
      cn->gap_rel = std::max(cn->gap_rel, gap);
      cn->since_confirm = 0;
      gap_pending = false;
    }
    if (all) {
      // every column below tolerance: accept once a true residual b - A^H x
      // (the restart pass) confirms it, or at once on the recursive residual
      // where it meets the tolerance with the measured margin (PETSc's KSP
      // tests its recursive residual alone); otherwise recompute it first
      if (just_restarted) {
        cn->last_true = true;
        break;
      }
      recursive_rel(hs, false, rec);
      if (accept_recursive(cn, rec)) {
        cn->last_true = false;
        ++cn->since_confirm;
        break;
      }
      gap_pending = true;
      restart = true;
      continue;
    }
    if (brk) restart = true;
  }
  // the step's correction to the extrapolated start goes into the history
  // (history_guess), otherwise a plain step leaves none
  bool keep = false;
  if (cn->history_guess && status == NRQ_OK) {
    if ((rc = nrqh::ensure_hist(h, cn->history_depth))) return rc;
    ProfScope ps(ctx, 1, (double)L.V * (1152.0 * 3 + 576.0));
    nrq::launch_hist_store(72 * L.V, cn->x, cn->b, h->P, hist_next(h), st);
    if ((rc = check_launch(ctx, "k_hist_store"))) return rc;
    keep = true;
  }
  // result -> propagator (swap buffers)
  std::swap(h->P, cn->x);
  if (keep) hist_push(h);
  else h->hist_count = 0;
  double maxrel = 0.0;
  bool conv = true;
  for (int k = 0; k < nrq::CN_COLS; ++k) {
    const double *s = hs + k * nrq::SC_STRIDE;
    const bool at_half = half_accept && s[nrq::SC_CONV] == 0.0;  // met the tolerance at the half step
    const double q = at_half ? s[nrq::SC_SS] : s[nrq::SC_RR];
    double rel = s[nrq::SC_BB] > 0 ? std::sqrt(q / s[nrq::SC_BB]) : 0.0;
    maxrel = std::max(maxrel, rel);
    conv = conv && (s[nrq::SC_CONV] != 0.0 || (at_half && s[nrq::SC_HALF] != 0.0));
  }
  cn->last_iterations = its;
  cn->last_matvecs = matvecs;
  cn->last_vecstreams = vstreams;
  if (stats) {
    stats->iterations = its;
    stats->matvecs = matvecs;
    stats->vector_streams = vstreams;
    stats->max_rel_residual = maxrel;
    stats->converged = conv ? 1 : 0;
    stats->initial_rel_residual = std::max(initial, 0.0);
  }
  return status;
}
