// Learned initial guess of the Crank-Nicolson solve (form 2), its training
// and its C ABI (nrq_learn_*).
//
// The reference's solve starts from zero (PETSc KSP, src/nrqcd.f90:1108-1123,
// without KSPSetInitialGuessNonzero); the plain and precision forms here
// start from x0 = 2 RHS - psi plus the polynomial extrapolation of the
// field's last corrections.  The learned form adds, per sample (site, species),
//   x0 = 2 b - psi + w1 u + w2 v,   u = b - psi,   v = history,
// where the history v = x_prev - (2 b_prev - psi_prev) is what the
// extrapolation missed in the previous step and (w1, w2) complex come from a
// per-sample MLP (16 -> 64 -> 64 -> 4, ReLU) of local invariants of the
// right-hand side and of the gauge field (plaquettes, E^2).  The network is
// trained on the method's own solves: the loss is the squared error of the
// guess, which per sample only needs the Gram statistics of (u, v, t),
// t = x - (2 b - psi).
//
// The dense layers run on the 5th-generation tensor cores: BF16 operands in
// shared memory (no-swizzle K-major tiles), FP32 accumulators in tensor
// memory, one elected thread issuing tcgen05.mma and committing to an
// mbarrier, tcgen05.ld for the epilogues.  The guess runs as four kernels:
// gauge invariants per site, features per sample (both streaming, high
// occupancy), the three layers on the tensor cores (persistent, 128-sample
// tiles), and the construction of x0 (streaming).  The training kernel runs
// forward and backward for 128 samples per CTA and writes per-CTA gradient
// partials that a second kernel reduces in a fixed order and feeds to Adam.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/nrqcd_b200.h"
#include "nrq_internal.h"
#include "nrq_kernels.cuh"
#include "tc.cuh"

using nrqh::check_launch;
using nrqh::set_device;

namespace nrq {
namespace learn {

constexpr int NIN = 16, NH = 64, NOUT = 6, NOUTP = 16;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NIN, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NOUT * NH, NPARAMS = OFF_B3 + 6 * NOUT;
constexpr int NGROUP = 6;  // output-bias groups: species (2) x history depth (0, 1, 2)
static_assert(NPARAMS == NRQ_LEARN_NPARAMS, "parameter count");
constexpr int NSTATS = 16;  // Gram statistics of (u, v1, v2; t)
constexpr int TILE = 128;              // samples per CTA tile (tensor memory lanes)
constexpr uint32_t kSpins = 1u << 24;  // bounded mbarrier polls

// device-side model: BF16 weights [out][in] row-major, FP32 biases; the
// output bias b3[group][6] is per species and history depth, read from
// features 9 (species sign) and 10 (depth / 2)
struct Model {
  const __nv_bfloat16 *w1, *w2, *w3;  // 64x16, 64x64, 6x64
  const float *b1, *b2, *b3;          // 64, 64, 6x6
};
constexpr int FEAT_SPECIES = 9, FEAT_DEPTH = 10;
__device__ __forceinline__ int bias_group(float fspecies, float fdepth) {
  const int d = (int)rintf(2.f * fdepth);
  return (fspecies < 0.f ? 3 : 0) + (d < 0 ? 0 : (d > 2 ? 2 : d));
}

// ------------------------------------------------------------ features
// Gauge invariants of site s (species independent): 1 - Re Tr P_ij / 3 for
// the planes (x,y), (y,z), (z,x) and sum_a,i E^a_i(s)^2.
__global__ void k_learn_gauge_features(Lat L, const double2 *__restrict__ U, const double *__restrict__ E,
                                       float4 *__restrict__ gf) {
  const int64_t V = L.V;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  float out[4];
#pragma unroll 1
  for (int pl = 0; pl < 3; ++pl) {
    const int i = pl, j = (pl + 1) % 3;
    const m3 a = mul(load_link(U, V, s, i), load_link(U, V, nb(L, s, i, +1), j));
    const m3 c = mul(load_link(U, V, s, j), load_link(U, V, nb(L, s, j, +1), i));
    double tr = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) tr += a.e[k].re * c.e[k].re + a.e[k].im * c.e[k].im;
    out[pl] = (float)(1.0 - tr / 3.0);
  }
  double e2 = 0.0;
#pragma unroll 4
  for (int k = 0; k < 24; ++k) {
    const double e = __ldg(E + (int64_t)k * V + s);
    e2 += e * e;
  }
  out[3] = (float)e2;
  gf[s] = make_float4(out[0], out[1], out[2], out[3]);
}

// 16 features of sample (site s, species sp); the oracle restates them.
// v1 = the last step's miss, v2 = the one before (null when absent).
__device__ void sample_features(const Lat &L, const double2 *__restrict__ psi, const double2 *__restrict__ b,
                                const float2 *__restrict__ v1, const float2 *__restrict__ v2,
                                const float4 *__restrict__ gf, double mass, double tau, int64_t s, int sp,
                                float f[NIN]) {
  const int64_t V = L.V;
  double nps = 0, nu = 0, n1 = 0, n2 = 0;
  cplx cpu = {0, 0}, cu1 = {0, 0}, c21 = {0, 0};
  const int64_t base = (int64_t)(sp * 36) * V + s;
#pragma unroll 6
  for (int k = 0; k < 36; ++k) {
    const int64_t o = base + (int64_t)k * V;
    const cplx p = ldg(psi + o);
    const cplx u = ldg(b + o) - p;
    cplx h1 = {0.0, 0.0}, h2 = {0.0, 0.0};
    if (v1) {
      const float2 h = __ldg(v1 + o);
      h1 = {(double)h.x, (double)h.y};
    }
    if (v2) {  // plain load: the record kernel overwrites v2 with the new history
      const float2 h = v2[o];
      h2 = {(double)h.x, (double)h.y};
    }
    nps += norm2(p);
    nu += norm2(u);
    n1 += norm2(h1);
    n2 += norm2(h2);
    cmac_cj(cpu, p, u);
    cmac_cj(cu1, u, h1);
    cmac_cj(c21, h2, h1);
  }
#pragma unroll
  for (int i = 0; i < NIN; ++i) f[i] = 0.f;
  if (nps > 0) {
    f[0] = (float)(cpu.re / (nps * tau));
    f[1] = (float)(cpu.im / (nps * tau));
    f[2] = (float)(sqrt(nu / nps) / fabs(tau));
  }
  if (nu > 0 && n1 > 0) {
    const double den = sqrt(nu * n1);
    f[3] = (float)(cu1.re / den);
    f[4] = (float)(cu1.im / den);
    f[5] = (float)fmin(sqrt(n1 / nu) / fabs(tau), 50.0);
  }
  if (n1 > 0 && n2 > 0) {
    const double den = sqrt(n1 * n2);
    f[6] = (float)(c21.re / den);
    f[7] = (float)(c21.im / den);
    f[8] = (float)fmin(sqrt(n1 / n2), 10.0);
  }
  f[9] = sp == 0 ? 1.f : -1.f;
  f[10] = 0.5f * ((v1 ? 1.f : 0.f) + (v2 ? 1.f : 0.f));
  const float4 g = __ldg(gf + s);
  f[11] = g.x;
  f[12] = g.y;
  f[13] = g.z;
  f[14] = g.w;
  f[15] = (float)(1.0 / mass);
}

// features of every sample (row sp*V + s of feat)
__global__ void __launch_bounds__(256) k_learn_features(Lat L, const double2 *__restrict__ psi,
                                                        const double2 *__restrict__ b,
                                                        const float2 *__restrict__ v1,
                                                        const float2 *__restrict__ v2,
                                                        const float4 *__restrict__ gf, double mass, double tau,
                                                        float *__restrict__ feat) {
  const int64_t V = L.V;
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= 2 * V) return;
  float f[NIN];
  sample_features(L, psi, b, v1, v2, gf, mass, tau, q % V, (int)(q / V), f);
  float4 *o = reinterpret_cast<float4 *>(feat + q * NIN);
#pragma unroll
  for (int k = 0; k < NIN / 4; ++k) o[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
}

// x = 2b - psi + w0 s0 u + w1 v1 + w2 v2 and hnew = w0 s0 u + w1 v1 + w2 v2
// (s0 = |tau| scales u, which is O(tau H psi), to the size of the misses),
// one thread per element of the 72 planes; w of sample (sp*V + s) from omega
// (8 floats per sample).  hnew may be the v2 buffer (read before written).
__global__ void k_learn_apply(int64_t V, const double2 *__restrict__ psi, const double2 *__restrict__ b,
                              const float2 *v1, const float2 *v2, const float4 *__restrict__ omega, double s0,
                              float2 *hnew, double2 *__restrict__ x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 72 * V) return;
  const int64_t plane = i / V, s = i - plane * V;
  const int sp = plane >= 36;
  const float4 wa = __ldg(omega + 2 * (sp * V + s)), wb = __ldg(omega + 2 * (sp * V + s) + 1);
  const cplx p = ldg(psi + i), bb = ldg(b + i);
  cplx d = (s0 * cplx{wa.x, wa.y}) * (bb - p);
  if (v1) {
    const float2 h = v1[i];
    d = d + cplx{wa.z, wa.w} * cplx{(double)h.x, (double)h.y};
  }
  if (v2) {
    const float2 h = v2[i];
    d = d + cplx{wb.x, wb.y} * cplx{(double)h.x, (double)h.y};
  }
  const cplx x0 = 2.0 * bb - p + d;
  x[i] = make_double2(x0.re, x0.im);
  hnew[i] = make_float2((float)d.re, (float)d.im);
}

// batched guess over the fields of a batch table: sample q of field f is
// row f*2V + q of feat / omega
__global__ void __launch_bounds__(256) k_batch_learn_features(Lat L, const BatchField *__restrict__ tab,
                                                              const float4 *__restrict__ gf,
                                                              float *__restrict__ feat) {
  const int64_t V = L.V;
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= 2 * V) return;
  const BatchField &f = tab[blockIdx.y];
  float v[NIN];
  sample_features(L, f.psi, f.b, f.h1, f.h2, gf, f.mass, f.tau, q % V, (int)(q / V), v);
  float4 *o = reinterpret_cast<float4 *>(feat + ((int64_t)blockIdx.y * 2 * V + q) * NIN);
#pragma unroll
  for (int k = 0; k < NIN / 4; ++k) o[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

__global__ void k_batch_learn_apply(int64_t V, const BatchField *__restrict__ tab,
                                    const float4 *__restrict__ omega) {
  const BatchField &f = tab[blockIdx.y];
  const float4 *om = omega + (int64_t)blockIdx.y * 2 * V * 2;
  const double s0 = fabs(f.tau);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 72 * V; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t plane = i / V, s = i - plane * V;
    const int sp = plane >= 36;
    const float4 wa = __ldg(om + 2 * (sp * V + s)), wb = __ldg(om + 2 * (sp * V + s) + 1);
    const cplx p = ldg(f.psi + i), bb = ldg(f.b + i);
    cplx d = (s0 * cplx{wa.x, wa.y}) * (bb - p);
    if (f.h1) {
      const float2 h = f.h1[i];
      d = d + cplx{wa.z, wa.w} * cplx{(double)h.x, (double)h.y};
    }
    if (f.h2) {
      const float2 h = f.h2[i];
      d = d + cplx{wb.x, wb.y} * cplx{(double)h.x, (double)h.y};
    }
    const cplx x0 = 2.0 * bb - p + d;
    f.x[i] = make_double2(x0.re, x0.im);
    f.hnew[i] = make_float2((float)d.re, (float)d.im);
  }
}

// ------------------------------------------------------------ shared staging
__device__ __forceinline__ void st_bf16(uint8_t *tile, int r, int k, int R, float x) {
  *reinterpret_cast<__nv_bfloat16 *>(tile + tc::kmajor_offset(r, k, R)) = __float2bfloat16_rn(x);
}
__device__ __forceinline__ float ld_bf16(const uint8_t *tile, int r, int k, int R) {
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(tile + tc::kmajor_offset(r, k, R)));
}

// weights as B operands (rows = output features, K = input features)
__device__ void stage_weights(const Model &M, uint8_t *W1s, uint8_t *W2s, uint8_t *W3s, float *bs) {
  for (int e = threadIdx.x; e < NH * NIN; e += blockDim.x) {
    const int r = e / NIN, k = e % NIN;
    *reinterpret_cast<__nv_bfloat16 *>(W1s + tc::kmajor_offset(r, k, NH)) = M.w1[e];
  }
  for (int e = threadIdx.x; e < NH * NH; e += blockDim.x) {
    const int r = e / NH, k = e % NH;
    *reinterpret_cast<__nv_bfloat16 *>(W2s + tc::kmajor_offset(r, k, NH)) = M.w2[e];
  }
  for (int e = threadIdx.x; e < NOUTP * NH; e += blockDim.x) {
    const int r = e / NH, k = e % NH;
    *reinterpret_cast<__nv_bfloat16 *>(W3s + tc::kmajor_offset(r, k, NOUTP)) =
        r < NOUT ? M.w3[r * NH + k] : __float2bfloat16_rn(0.f);
  }
  for (int e = threadIdx.x; e < NH; e += blockDim.x) {
    bs[e] = M.b1[e];
    bs[NH + e] = M.b2[e];
  }
  for (int e = threadIdx.x; e < NGROUP * NOUTP; e += blockDim.x) {
    const int gr = e / NOUTP, j = e % NOUTP;
    bs[2 * NH + e] = j < NOUT ? M.b3[gr * NOUT + j] : 0.f;
  }
}

// Wait for the MMAs committed to `bar`; the outcome is made uniform over the
// CTA (the tensor-memory loads that follow are warp-collective).  On expiry
// the error is recorded and the phase is kept, so that drain() can wait for
// the same completion once more before the tensor memory is released.
__device__ __forceinline__ bool wait_mma(uint64_t *bar, uint32_t &phase, int *err) {
  bool ok = tc::mbar_wait_bounded(bar, phase, kSpins);
  ok = __syncthreads_and(ok) != 0;
  if (ok) phase ^= 1u;
  else if (threadIdx.x == 0 && err) atomicExch(err, NRQ_ERR_TIMEOUT);
  tc::fence_after_sync();
  return ok;
}
// after an expired wait: wait (bounded) for the outstanding commit
__device__ __forceinline__ void drain(uint64_t *bar, uint32_t phase, bool ok) {
  if (!ok) tc::mbar_wait_bounded(bar, phase, kSpins);
}
// barrier initialisation visible to the tensor core's commit
__device__ __forceinline__ void init_bar(uint64_t *bar) {
  tc::mbar_init(bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// hidden layer epilogue: 64 accumulator columns of this thread's lane +
// bias, ReLU, BF16 into the activation tile row `row`
__device__ __forceinline__ void hidden_epilogue(uint32_t tbase, const float *bias, uint8_t *Hs, int row) {
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int c0 = 0; c0 < NH; c0 += 16) {
    float v[16];
    tc::tmem_ld16(tc::tmem_addr(tbase, 32 * warp, c0), v);
#pragma unroll
    for (int j = 0; j < 16; ++j) st_bf16(Hs, row, c0 + j, TILE, fmaxf(v[j] + bias[c0 + j], 0.f));
  }
}

// issue layer MMAs (thread 0) after every thread's operand writes
__device__ __forceinline__ void sync_operands() {
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

// forward of the tile whose features sit in Xs; returns the 4 outputs of
// this thread's sample.  `ok` turns false after an expired wait.
__device__ void forward_tile(uint32_t tbase, uint8_t *Xs, uint8_t *Hs, uint8_t *W1s, uint8_t *W2s, uint8_t *W3s,
                             const float *bs, uint64_t *bar, uint32_t &phase, int *err, bool &ok, int grp,
                             float y[NOUT]) {
  const int t = threadIdx.x;
  sync_operands();
  if (t == 0 && ok) {
    tc::mma_bf16(tbase, tc::smem_desc(tc::smem_u32(Xs), TILE, 0), tc::smem_desc(tc::smem_u32(W1s), NH, 0),
                 tc::idesc_bf16_f32(TILE, NH), false);
    tc::mma_commit(bar);
  }
  ok = ok && wait_mma(bar, phase, err);
  if (ok) hidden_epilogue(tbase, bs, Hs, t);
  sync_operands();
  if (t == 0 && ok) {
    for (int s = 0; s < NH / 16; ++s)
      tc::mma_bf16(tbase, tc::smem_desc(tc::smem_u32(Hs), TILE, s), tc::smem_desc(tc::smem_u32(W2s), NH, s),
                   tc::idesc_bf16_f32(TILE, NH), s > 0);
    tc::mma_commit(bar);
  }
  ok = ok && wait_mma(bar, phase, err);
  if (ok) hidden_epilogue(tbase, bs + NH, Hs, t);
  sync_operands();
  if (t == 0 && ok) {
    for (int s = 0; s < NH / 16; ++s)
      tc::mma_bf16(tbase, tc::smem_desc(tc::smem_u32(Hs), TILE, s), tc::smem_desc(tc::smem_u32(W3s), NOUTP, s),
                   tc::idesc_bf16_f32(TILE, NOUTP), s > 0);
    tc::mma_commit(bar);
  }
  ok = ok && wait_mma(bar, phase, err);
  float v[16];
  if (ok) {
    tc::tmem_ld16(tc::tmem_addr(tbase, 32 * (t >> 5), 0), v);
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = 0.f;
  }
#pragma unroll
  for (int j = 0; j < NOUT; ++j) y[j] = ok ? v[j] + bs[2 * NH + grp * NOUTP + j] : 0.f;
  tc::fence_before_sync();
  __syncthreads();
}

// shared memory of the forward kernels
struct FwdSmem {
  alignas(128) uint8_t W1s[NH * NIN * 2];
  alignas(128) uint8_t W2s[NH * NH * 2];
  alignas(128) uint8_t W3s[NOUTP * NH * 2];
  alignas(128) uint8_t Xs[TILE * NIN * 2];
  alignas(128) uint8_t Hs[TILE * NH * 2];
  float bs[2 * NH + NGROUP * NOUTP];
  uint64_t bar;
  uint32_t tslot;
};

// ------------------------------------------------------------ inference
// MLP outputs of n samples (persistent over tiles of 128): row i of out
// (stride ostride) = (Re w0, Im w0, Re w1, Im w1, Re w2, Im w2) of feature row i
__global__ void __launch_bounds__(TILE, 1)
    k_learn_forward(Model M, const float *__restrict__ feat, int64_t n, float *__restrict__ out, int ostride,
                    int *err) {
  __shared__ FwdSmem sm;
  const int t = threadIdx.x;
  if (t < 32) tc::tmem_alloc(&sm.tslot, 64);
  if (t == 0) init_bar(&sm.bar);
  stage_weights(M, sm.W1s, sm.W2s, sm.W3s, sm.bs);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = sm.tslot;
  uint32_t phase = 0;
  bool ok = true;
  const int64_t ntiles = (n + TILE - 1) / TILE;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t i = tile * TILE + t;
#pragma unroll
    for (int k = 0; k < NIN; ++k) st_bf16(sm.Xs, t, k, TILE, i < n ? feat[i * NIN + k] : 0.f);
    const int grp = i < n ? bias_group(feat[i * NIN + FEAT_SPECIES], feat[i * NIN + FEAT_DEPTH]) : 0;
    float y[NOUT];
    forward_tile(tbase, sm.Xs, sm.Hs, sm.W1s, sm.W2s, sm.W3s, sm.bs, &sm.bar, phase, err, ok, grp, y);
    if (i < n)
      for (int k = 0; k < NOUT; ++k) out[i * ostride + k] = y[k];
  }
  drain(&sm.bar, phase, ok);
  tc::fence_before_sync();
  __syncthreads();
  if (t < 32) tc::tmem_dealloc(tbase, 64);
}

// ------------------------------------------------------------ training
struct TrainSmem {
  alignas(128) uint8_t W1s[NH * NIN * 2];    // B of layer 1: [64 x 16]
  alignas(128) uint8_t W2s[NH * NH * 2];     // B of layer 2: [64 x 64]
  alignas(128) uint8_t W3s[NOUTP * NH * 2];  // B of layer 3: [16 x 64]
  alignas(128) uint8_t W2Ts[NH * NH * 2];    // B of dH1 = dH2 W2: [in 64 x out 64]
  alignas(128) uint8_t W3Ts[NH * NOUTP * 2]; // B of dH2 = dY W3: [in 64 x out 16]
  alignas(128) uint8_t Xs[TILE * NIN * 2];
  alignas(128) uint8_t H1s[TILE * NH * 2];
  alignas(128) uint8_t H2s[TILE * NH * 2];
  alignas(128) uint8_t Gs[TILE * NH * 2];    // gradient A operand (dY or dH)
  alignas(128) uint8_t TA[TILE * TILE * 2];  // transposed activations [in (pad 128) x samples]
  alignas(128) uint8_t TB[NH * TILE * 2];    // transposed gradients [out x samples]
  float bs[2 * NH + NGROUP * NOUTP];
  float red[4][NH];                          // per-warp bias-gradient partials
  float lred[4];
  uint64_t bar;
  uint32_t tslot;
};

// column sums over the CTA's 128 samples of 64 per-thread values, added to g
// in a fixed order (warp shuffles, then the 4 warp partials)
__device__ void column_sums(float (&vals)[NH], TrainSmem &sm, float *g) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NH; ++c) {
    float v = vals[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sm.red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < NH) g[threadIdx.x] = sm.red[0][threadIdx.x] + sm.red[1][threadIdx.x] + sm.red[2][threadIdx.x] +
                                         sm.red[3][threadIdx.x];
  __syncthreads();
}

// One CTA: forward and backward of 128 samples, gradient partial of this
// CTA into gpart[cta][NPARAMS], loss partial into lpart[cta].  Samples are
// idx[i] (or i when idx == nullptr) of the dataset, i in [cta*128, +128) < n.
// scale = 1 / batch size.
__global__ void __launch_bounds__(TILE, 1)
    k_learn_train(Model M, const float *__restrict__ feat, const float *__restrict__ stats,
                  const int64_t *__restrict__ idx, int64_t n, float scale, float *__restrict__ gpart,
                  float *__restrict__ lpart, int *err) {
  extern __shared__ __align__(1024) uint8_t smraw[];
  TrainSmem &sm = *reinterpret_cast<TrainSmem *>(smraw);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (t < 32) tc::tmem_alloc(&sm.tslot, 256);
  if (t == 0) init_bar(&sm.bar);
  stage_weights(M, sm.W1s, sm.W2s, sm.W3s, sm.bs);
  // transposed weights for the input gradients
  for (int e = t; e < NH * NH; e += TILE) {
    const int o = e / NH, i = e % NH;  // W2[o][i]
    *reinterpret_cast<__nv_bfloat16 *>(sm.W2Ts + tc::kmajor_offset(i, o, NH)) = M.w2[e];
  }
  for (int e = t; e < NH * NOUTP; e += TILE) {
    const int i = e / NOUTP, o = e % NOUTP;
    *reinterpret_cast<__nv_bfloat16 *>(sm.W3Ts + tc::kmajor_offset(i, o, NH)) =
        o < NOUT ? M.w3[o * NH + i] : __float2bfloat16_rn(0.f);
  }
  for (int e = t; e < TILE * TILE; e += TILE) *reinterpret_cast<__nv_bfloat16 *>(sm.TA + 2 * e) = 0;
  const int64_t i = (int64_t)blockIdx.x * TILE + t;
  const bool active = i < n;
  const int64_t si = active ? (idx ? idx[i] : i) : 0;
  float f[NIN], st[NSTATS];
#pragma unroll
  for (int k = 0; k < NIN; ++k) f[k] = active ? feat[si * NIN + k] : 0.f;
#pragma unroll
  for (int k = 0; k < NSTATS; ++k) st[k] = active ? stats[si * NSTATS + k] : 0.f;
#pragma unroll
  for (int k = 0; k < NIN; ++k) st_bf16(sm.Xs, t, k, TILE, f[k]);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tb = sm.tslot;
  uint32_t phase = 0;
  bool ok = true;
  float y[NOUT];
  // forward (layer 1 activations go to H1s and stay there)
  sync_operands();
  if (t == 0) {
    tc::mma_bf16(tb, tc::smem_desc(tc::smem_u32(sm.Xs), TILE, 0), tc::smem_desc(tc::smem_u32(sm.W1s), NH, 0),
                 tc::idesc_bf16_f32(TILE, NH), false);
    tc::mma_commit(&sm.bar);
  }
  ok = ok && wait_mma(&sm.bar, phase, err);
  if (ok) hidden_epilogue(tb, sm.bs, sm.H1s, t);
  sync_operands();
  if (t == 0 && ok) {
    for (int s = 0; s < NH / 16; ++s)
      tc::mma_bf16(tb, tc::smem_desc(tc::smem_u32(sm.H1s), TILE, s), tc::smem_desc(tc::smem_u32(sm.W2s), NH, s),
                   tc::idesc_bf16_f32(TILE, NH), s > 0);
    tc::mma_commit(&sm.bar);
  }
  ok = ok && wait_mma(&sm.bar, phase, err);
  if (ok) hidden_epilogue(tb, sm.bs + NH, sm.H2s, t);
  sync_operands();
  if (t == 0 && ok) {
    for (int s = 0; s < NH / 16; ++s)
      tc::mma_bf16(tb, tc::smem_desc(tc::smem_u32(sm.H2s), TILE, s), tc::smem_desc(tc::smem_u32(sm.W3s), NOUTP, s),
                   tc::idesc_bf16_f32(TILE, NOUTP), s > 0);
    tc::mma_commit(&sm.bar);
  }
  ok = ok && wait_mma(&sm.bar, phase, err);
  const int grp = bias_group(f[FEAT_SPECIES], f[FEAT_DEPTH]);
  {
    float v[16];
    if (ok) tc::tmem_ld16(tc::tmem_addr(tb, 32 * warp, 0), v);
#pragma unroll
    for (int j = 0; j < NOUT; ++j) y[j] = ok ? v[j] + sm.bs[2 * NH + grp * NOUTP + j] : 0.f;
  }
  // loss |sum_j w_j e_j - t|^2 = w^H G w - 2 Re(w^H g) + Gtt and dL/dy (FP32)
  float dy[NOUT], loss;
  {
    float Gr[3][3], Gi[3][3];
    Gr[0][0] = st[0];
    Gr[1][1] = st[1];
    Gr[2][2] = st[2];
    Gi[0][0] = Gi[1][1] = Gi[2][2] = 0.f;
    Gr[0][1] = st[3], Gi[0][1] = st[4];
    Gr[0][2] = st[5], Gi[0][2] = st[6];
    Gr[1][2] = st[7], Gi[1][2] = st[8];
    Gr[1][0] = Gr[0][1], Gi[1][0] = -Gi[0][1];
    Gr[2][0] = Gr[0][2], Gi[2][0] = -Gi[0][2];
    Gr[2][1] = Gr[1][2], Gi[2][1] = -Gi[1][2];
    const float gr[3] = {st[9], st[11], st[13]}, gi[3] = {st[10], st[12], st[14]};
    const float wr[3] = {y[0], y[2], y[4]}, wi[3] = {y[1], y[3], y[5]};
    loss = st[15];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      // (G w)_j - g_j
      float dr = -gr[j], di = -gi[j];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        dr += Gr[j][k] * wr[k] - Gi[j][k] * wi[k];
        di += Gr[j][k] * wi[k] + Gi[j][k] * wr[k];
      }
      // conj(w_j) ((G w)_j - 2 g_j + g_j): loss = sum_j Re(conj(w_j)((Gw)_j - g_j)) - Re(conj(w_j) g_j) + Gtt
      loss += (wr[j] * dr + wi[j] * di) - (wr[j] * gr[j] + wi[j] * gi[j]);
      dy[2 * j] = 2.f * dr * scale;
      dy[2 * j + 1] = 2.f * di * scale;
    }
    loss *= scale;
    if (!active) {
      loss = 0.f;
#pragma unroll
      for (int j = 0; j < NOUT; ++j) dy[j] = 0.f;
    }
  }
  float *g = gpart + (int64_t)blockIdx.x * NPARAMS;
  {  // loss and the b3 gradient of every bias group
    float l = loss;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if (lane == 0) sm.lred[warp] = l;
#pragma unroll 1
    for (int gq = 0; gq < NGROUP; ++gq) {
      float d[NOUT];
#pragma unroll
      for (int j = 0; j < NOUT; ++j) d[j] = grp == gq ? dy[j] : 0.f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < NOUT; ++j) d[j] += __shfl_xor_sync(0xffffffffu, d[j], o);
      if (lane == 0)
#pragma unroll
        for (int j = 0; j < NOUT; ++j) sm.red[warp][gq * NOUT + j] = d[j];
    }
    __syncthreads();
    if (t == 0) lpart[blockIdx.x] = sm.lred[0] + sm.lred[1] + sm.lred[2] + sm.lred[3];
    if (t < NGROUP * NOUT) g[OFF_B3 + t] = sm.red[0][t] + sm.red[1][t] + sm.red[2][t] + sm.red[3][t];
    __syncthreads();
  }
  // Gs = dY [128 x 16], TB = dY^T [16 x 128], TA rows 0..63 = H2^T
#pragma unroll
  for (int j = 0; j < NOUTP; ++j) {
    const float d = j < NOUT ? dy[j] : 0.f;
    st_bf16(sm.Gs, t, j, TILE, d);
    st_bf16(sm.TB, j, t, NOUTP, d);
  }
  for (int k = 0; k < NH; ++k)
    *reinterpret_cast<__nv_bfloat16 *>(sm.TA + tc::kmajor_offset(k, t, TILE)) =
        *reinterpret_cast<const __nv_bfloat16 *>(sm.H2s + tc::kmajor_offset(t, k, TILE));
  sync_operands();
  if (t == 0 && ok) {
    // dH2pre (cols 0..63) = dY W3 ; dW3^T (cols 64..79) = H2^T dY
    tc::mma_bf16(tb, tc::smem_desc(tc::smem_u32(sm.Gs), TILE, 0), tc::smem_desc(tc::smem_u32(sm.W3Ts), NH, 0),
                 tc::idesc_bf16_f32(TILE, NH), false);
    for (int s = 0; s < TILE / 16; ++s)
      tc::mma_bf16(tb + 64, tc::smem_desc(tc::smem_u32(sm.TA), TILE, s), tc::smem_desc(tc::smem_u32(sm.TB), NOUTP, s),
                   tc::idesc_bf16_f32(TILE, NOUTP), s > 0);
    tc::mma_commit(&sm.bar);
  }
  ok = ok && wait_mma(&sm.bar, phase, err);
  float dh[NH];
  // dH2 = dH2pre * (H2 > 0)
#pragma unroll
  for (int c0 = 0; c0 < NH; c0 += 16) {
    float v[16];
    if (ok) tc::tmem_ld16(tc::tmem_addr(tb, 32 * warp, c0), v);
#pragma unroll
    for (int j = 0; j < 16; ++j) dh[c0 + j] = (ok && ld_bf16(sm.H2s, t, c0 + j, TILE) > 0.f) ? v[j] : 0.f;
  }
  tc::fence_before_sync();
  column_sums(dh, sm, g + OFF_B2);
  // Gs = dH2 [128 x 64], TB = dH2^T [64 x 128], TA rows 0..63 = H1^T
#pragma unroll
  for (int j = 0; j < NH; ++j) {
    st_bf16(sm.Gs, t, j, TILE, dh[j]);
    st_bf16(sm.TB, j, t, NH, dh[j]);
  }
  for (int k = 0; k < NH; ++k)
    *reinterpret_cast<__nv_bfloat16 *>(sm.TA + tc::kmajor_offset(k, t, TILE)) =
        *reinterpret_cast<const __nv_bfloat16 *>(sm.H1s + tc::kmajor_offset(t, k, TILE));
  sync_operands();
  if (t == 0 && ok) {
    // dH1pre (cols 0..63) = dH2 W2 ; dW2^T (cols 128..191) = H1^T dH2
    for (int s = 0; s < NH / 16; ++s)
      tc::mma_bf16(tb, tc::smem_desc(tc::smem_u32(sm.Gs), TILE, s), tc::smem_desc(tc::smem_u32(sm.W2Ts), NH, s),
                   tc::idesc_bf16_f32(TILE, NH), s > 0);
    for (int s = 0; s < TILE / 16; ++s)
      tc::mma_bf16(tb + 128, tc::smem_desc(tc::smem_u32(sm.TA), TILE, s), tc::smem_desc(tc::smem_u32(sm.TB), NH, s),
                   tc::idesc_bf16_f32(TILE, NH), s > 0);
    tc::mma_commit(&sm.bar);
  }
  ok = ok && wait_mma(&sm.bar, phase, err);
#pragma unroll
  for (int c0 = 0; c0 < NH; c0 += 16) {
    float v[16];
    if (ok) tc::tmem_ld16(tc::tmem_addr(tb, 32 * warp, c0), v);
#pragma unroll
    for (int j = 0; j < 16; ++j) dh[c0 + j] = (ok && ld_bf16(sm.H1s, t, c0 + j, TILE) > 0.f) ? v[j] : 0.f;
  }
  tc::fence_before_sync();
  column_sums(dh, sm, g + OFF_B1);
  // TB = dH1^T [64 x 128], TA rows 0..15 = X^T, rows 16..63 cleared
#pragma unroll
  for (int j = 0; j < NH; ++j) st_bf16(sm.TB, j, t, NH, dh[j]);
  for (int k = 0; k < NH; ++k)
    *reinterpret_cast<__nv_bfloat16 *>(sm.TA + tc::kmajor_offset(k, t, TILE)) =
        k < NIN ? *reinterpret_cast<const __nv_bfloat16 *>(sm.Xs + tc::kmajor_offset(t, k, TILE))
                : __float2bfloat16_rn(0.f);
  sync_operands();
  if (t == 0 && ok) {
    // dW1^T (cols 192..255) = X^T dH1
    for (int s = 0; s < TILE / 16; ++s)
      tc::mma_bf16(tb + 192, tc::smem_desc(tc::smem_u32(sm.TA), TILE, s), tc::smem_desc(tc::smem_u32(sm.TB), NH, s),
                   tc::idesc_bf16_f32(TILE, NH), s > 0);
    tc::mma_commit(&sm.bar);
  }
  ok = ok && wait_mma(&sm.bar, phase, err);
  // weight gradients: lane = input feature i, column = output feature o
  if (warp < 2) {
    const int in = t;  // lanes 0..63
    float v[16];
#pragma unroll
    for (int c0 = 0; c0 < NH; c0 += 16) {  // dW2[o][i]
      if (ok) tc::tmem_ld16(tc::tmem_addr(tb, 32 * warp, 128 + c0), v);
#pragma unroll
      for (int j = 0; j < 16; ++j) g[OFF_W2 + (c0 + j) * NH + in] = ok ? v[j] : 0.f;
    }
    if (ok) tc::tmem_ld16(tc::tmem_addr(tb, 32 * warp, 64), v);  // dW3[o][i]
#pragma unroll
    for (int j = 0; j < NOUT; ++j) g[OFF_W3 + j * NH + in] = ok ? v[j] : 0.f;
#pragma unroll
    for (int c0 = 0; c0 < NH; c0 += 16) {  // dW1[o][i], i < 16
      if (ok) tc::tmem_ld16(tc::tmem_addr(tb, 32 * warp, 192 + c0), v);
      if (in < NIN)
#pragma unroll
        for (int j = 0; j < 16; ++j) g[OFF_W1 + (c0 + j) * NIN + in] = ok ? v[j] : 0.f;
    }
  }
  drain(&sm.bar, phase, ok);
  tc::fence_before_sync();
  __syncthreads();
  if (t < 32) tc::tmem_dealloc(tb, 256);
}

// fixed-order sum of the per-CTA partials; Adam step (step >= 1) when lr > 0,
// then the BF16 weight copies.  grad_out (optional) receives the summed
// gradient, loss_out the summed loss.
__global__ void k_learn_reduce_adam(const float *__restrict__ gpart, const float *__restrict__ lpart, int nparts,
                                    float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                                    int64_t step, float lr, float *grad_out, double *loss_out,
                                    __nv_bfloat16 *w1, __nv_bfloat16 *w2, __nv_bfloat16 *w3, float *bias) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0 && loss_out) {
    double l = 0.0;
    for (int c = 0; c < nparts; ++c) l += lpart[c];
    *loss_out = l;
  }
  if (k >= NPARAMS) return;
  float gs = 0.f;
  for (int c = 0; c < nparts; ++c) gs += gpart[(int64_t)c * NPARAMS + k];
  if (grad_out) grad_out[k] = gs;
  float pk = p[k];
  if (lr > 0.f) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mk = b1 * m[k] + (1.f - b1) * gs;
    const float vk = b2 * v[k] + (1.f - b2) * gs * gs;
    m[k] = mk;
    v[k] = vk;
    const float mh = mk / (1.f - powf(b1, (float)step)), vh = vk / (1.f - powf(b2, (float)step));
    pk -= lr * mh / (sqrtf(vh) + eps);
    p[k] = pk;
  }
  if (k < OFF_B1) w1[k - OFF_W1] = __float2bfloat16_rn(pk);
  else if (k < OFF_W2) bias[k - OFF_B1] = pk;
  else if (k < OFF_B2) w2[k - OFF_W2] = __float2bfloat16_rn(pk);
  else if (k < OFF_W3) bias[NH + k - OFF_B2] = pk;
  else if (k < OFF_B3) w3[k - OFF_W3] = __float2bfloat16_rn(pk);
  else bias[2 * NH + k - OFF_B3] = pk;  // b3[group][6]
}

// batch indices of iteration `it`: splitmix64 of (seed, it, j) modulo n
__global__ void k_learn_indices(int64_t *idx, int64_t batch, int64_t n, uint64_t seed, int64_t it) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= batch) return;
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(it * batch + j + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  idx[j] = (int64_t)(z % (uint64_t)n);
}

// ------------------------------------------------------------ data recording
// Features and Gram statistics of every sample of one solved step (psi, b,
// x = solution, v1/v2 = history or null) for the basis (|tau| u, v1, v2);
// hnew = t, the newest history (may be the v2 buffer).  Samples go to rows
// off + sp*V + s.
__global__ void k_learn_record(Lat L, const double2 *__restrict__ psi, const double2 *__restrict__ b,
                               const double2 *__restrict__ x, const float2 *v1, const float2 *v2, float2 *hnew,
                               const float4 *__restrict__ gf, double mass, double tau, float *__restrict__ feat,
                               float *__restrict__ stats, int64_t off) {
  const int64_t V = L.V;
  const double s0 = fabs(tau);  // scale of the u basis vector (k_learn_apply)
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= 2 * V) return;
  const int sp = (int)(q / V);
  const int64_t s = q % V;
  float f[NIN];
  sample_features(L, psi, b, v1, v2, gf, mass, tau, s, sp, f);
  double G00 = 0, G11 = 0, G22 = 0, Gtt = 0;
  cplx G01 = {0, 0}, G02 = {0, 0}, G12 = {0, 0}, g0 = {0, 0}, g1 = {0, 0}, g2 = {0, 0};
  const int64_t base = (int64_t)(sp * 36) * V + s;
  for (int k = 0; k < 36; ++k) {
    const int64_t o = base + (int64_t)k * V;
    const cplx p = ldg(psi + o), bb = ldg(b + o), xx = ldg(x + o);
    const cplx u = s0 * (bb - p);
    cplx h1 = {0, 0}, h2 = {0, 0};
    if (v1) {
      const float2 h = v1[o];
      h1 = {(double)h.x, (double)h.y};
    }
    if (v2) {
      const float2 h = v2[o];
      h2 = {(double)h.x, (double)h.y};
    }
    const cplx tt = xx - (2.0 * bb - p);
    G00 += norm2(u);
    G11 += norm2(h1);
    G22 += norm2(h2);
    Gtt += norm2(tt);
    cmac_cj(G01, u, h1);
    cmac_cj(G02, u, h2);
    cmac_cj(G12, h1, h2);
    cmac_cj(g0, u, tt);
    cmac_cj(g1, h1, tt);
    cmac_cj(g2, h2, tt);
    hnew[o] = make_float2((float)tt.re, (float)tt.im);
  }
  float *fo = feat + (off + q) * NIN;
#pragma unroll
  for (int k = 0; k < NIN; ++k) fo[k] = f[k];
  float *so = stats + (off + q) * NSTATS;
  const double vals[NSTATS] = {G00, G11, G22, G01.re, G01.im, G02.re, G02.im, G12.re, G12.im,
                               g0.re, g0.im, g1.re, g1.im, g2.re, g2.im, Gtt};
#pragma unroll
  for (int k = 0; k < NSTATS; ++k) so[k] = (float)vals[k];
}

// Closed-form refit of the output bias.  The loss is quadratic in the
// per-sample weights w_s, so a common shift d of the bias minimises
// sum_s (w_s+d)^H G_s (w_s+d) - 2 Re((w_s+d)^H g_s) at (sum_s G_s) d =
// sum_s (g_s - G_s w_s).  Per block: the 15 real components of sum G
// (3 diagonal, 3 complex off-diagonal) and sum (g - G w) (3 complex), FP64.
__global__ void k_learn_bias_sums(const float *__restrict__ omega, int ostride, const float *__restrict__ stats,
                                  const float *__restrict__ feat, int group, int64_t n,
                                  double *__restrict__ part) {
  __shared__ double sh[15][256];
  double a[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) a[k] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (bias_group(feat[i * NIN + FEAT_SPECIES], feat[i * NIN + FEAT_DEPTH]) != group) continue;
    const float *st = stats + i * NSTATS;
    const float *w = omega + i * ostride;
    double Gr[3][3], Gi[3][3];
    Gr[0][0] = st[0], Gr[1][1] = st[1], Gr[2][2] = st[2];
    Gi[0][0] = Gi[1][1] = Gi[2][2] = 0.0;
    Gr[0][1] = st[3], Gi[0][1] = st[4], Gr[0][2] = st[5], Gi[0][2] = st[6], Gr[1][2] = st[7], Gi[1][2] = st[8];
    Gr[1][0] = Gr[0][1], Gi[1][0] = -Gi[0][1], Gr[2][0] = Gr[0][2], Gi[2][0] = -Gi[0][2];
    Gr[2][1] = Gr[1][2], Gi[2][1] = -Gi[1][2];
    for (int k = 0; k < 9; ++k) a[k] += st[k];
    for (int j = 0; j < 3; ++j) {
      double rr = st[9 + 2 * j], ri = st[10 + 2 * j];
      for (int k = 0; k < 3; ++k) {
        rr -= Gr[j][k] * w[2 * k] - Gi[j][k] * w[2 * k + 1];
        ri -= Gr[j][k] * w[2 * k + 1] + Gi[j][k] * w[2 * k];
      }
      a[9 + 2 * j] += rr;
      a[10 + 2 * j] += ri;
    }
  }
#pragma unroll
  for (int k = 0; k < 15; ++k) sh[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int wd = blockDim.x / 2; wd > 0; wd >>= 1) {
    if (threadIdx.x < wd)
      for (int k = 0; k < 15; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + wd];
    __syncthreads();
  }
  if (threadIdx.x < 15) part[blockIdx.x * 15 + threadIdx.x] = sh[threadIdx.x][0];
}

// b3[group] += d (6 floats) in the FP32 parameters
__global__ void k_learn_shift_b3(float *p, int group, double d0, double d1, double d2, double d3, double d4,
                                 double d5) {
  const double d[6] = {d0, d1, d2, d3, d4, d5};
  if (threadIdx.x < NOUT) p[OFF_B3 + group * NOUT + threadIdx.x] += (float)d[threadIdx.x];
}

// sum of Gtt over rows [off, off+cnt) into *out (one block, fixed order per thread stride)
__global__ void k_learn_sum_gtt(const float *__restrict__ stats, int64_t off, int64_t cnt, double *out) {
  __shared__ double sh[256];
  double a = 0.0;
  for (int64_t r = threadIdx.x; r < cnt; r += blockDim.x) a += stats[(off + r) * NSTATS + NSTATS - 1];
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}
// stats of rows [off, off+cnt) *= cnt / sum
__global__ void k_learn_scale(float *stats, int64_t off, int64_t cnt, const double *sum) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= cnt) return;
  const double s = *sum;
  const float sc = s > 0 ? (float)((double)cnt / s) : 0.f;
  for (int k = 0; k < NSTATS; ++k) stats[(off + r) * NSTATS + k] *= sc;
}

// x += e and hist += e (the refinement corrections complete the history)
__global__ void k_add_e_hist(int64_t n, double2 *__restrict__ X, const float2 *__restrict__ Ev,
                             float2 *__restrict__ H) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 e = Ev[i];
  const double2 x = X[i];
  X[i] = make_double2(x.x + (double)e.x, x.y + (double)e.y);
  const float2 h = H[i];
  H[i] = make_float2(h.x + e.x, h.y + e.y);
}

}  // namespace learn
}  // namespace nrq

// ====================================================================== host
using namespace nrq::learn;

struct nrq_learn {
  nrq_ctx *ctx = nullptr;
  float *p = nullptr, *m = nullptr, *v = nullptr;  // FP32 parameters and Adam moments
  __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
  float *bias = nullptr;  // b1, b2, b3 (FP32)
  int64_t step = 0;
  float *feat = nullptr, *stats = nullptr;  // dataset
  int64_t n = 0, cap = 0;
  float *gpart = nullptr, *lpart = nullptr, *grad = nullptr;
  int64_t *idx = nullptr;
  int64_t part_cap = 0;
  double *d_scalar = nullptr;  // loss / Gtt sums
  int *err = nullptr;
  bool trained = false;
  // guess scratch for a lattice of scr_V sites: gauge features (V), sample
  // features (2V x 16), network outputs (2V x 8 floats)
  float4 *gf = nullptr;
  float *fbuf = nullptr;
  float4 *omega = nullptr;
  int64_t scr_V = 0;
};

namespace {

nrq::learn::Model model_of(const nrq_learn *net) {
  return {net->w1, net->w2, net->w3, net->bias, net->bias + NH, net->bias + 2 * NH};
}

int learn_err(nrq_learn *net) {
  int e = 0;
  NRQ_CUDA_TRY(net->ctx, cudaMemcpyAsync(&e, net->err, sizeof(int), cudaMemcpyDeviceToHost, net->ctx->stream));
  NRQ_CUDA_TRY(net->ctx, cudaStreamSynchronize(net->ctx->stream));
  if (e) {
    cudaMemsetAsync(net->err, 0, sizeof(int), net->ctx->stream);
    net->ctx->last_error = "learned MLP: a bounded tensor-core wait expired";
    return NRQ_ERR_TIMEOUT;
  }
  return NRQ_OK;
}

// refresh the BF16 copies from the FP32 parameters (no Adam step)
int refresh_copies(nrq_learn *net) {
  nrq::learn::k_learn_reduce_adam<<<(NPARAMS + 255) / 256, 256, 0, net->ctx->stream>>>(
      nullptr, nullptr, 0, net->p, net->m, net->v, 0, 0.f, nullptr, nullptr, net->w1, net->w2, net->w3, net->bias);
  return check_launch(net->ctx, "learned refresh");
}

int ensure_parts(nrq_learn *net, int64_t nctas) {
  if (net->part_cap >= nctas) return NRQ_OK;
  for (void *q : {(void *)net->gpart, (void *)net->lpart, (void *)net->idx})
    if (q) cudaFree(q);
  net->gpart = nullptr;
  net->lpart = nullptr;
  net->idx = nullptr;
  net->part_cap = 0;
  NRQ_CUDA_TRY(net->ctx, cudaMalloc(&net->gpart, sizeof(float) * NPARAMS * nctas));
  NRQ_CUDA_TRY(net->ctx, cudaMalloc(&net->lpart, sizeof(float) * nctas));
  NRQ_CUDA_TRY(net->ctx, cudaMalloc(&net->idx, sizeof(int64_t) * nctas * TILE));
  net->part_cap = nctas;
  return NRQ_OK;
}

int ensure_scratch(nrq_learn *net, int64_t V) {
  if (net->scr_V >= V) return NRQ_OK;
  for (void *q : {(void *)net->gf, (void *)net->fbuf, (void *)net->omega})
    if (q) cudaFree(q);
  net->gf = nullptr;
  net->fbuf = nullptr;
  net->omega = nullptr;
  net->scr_V = 0;
  NRQ_CUDA_TRY(net->ctx, cudaMalloc(&net->gf, sizeof(float4) * V));
  NRQ_CUDA_TRY(net->ctx, cudaMalloc(&net->fbuf, sizeof(float) * NIN * 2 * V));
  NRQ_CUDA_TRY(net->ctx, cudaMalloc(&net->omega, sizeof(float4) * 2 * 2 * V));
  net->scr_V = V;
  return NRQ_OK;
}

int train_smem_attr(nrq_ctx *ctx) {
  NRQ_CUDA_TRY(ctx, cudaFuncSetAttribute(nrq::learn::k_learn_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(nrq::learn::TrainSmem)));
  return NRQ_OK;
}

// loss and gradient of `n` dataset samples (feat/stats device pointers,
// idx optional), summed into grad (device, optional) and *loss (host)
int grad_pass(nrq_learn *net, const float *feat, const float *stats, const int64_t *idx, int64_t n, float lr,
              double *loss) {
  nrq_ctx *ctx = net->ctx;
  const int64_t nct = (n + TILE - 1) / TILE;
  int rc = ensure_parts(net, nct);
  if (!rc) rc = train_smem_attr(ctx);
  if (rc) return rc;
  nrq::learn::k_learn_train<<<(unsigned)nct, TILE, sizeof(nrq::learn::TrainSmem), ctx->stream>>>(
      model_of(net), feat, stats, idx, n, 1.f / (float)n, net->gpart, net->lpart, net->err);
  if ((rc = check_launch(ctx, "k_learn_train"))) return rc;
  if (lr > 0.f) net->step++;
  nrq::learn::k_learn_reduce_adam<<<(NPARAMS + 255) / 256, 256, 0, ctx->stream>>>(
      net->gpart, net->lpart, (int)nct, net->p, net->m, net->v, net->step, lr, net->grad, net->d_scalar, net->w1,
      net->w2, net->w3, net->bias);
  if ((rc = check_launch(ctx, "k_learn_reduce_adam"))) return rc;
  if (loss) {
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(loss, net->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return NRQ_OK;
}

// splitmix64 + Box-Muller normal deviates for the initial weights
struct InitRng {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double normal() { return std::sqrt(-2.0 * std::log(uniform())) * std::cos(6.283185307179586 * uniform()); }
};

}  // namespace

namespace nrqh {
// learned guess of the CN solve (see nrq_internal.h)
int learned_guess(nrq_learn *net, const nrq_ctx *ctx, const double2 *psi, const double2 *b, const float2 *v1,
                  const float2 *v2, float2 *hnew, const double2 *U, const double *E, double mass, double dt,
                  double2 *x, cudaStream_t st) {
  nrq_ctx *c = const_cast<nrq_ctx *>(ctx);
  const int64_t V = ctx->lat.V;
  int rc = ensure_scratch(net, V);
  if (rc) return rc;
  const double tau = dt * ctx->a[0] / 2.0;
  nrq::learn::k_learn_gauge_features<<<(unsigned)((V + 127) / 128), 128, 0, st>>>(ctx->lat, U, E, net->gf);
  nrq::learn::k_learn_features<<<(unsigned)((2 * V + 255) / 256), 256, 0, st>>>(ctx->lat, psi, b, v1, v2, net->gf,
                                                                              mass, tau, net->fbuf);
  const int64_t ntiles = (2 * V + TILE - 1) / TILE;
  nrq::learn::k_learn_forward<<<(unsigned)std::min<int64_t>(ntiles, (int64_t)ctx->sm_count * 4), TILE, 0, st>>>(
      model_of(net), net->fbuf, 2 * V, reinterpret_cast<float *>(net->omega), 8, net->err);
  nrq::learn::k_learn_apply<<<(unsigned)((72 * V + 255) / 256), 256, 0, st>>>(V, psi, b, v1, v2, net->omega,
                                                                              std::fabs(tau), hnew, x);
  return check_launch(c, "learned guess");
}
// learned guess of every field of a batch (table on the device): gauge
// features of the member (U, E), features, the MLP, x and the new history
int learned_guess_batch(nrq_learn *net, const nrq_ctx *ctx, const nrq::BatchField *tab, int nfields,
                        const double2 *U, const double *E, float4 *gf, float *fbuf, float4 *omega,
                        cudaStream_t st) {
  nrq_ctx *c = const_cast<nrq_ctx *>(ctx);
  const int64_t V = ctx->lat.V;
  nrq::learn::k_learn_gauge_features<<<(unsigned)((V + 127) / 128), 128, 0, st>>>(ctx->lat, U, E, gf);
  nrq::learn::k_batch_learn_features<<<dim3((unsigned)((2 * V + 255) / 256), (unsigned)nfields), 256, 0, st>>>(
      ctx->lat, tab, gf, fbuf);
  const int64_t n = 2 * V * nfields;
  const int64_t ntiles = (n + TILE - 1) / TILE;
  nrq::learn::k_learn_forward<<<(unsigned)std::min<int64_t>(ntiles, (int64_t)ctx->sm_count * 4), TILE, 0, st>>>(
      model_of(net), fbuf, n, reinterpret_cast<float *>(omega), 8, net->err);
  nrq::learn::k_batch_learn_apply<<<dim3((unsigned)std::min<int64_t>((72 * V + 255) / 256, 2048), (unsigned)nfields),
                                    256, 0, st>>>(V, tab, omega);
  return check_launch(c, "batched learned guess");
}
int ensure_hist(nrq_heavy *h, int depth) {
  depth = std::min(std::max(depth, 2), (int)nrq_heavy::kMaxHist);
  for (int k = 0; k < depth; ++k)
    if (!h->hist[k]) NRQ_CUDA_TRY(h->ctx, cudaMalloc(&h->hist[k], sizeof(float2) * 72 * h->ctx->lat.V));
  if (depth > h->hist_cap) {  // a larger ring: its order starts afresh
    h->hist_cap = depth;
    h->hist_count = 0;
    h->hist_head = 0;
  }
  return NRQ_OK;
}
void add_e_hist(int64_t n, double2 *x, const float2 *e, float2 *hist, cudaStream_t st) {
  nrq::learn::k_add_e_hist<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, x, e, hist);
}
int learned_check(nrq_learn *net) { return learn_err(net); }
const nrq_ctx *learned_ctx(const nrq_learn *net) { return net ? net->ctx : nullptr; }
bool learned_ready(const nrq_learn *net) { return net && net->trained; }
}  // namespace nrqh

extern "C" int nrq_learn_create(nrq_ctx *ctx, uint64_t seed, nrq_learn **out) {
  if (!ctx || !out) return NRQ_ERR_BAD_ARG;
  int rc = set_device(ctx);
  if (rc) return rc;
  nrq_learn *net = new (std::nothrow) nrq_learn();
  if (!net) return NRQ_ERR_OOM;
  net->ctx = ctx;
  auto fail = [&](cudaError_t e) {
    ctx->last_error = std::string("learned allocation: ") + cudaGetErrorString(e);
    nrq_learn_destroy(net);
    return e == cudaErrorMemoryAllocation ? NRQ_ERR_OOM : NRQ_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&net->p, sizeof(float) * NPARAMS)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->m, sizeof(float) * NPARAMS)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->v, sizeof(float) * NPARAMS)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->grad, sizeof(float) * NPARAMS)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->w1, sizeof(__nv_bfloat16) * NH * NIN)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->w2, sizeof(__nv_bfloat16) * NH * NH)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->w3, sizeof(__nv_bfloat16) * NOUT * NH)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->bias, sizeof(float) * (2 * NH + NGROUP * NOUT))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->d_scalar, sizeof(double) * 2)) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&net->err, sizeof(int))) != cudaSuccess) return fail(e);
  cudaMemsetAsync(net->err, 0, sizeof(int), ctx->stream);
  cudaMemsetAsync(net->m, 0, sizeof(float) * NPARAMS, ctx->stream);
  cudaMemsetAsync(net->v, 0, sizeof(float) * NPARAMS, ctx->stream);
  // He-normal hidden layers, small output layer, zero biases: the untrained
  // network starts near the plain extrapolated guess
  std::vector<float> p(NPARAMS, 0.f);
  InitRng r{seed};
  for (int k = 0; k < NH * NIN; ++k) p[OFF_W1 + k] = (float)(r.normal() * std::sqrt(2.0 / NIN));
  for (int k = 0; k < NH * NH; ++k) p[OFF_W2 + k] = (float)(r.normal() * std::sqrt(2.0 / NH));
  for (int k = 0; k < NOUT * NH; ++k) p[OFF_W3 + k] = (float)(r.normal() * 1e-3);
  int rc2 = nrq_learn_params(net, p.data(), 1);
  if (rc2) {
    nrq_learn_destroy(net);
    return rc2;
  }
  *out = net;
  return NRQ_OK;
}

extern "C" int nrq_learn_destroy(nrq_learn *net) {
  if (!net) return NRQ_ERR_NOT_INITIALISED;
  cudaSetDevice(net->ctx->device);
  cudaStreamSynchronize(net->ctx->stream);
  for (void *q : {(void *)net->p, (void *)net->m, (void *)net->v, (void *)net->grad, (void *)net->w1,
                  (void *)net->w2, (void *)net->w3, (void *)net->bias, (void *)net->d_scalar, (void *)net->err,
                  (void *)net->feat, (void *)net->stats, (void *)net->gpart, (void *)net->lpart, (void *)net->idx,
                  (void *)net->gf, (void *)net->fbuf, (void *)net->omega})
    if (q) cudaFree(q);
  delete net;
  return NRQ_OK;
}

extern "C" int nrq_learn_params(nrq_learn *net, float *params, int set) {
  if (!net || !params) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = net->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  if (set) {
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(net->p, params, sizeof(float) * NPARAMS, cudaMemcpyHostToDevice, ctx->stream));
    NRQ_CUDA_TRY(ctx, cudaMemsetAsync(net->m, 0, sizeof(float) * NPARAMS, ctx->stream));
    NRQ_CUDA_TRY(ctx, cudaMemsetAsync(net->v, 0, sizeof(float) * NPARAMS, ctx->stream));
    net->step = 0;
    if ((rc = refresh_copies(net))) return rc;
    NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  } else {
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(params, net->p, sizeof(float) * NPARAMS, cudaMemcpyDeviceToHost, ctx->stream));
    NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return NRQ_OK;
}

extern "C" int nrq_learn_set_trained(nrq_learn *net, int trained) {
  if (!net) return NRQ_ERR_BAD_ARG;
  net->trained = trained != 0;
  return NRQ_OK;
}

extern "C" int nrq_learn_loss_grad(nrq_learn *net, const float *features, const float *stats, int64_t n,
                                   double *loss, float *grad) {
  if (!net || !features || !stats || n <= 0) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = net->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  float *df = nullptr, *ds = nullptr;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&df, sizeof(float) * NIN * n));
  cudaError_t e = cudaMalloc(&ds, sizeof(float) * NSTATS * n);
  if (e != cudaSuccess) {
    cudaFree(df);
    ctx->last_error = cudaGetErrorString(e);
    return NRQ_ERR_CUDA;
  }
  cudaMemcpyAsync(df, features, sizeof(float) * NIN * n, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(ds, stats, sizeof(float) * NSTATS * n, cudaMemcpyHostToDevice, ctx->stream);
  double l = 0.0;
  rc = grad_pass(net, df, ds, nullptr, n, 0.f, &l);
  if (!rc) rc = learn_err(net);
  if (!rc && grad) {
    cudaMemcpyAsync(grad, net->grad, sizeof(float) * NPARAMS, cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
  }
  cudaFree(df);
  cudaFree(ds);
  if (loss) *loss = l;
  return rc;
}

extern "C" int nrq_learn_forward(nrq_learn *net, const float *features, int64_t n, float *out) {
  if (!net || !features || !out || n <= 0) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = net->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  float *df = nullptr, *dout = nullptr;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&df, sizeof(float) * NIN * n));
  cudaError_t e = cudaMalloc(&dout, sizeof(float) * NOUT * n);
  if (e != cudaSuccess) {
    cudaFree(df);
    ctx->last_error = cudaGetErrorString(e);
    return NRQ_ERR_CUDA;
  }
  cudaMemcpyAsync(df, features, sizeof(float) * NIN * n, cudaMemcpyHostToDevice, ctx->stream);
  const int64_t ntiles = (n + TILE - 1) / TILE;
  nrq::learn::k_learn_forward<<<(unsigned)std::min<int64_t>(ntiles, ctx->sm_count * 4), TILE, 0, ctx->stream>>>(
      model_of(net), df, n, dout, NOUT, net->err);
  rc = check_launch(ctx, "k_learn_forward");
  if (!rc) rc = learn_err(net);
  if (!rc) {
    cudaMemcpyAsync(out, dout, sizeof(float) * NOUT * n, cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
  }
  cudaFree(df);
  cudaFree(dout);
  return rc;
}

extern "C" int nrq_learn_dataset_reserve(nrq_learn *net, int64_t max_samples) {
  if (!net || max_samples <= 0) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = net->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  if (net->feat) cudaFree(net->feat);
  if (net->stats) cudaFree(net->stats);
  net->feat = nullptr;
  net->stats = nullptr;
  net->n = net->cap = 0;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&net->feat, sizeof(float) * NIN * max_samples));
  NRQ_CUDA_TRY(ctx, cudaMalloc(&net->stats, sizeof(float) * NSTATS * max_samples));
  net->cap = max_samples;
  return NRQ_OK;
}

extern "C" int nrq_learn_dataset_size(const nrq_learn *net, int64_t *n) {
  if (!net || !n) return NRQ_ERR_BAD_ARG;
  *n = net->n;
  return NRQ_OK;
}

extern "C" int nrq_learn_dataset_read(nrq_learn *net, int64_t first, int64_t count, float *features, float *stats) {
  if (!net || first < 0 || count <= 0 || first + count > net->n) return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = net->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  if (features)
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(features, net->feat + first * NIN, sizeof(float) * NIN * count,
                                      cudaMemcpyDeviceToHost, ctx->stream));
  if (stats)
    NRQ_CUDA_TRY(ctx, cudaMemcpyAsync(stats, net->stats + first * NSTATS, sizeof(float) * NSTATS * count,
                                      cudaMemcpyDeviceToHost, ctx->stream));
  NRQ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return NRQ_OK;
}

namespace nrqh {
// append the samples of one solved step; hist (valid or not) -> t
int learn_record(nrq_learn *net, const nrq_ctx *ctx, const double2 *psi, const double2 *b, const double2 *x,
                 const float2 *v1, const float2 *v2, float2 *hnew, const double2 *U, const double *E, double mass,
                 double dt) {
  const int64_t V = ctx->lat.V;
  if (net->n + 2 * V > net->cap) return NRQ_ERR_CAPACITY;
  cudaStream_t st = ctx->stream;
  const double tau = dt * ctx->a[0] / 2.0;
  int rc0 = ensure_scratch(net, V);
  if (rc0) return rc0;
  nrq::learn::k_learn_gauge_features<<<(unsigned)((V + 127) / 128), 128, 0, st>>>(ctx->lat, U, E, net->gf);
  nrq::learn::k_learn_record<<<(unsigned)((2 * V + 127) / 128), 128, 0, st>>>(
      ctx->lat, psi, b, x, v1, v2, hnew, net->gf, mass, tau, net->feat, net->stats, net->n);
  nrq::learn::k_learn_sum_gtt<<<1, 256, 0, st>>>(net->stats, net->n, 2 * V, net->d_scalar + 1);
  nrq::learn::k_learn_scale<<<(unsigned)((2 * V + 255) / 256), 256, 0, st>>>(net->stats, net->n, 2 * V,
                                                                             net->d_scalar + 1);
  int rc = check_launch(const_cast<nrq_ctx *>(ctx), "k_learn_record");
  if (rc) return rc;
  net->n += 2 * V;
  return NRQ_OK;
}
}  // namespace nrqh

namespace {
// solve the 3x3 complex hermitian system G d = r (partial pivoting, small ridge)
bool solve3(const double *S, double d[6]) {
  std::complex<double> G[3][3], r[3];
  G[0][0] = S[0], G[1][1] = S[1], G[2][2] = S[2];
  G[0][1] = {S[3], S[4]}, G[0][2] = {S[5], S[6]}, G[1][2] = {S[7], S[8]};
  G[1][0] = std::conj(G[0][1]), G[2][0] = std::conj(G[0][2]), G[2][1] = std::conj(G[1][2]);
  for (int j = 0; j < 3; ++j) r[j] = {S[9 + 2 * j], S[10 + 2 * j]};
  const double ridge = 1e-12 * (S[0] + S[1] + S[2]) + 1e-300;
  for (int j = 0; j < 3; ++j) G[j][j] += ridge;
  for (int c = 0; c < 3; ++c) {
    int piv = c;
    for (int k = c + 1; k < 3; ++k)
      if (std::abs(G[k][c]) > std::abs(G[piv][c])) piv = k;
    if (std::abs(G[piv][c]) == 0.0) return false;
    for (int k = 0; k < 3; ++k) std::swap(G[c][k], G[piv][k]);
    std::swap(r[c], r[piv]);
    for (int k = c + 1; k < 3; ++k) {
      const std::complex<double> f = G[k][c] / G[c][c];
      for (int m = c; m < 3; ++m) G[k][m] -= f * G[c][m];
      r[k] -= f * r[c];
    }
  }
  std::complex<double> x[3];
  for (int c = 2; c >= 0; --c) {
    std::complex<double> acc = r[c];
    for (int k = c + 1; k < 3; ++k) acc -= G[c][k] * x[k];
    x[c] = acc / G[c][c];
  }
  for (int j = 0; j < 3; ++j) {
    d[2 * j] = x[j].real();
    d[2 * j + 1] = x[j].imag();
    if (!std::isfinite(d[2 * j]) || !std::isfinite(d[2 * j + 1])) return false;
  }
  return true;
}

// exact least-squares shift of the output bias over the whole dataset
int refit_output_bias(nrq_learn *net) {
  nrq_ctx *ctx = net->ctx;
  cudaStream_t st = ctx->stream;
  float *om = nullptr;
  double *part = nullptr;
  const int nblk = 512;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&om, sizeof(float) * 8 * net->n));
  cudaError_t e = cudaMalloc(&part, sizeof(double) * 15 * nblk);
  if (e != cudaSuccess) {
    cudaFree(om);
    ctx->last_error = cudaGetErrorString(e);
    return NRQ_ERR_CUDA;
  }
  const int64_t ntiles = (net->n + TILE - 1) / TILE;
  nrq::learn::k_learn_forward<<<(unsigned)std::min<int64_t>(ntiles, ctx->sm_count * 4), TILE, 0, st>>>(
      model_of(net), net->feat, net->n, om, 8, net->err);
  std::vector<double> h(15 * nblk);
  double S[NGROUP][15] = {{0}};
  for (int gq = 0; gq < NGROUP; ++gq) {
    nrq::learn::k_learn_bias_sums<<<nblk, 256, 0, st>>>(om, 8, net->stats, net->feat, gq, net->n, part);
    cudaMemcpyAsync(h.data(), part, sizeof(double) * 15 * nblk, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    for (int b = 0; b < nblk; ++b)
      for (int k = 0; k < 15; ++k) S[gq][k] += h[b * 15 + k];
  }
  cudaFree(om);
  cudaFree(part);
  int rc = learn_err(net);
  if (rc) return rc;
  for (int gq = 0; gq < NGROUP; ++gq) {
    double d[6];
    if (S[gq][0] <= 0.0 || !solve3(S[gq], d)) continue;  // no data or degenerate: keep the trained bias
    nrq::learn::k_learn_shift_b3<<<1, 32, 0, st>>>(net->p, gq, d[0], d[1], d[2], d[3], d[4], d[5]);
  }
  if ((rc = check_launch(ctx, "k_learn_shift_b3"))) return rc;
  return refresh_copies(net);
}
}  // namespace

extern "C" int nrq_learn_train(nrq_learn *net, int64_t iterations, int64_t batch, double lr, uint64_t seed,
                               double *loss_first, double *loss_last) {
  if (!net || iterations <= 0 || batch <= 0 || !(lr > 0.0)) return NRQ_ERR_BAD_ARG;
  if (net->n <= 0) {
    net->ctx->last_error = "learned: empty dataset";
    return NRQ_ERR_BAD_ARG;
  }
  nrq_ctx *ctx = net->ctx;
  int rc = set_device(ctx);
  if (rc) return rc;
  batch = (batch + TILE - 1) / TILE * TILE;
  if ((rc = ensure_parts(net, batch / TILE))) return rc;
  double l0 = 0.0, l1 = 0.0;
  for (int64_t it = 0; it < iterations; ++it) {
    // cosine decay of the learning rate to 5% at the end
    const double frac = (double)it / (double)iterations;
    const float lr_it = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.141592653589793 * frac))));
    nrq::learn::k_learn_indices<<<(unsigned)((batch + 255) / 256), 256, 0, ctx->stream>>>(net->idx, batch, net->n,
                                                                                        seed, it);
    if ((rc = grad_pass(net, net->feat, net->stats, net->idx, batch, lr_it, it == 0 ? &l0 : nullptr))) return rc;
    // the correlated history directions make the loss ill-conditioned for a
    // first-order method: every quarter the output bias is refitted exactly
    if ((it + 1) % std::max<int64_t>(1, iterations / 4) == 0 && (rc = refit_output_bias(net))) return rc;
  }
  // loss of the last batch with the final parameters
  if ((rc = grad_pass(net, net->feat, net->stats, net->idx, batch, 0.f, &l1))) return rc;
  if ((rc = learn_err(net))) return rc;
  if (loss_first) *loss_first = l0;
  if (loss_last) *loss_last = l1;
  net->trained = true;
  return NRQ_OK;
}

extern "C" int nrq_cn_attach_learned(nrq_cn *cn, nrq_learn *net) {
  if (!cn || (net && net->ctx != cn->ctx)) return NRQ_ERR_BAD_ARG;
  cn->learn = net;
  return NRQ_OK;
}

extern "C" int nrq_learn_record(nrq_learn *net, nrq_cn *cn, nrq_heavy *h, const nrq_gauge *g, double mass,
                                const double c[8], double dt, nrq_cn_stats *stats) {
  if (!net || !cn || !h || !g || !c || net->ctx != cn->ctx || h->ctx != cn->ctx || g->ctx != cn->ctx)
    return NRQ_ERR_BAD_ARG;
  nrq_ctx *ctx = cn->ctx;
  if (net->n + 2 * ctx->lat.V > net->cap) {
    ctx->last_error = "learned: dataset full (nrq_learn_dataset_reserve)";
    return NRQ_ERR_CAPACITY;
  }
  int rc = set_device(ctx);
  if (!rc) rc = nrqh::ensure_hist(h);
  if (rc) return rc;
  // the step itself runs without the learned guess and without the
  // history start (which would also write the history); the history it
  // leaves is the exact t = x - (2 RHS - psi)
  const int cnt = h->hist_count, head = h->hist_head;
  nrq_learn *saved = cn->learn;
  const bool saved_hist = cn->history_guess;
  cn->learn = nullptr;
  cn->history_guess = false;
  rc = nrq_heavy_update_cn(cn, h, g, mass, c, dt, stats);
  cn->learn = saved;
  cn->history_guess = saved_hist;
  h->hist_count = cnt;
  h->hist_head = head;
  if (rc) {
    h->hist_count = 0;
    return rc;
  }
  // after the update: h->P = x, cn->x = psi of the step, cn->b = RHS
  rc = nrqh::learn_record(net, ctx, cn->x, cn->b, h->P, hist_v1(h), hist_v2(h), hist_next(h), g->U, g->E, mass,
                          dt);
  if (rc) {
    h->hist_count = 0;
    return rc;
  }
  hist_push(h);
  return NRQ_OK;
}
