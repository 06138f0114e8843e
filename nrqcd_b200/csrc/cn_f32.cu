// Precision form of the Crank-Nicolson solve: FP32 inner iterations inside
// an FP64 iterative refinement (the FP64 outer residual and update live in
// capi.cu / cn_mv3.cu).
//
// Inner solver: Chebyshev iteration for A^H e = r.  With real Wilson
// coefficients A^H = 1 + i tau H, H hermitian (cn.cu), so the spectrum of A^H
// lies on the segment {1 + i tau lambda : lambda in [lo, hi]}, which
// k_cn_bounds encloses per step (block Gershgorin).  With centre theta and
// half-length delta of that segment, sigma = theta/delta, rho_0 = 1/sigma,
// d_0 = r_0/theta and
//   e_{k+1} = e_k + d_k,   r_{k+1} = r_k - A^H d_k,
//   rho_{k+1} = 1/(2 sigma - rho_k),
//   d_{k+1} = rho_{k+1} rho_k d_k + (2 rho_{k+1}/delta) r_{k+1}
// (Chebyshev acceleration, e.g. Saad, Iterative Methods for Sparse Linear
// Systems, sec. 12.1).  The scalars need no inner products, so one stencil
// launch per iteration carries every vector update in its epilogue and no
// host synchronisation is needed inside the inner solve.
//
// Stencil layout as cn_mv.cu (32 sites x 6 warps per block; a thread owns
// the rows (c, s) of the 6 columns of its species) in FP32 on FP32 copies of
// the per-step gauge-derived matrices.
#include <algorithm>
#include <type_traits>

#include "nrq_kernels.cuh"

namespace nrq {

struct cf {
  float re, im;
};
__device__ __forceinline__ cf operator+(cf a, cf b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cf operator-(cf a, cf b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cf operator-(cf a) { return {-a.re, -a.im}; }
__device__ __forceinline__ cf operator*(cf a, cf b) {
  return {fmaf(a.re, b.re, -a.im * b.im), fmaf(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ cf operator*(float s, cf a) { return {s * a.re, s * a.im}; }
__device__ __forceinline__ cf conjf_(cf a) { return {a.re, -a.im}; }
__device__ __forceinline__ cf timesi(cf a) { return {-a.im, a.re}; }
__device__ __forceinline__ void cmacf(cf &acc, cf a, cf b) {
  acc.re = fmaf(a.re, b.re, fmaf(-a.im, b.im, acc.re));
  acc.im = fmaf(a.re, b.im, fmaf(a.im, b.re, acc.im));
}
__device__ __forceinline__ cf ldf(const float2 *p) {
  float2 v = __ldg(p);
  return {v.x, v.y};
}
__device__ __forceinline__ void stf(float2 *p, cf a) { *p = make_float2(a.re, a.im); }
__device__ __forceinline__ cf tof(cplx a) { return {(float)a.re, (float)a.im}; }

template <int K>
__device__ __forceinline__ cf sigf(int s, int t, cf v) {
  if (K == 0) return (s != t) ? v : cf{0.f, 0.f};
  if (K == 1) {
    if (s == 0 && t == 1) return -timesi(v);
    if (s == 1 && t == 0) return timesi(v);
    return {0.f, 0.f};
  }
  if (s != t) return {0.f, 0.f};
  return (s == 0) ? v : -v;
}

// ------------------------------------------------------------------ FP32 copies
__global__ void k_cn_to_f32(int64_t V, const double2 *__restrict__ U, const double2 *__restrict__ DE,
                            const double2 *__restrict__ D, const double *__restrict__ B, float2 *__restrict__ U32,
                            float2 *__restrict__ DE32, float2 *__restrict__ D32, float *__restrict__ B32) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  for (int k = 0; k < 27; ++k) {
    double2 v = U[(int64_t)k * V + s];
    U32[(int64_t)k * V + s] = make_float2((float)v.x, (float)v.y);
  }
  for (int k = 0; k < 54; ++k) {
    double2 v = DE[(int64_t)k * V + s];
    DE32[(int64_t)k * V + s] = make_float2((float)v.x, (float)v.y);
  }
  for (int k = 0; k < 9; ++k) {
    double2 v = D[(int64_t)k * V + s];
    D32[(int64_t)k * V + s] = make_float2((float)v.x, (float)v.y);
    B32[(int64_t)k * V + s] = (float)B[(int64_t)k * V + s];
  }
}

// ------------------------------------------------------------------ spectral bounds
// Per site and species: lower/upper Gershgorin ends of the hermitian H with
// A^H = 1 + i tau H (real coefficients r_t = Im(conj(alpha_t)) / tau).
// partials[b*4 + {0,1,2,3}] = {min lo_q, max hi_q, min lo_a, max hi_a}.
// bound on the spectral norm of a near-unitary link: sqrt of the largest
// absolute row sum of U^+ U (Gershgorin)
__device__ __forceinline__ double link_norm(const double2 *M, int64_t V, int64_t y) {
  cplx u[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) u[k] = ldg(M + (int64_t)k * V + y);
  double mx = 0.0;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    double row = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cplx a = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) cmac_cj(a, u[k * 3 + r], u[k * 3 + c]);
      row += hypot(a.re, a.im);
    }
    mx = fmax(mx, row);
  }
  return sqrt(mx);
}

__device__ __forceinline__ double frob(const double2 *M, int64_t V, int64_t y) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double2 v = __ldg(M + (int64_t)k * V + y);
    s += v.x * v.x + v.y * v.y;
  }
  return sqrt(s);
}

__global__ void __launch_bounds__(256) k_cn_bounds(Lat L, CnCoef C, double tau, const double2 *__restrict__ U,
                                                   const double2 *__restrict__ Dsum, const double *__restrict__ Bsum,
                                                   const double2 *__restrict__ DE, double *partials) {
  int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double v[4] = {1e300, -1e300, 1e300, -1e300};
  if (x < L.V) {
    const int64_t V = L.V;
    // neighbour block norms are species independent up to the coefficients
    double nU[6], nDE[6];
    for (int i = 0; i < 3; ++i) {
      const int64_t xm = nb(L, x, i, -1);
      nU[2 * i] = link_norm(U + (int64_t)(i * 9) * V, V, x);
      nU[2 * i + 1] = link_norm(U + (int64_t)(i * 9) * V, V, xm);
      nDE[2 * i] = frob(DE + (int64_t)((i * 2) * 9) * V, V, x) + frob(DE + (int64_t)((i * 2 + 1) * 9) * V, V, x);
      nDE[2 * i + 1] = frob(DE + (int64_t)((i * 2) * 9) * V, V, xm) + frob(DE + (int64_t)((i * 2 + 1) * 9) * V, V, xm);
    }
    for (int sp = 0; sp < 2; ++sp) {
      // conj(alpha) = i tau r  ->  r = Im(conj(alpha)) / tau
      const double rk = C.kin[sp].im / tau, rm = C.mag[sp].im / tau, rd = C.dar[sp].im / tau,
                   rs = C.so[sp].im / tau;
      // diagonal colour block rk*dkin 1 + rd D^T + rm B (hermitian)
      double M_re[9], M_im[9];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          double2 dv = __ldg(Dsum + (int64_t)(c * 3 + r) * V + x);  // D^T[r][c]
          double bv = __ldg(Bsum + (int64_t)(c * 3 + r) * V + x);
          M_re[r * 3 + c] = rd * dv.x + rm * bv + (r == c ? rk * C.dkin : 0.0);
          M_im[r * 3 + c] = rd * dv.y;
        }
      const double cen = (M_re[0] + M_re[4] + M_re[8]) / 3.0;
      double dev = 0.0;
      for (int k = 0; k < 9; ++k) {
        const double re = M_re[k] - ((k % 4 == 0) ? cen : 0.0);
        dev += re * re + M_im[k] * M_im[k];
      }
      double R = sqrt(dev);
      for (int n = 0; n < 6; ++n) R += fabs(rk) * 0.5 * C.inva2[n / 2] * nU[n] + fabs(rs) * nDE[n];
      R *= 1.0 + 1e-9;
      v[2 * sp] = cen - R;
      v[2 * sp + 1] = cen + R;
    }
  }
  __shared__ double sh[8][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v[0] = fmin(v[0], __shfl_down_sync(0xffffffffu, v[0], o));
    v[1] = fmax(v[1], __shfl_down_sync(0xffffffffu, v[1], o));
    v[2] = fmin(v[2], __shfl_down_sync(0xffffffffu, v[2], o));
    v[3] = fmax(v[3], __shfl_down_sync(0xffffffffu, v[3], o));
  }
  if (lane == 0)
    for (int k = 0; k < 4; ++k) sh[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double a[4] = {1e300, -1e300, 1e300, -1e300};
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a[0] = fmin(a[0], sh[w][0]);
      a[1] = fmax(a[1], sh[w][1]);
      a[2] = fmin(a[2], sh[w][2]);
      a[3] = fmax(a[3], sh[w][3]);
    }
    for (int k = 0; k < 4; ++k) partials[blockIdx.x * 4 + k] = a[k];
  }
}

__global__ void k_cn_bounds_final(const double *__restrict__ partials, int64_t nblk, double *out) {
  __shared__ double sh[4][256];
  double a[4] = {1e300, -1e300, 1e300, -1e300};
  for (int64_t b = threadIdx.x; b < nblk; b += blockDim.x) {
    a[0] = fmin(a[0], partials[b * 4]);
    a[1] = fmax(a[1], partials[b * 4 + 1]);
    a[2] = fmin(a[2], partials[b * 4 + 2]);
    a[3] = fmax(a[3], partials[b * 4 + 3]);
  }
  for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] = fmin(sh[0][threadIdx.x], sh[0][threadIdx.x + w]);
      sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + w]);
      sh[2][threadIdx.x] = fmin(sh[2][threadIdx.x], sh[2][threadIdx.x + w]);
      sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = sh[threadIdx.x][0];
}

// ------------------------------------------------------------------ FP32 Chebyshev step
// t = A^H d (FP32, all 12 columns), then per site and row:
//   r <- r - t ; e <- e + d ; d' = c1 d + c2 r      (c1, c2 per species)
// One 32-site tile of one Chebyshev step for NF fields that share the same
// operator (same mass): the gauge-derived weights are loaded and assembled
// once per neighbour and applied to every field of the tile.
template <bool FIRST, int NF>
__device__ __forceinline__ void cheb32_tile(const Lat &L, const CnCoef &C, const float2 *__restrict__ U,
                                            const float2 *__restrict__ Dsum, const float *__restrict__ Bsum,
                                            const float2 *__restrict__ DE, const float2 *const (&D)[NF],
                                            float2 *const (&Dn)[NF], float2 *const (&R)[NF],
                                            float2 *const (&Ev)[NF], const ChebCoef &K, int64_t block) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sp = warp / 3, c = warp % 3;
  const int64_t V = L.V;
  const int64_t x0 = block * 32 + lane;
  const bool active = x0 < V;
  const int64_t x = active ? x0 : 0;
  const int64_t pb = (int64_t)(sp * 36) * V;
  auto load_w = [&](const float2 *Df, int64_t y, int col, cf w[6]) {
    const float2 *p = Df + pb + (int64_t)(col * 6) * V + y;
#pragma unroll
    for (int r = 0; r < 6; ++r) w[r] = ldf(p + (int64_t)r * V);
  };
  const cf ak = tof(C.kin[sp]), am = tof(C.mag[sp]), ad = tof(C.dar[sp]), aso = tof(C.so[sp]);
  cf acc[NF][6][2];
  {
    cf Cd[3];
#pragma unroll
    for (int cp = 0; cp < 3; ++cp) {
      cf dv = ldf(Dsum + (int64_t)(cp * 3 + c) * V + x);
      float bv = __ldg(Bsum + (int64_t)(cp * 3 + c) * V + x);
      Cd[cp] = ad * dv + bv * am;
    }
    Cd[c] = Cd[c] + (float)C.dkin * ak + cf{1.f, 0.f};
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int col = 0; col < 6; ++col) {
        cf w[6];
        load_w(D[f], x, col, w);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          cf a_ = Cd[0] * w[s];
          cmacf(a_, Cd[1], w[2 + s]);
          cmacf(a_, Cd[2], w[4 + s]);
          acc[f][col][s] = a_;
        }
      }
  }
  const cf cs0 = timesi(aso), cs1 = -timesi(aso);
  auto neighbour = [&](auto Ic, auto DIRc) {
    constexpr int I = decltype(Ic)::value, DIR = decltype(DIRc)::value;
    constexpr int K0 = (I + 2) % 3, K1 = (I + 1) % 3;
    const int64_t y = nb(L, x, I, DIR == 0 ? +1 : -1);
    const int64_t ms = DIR == 0 ? x : y;
    const float2 *Up = U + (int64_t)(I * 9) * V + ms;
    const float2 *D0 = DE + (int64_t)((I * 2 + 0) * 9) * V + ms;
    const float2 *D1 = DE + (int64_t)((I * 2 + 1) * 9) * V + ms;
    const cf ck = (-0.5f * (float)C.inva2[I]) * ak;
    const cf s0 = DIR == 0 ? cs0 : -cs0, s1 = DIR == 0 ? cs1 : -cs1;
    cf Wm[2][3][2];
#pragma unroll
    for (int cp = 0; cp < 3; ++cp) {
      const int e = DIR == 0 ? (cp * 3 + c) : (c * 3 + cp);
      cf u = ldf(Up + (int64_t)e * V), d0 = ldf(D0 + (int64_t)e * V), d1 = ldf(D1 + (int64_t)e * V);
      if (DIR == 1) {
        u = conjf_(u);
        d0 = conjf_(d0);
        d1 = conjf_(d1);
      }
      const cf ku = ck * u, e0 = s0 * d0, e1 = s1 * d1;
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          cf v = (s == t) ? ku : cf{0.f, 0.f};
          v = v + sigf<K0>(s, t, e0);
          v = v + sigf<K1>(s, t, e1);
          Wm[s][cp][t] = v;
        }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int col = 0; col < 6; ++col) {
        cf w[6];
        load_w(D[f], y, col, w);
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
          for (int cp = 0; cp < 3; ++cp) {
            cmacf(acc[f][col][s], Wm[s][cp][0], w[2 * cp]);
            cmacf(acc[f][col][s], Wm[s][cp][1], w[2 * cp + 1]);
          }
      }
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  neighbour(I0{}, I0{});
  neighbour(I0{}, I1{});
  neighbour(I1{}, I0{});
  neighbour(I1{}, I1{});
  neighbour(I2{}, I0{});
  neighbour(I2{}, I1{});

  if (!active) return;
  const cf c1 = tof(K.c1[sp]), c2 = tof(K.c2[sp]);
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int col = 0; col < 6; ++col)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int64_t o = pb + (int64_t)(col * 6 + 2 * c + s) * V + x;
        const cf d = ldf(D[f] + o);
        const cf r = ldf(R[f] + o) - acc[f][col][s];
        stf(R[f] + o, r);
        stf(Ev[f] + o, FIRST ? d : ldf(Ev[f] + o) + d);
        stf(Dn[f] + o, c1 * d + c2 * r);
      }
}

template <bool FIRST>
__global__ void __launch_bounds__(192, 2) k_cheb32(Lat L, CnCoef C, const float2 *__restrict__ U,
                                                   const float2 *__restrict__ Dsum, const float *__restrict__ Bsum,
                                                   const float2 *__restrict__ DE, const float2 *__restrict__ D,
                                                   float2 *__restrict__ Dn, float2 *__restrict__ R,
                                                   float2 *__restrict__ Ev, ChebCoef K) {
  const float2 *const d[1] = {D};
  float2 *const dn[1] = {Dn};
  float2 *const r[1] = {R};
  float2 *const e[1] = {Ev};
  cheb32_tile<FIRST, 1>(L, C, U, Dsum, Bsum, DE, d, dn, r, e, K, blockIdx.x);
}

// ------------------------------------------------------------------ batched
// Step `step` of the inner Chebyshev solve for every field of a batch in one
// launch.  The table holds the fields grouped by mass in tiles of NF fields;
// the flattened block index is split into (tile, site block) with the tile
// fastest (ORDER 0: consecutive blocks share the gauge-derived tiles in L2)
// or the site block fastest (ORDER 1).
// MINB resident blocks per SM (the register budget: 2 -> 168, 3 -> 113);
// two-field tiles double the accumulators and run one block per SM
template <bool FIRST, int NF, int ORDER, int MINB>
__global__ void __launch_bounds__(192, MINB) k_batch_cheb32(Lat L, const float2 *__restrict__ U,
                                                         const float2 *__restrict__ Dsum,
                                                         const float *__restrict__ Bsum,
                                                         const float2 *__restrict__ DE,
                                                         const BatchField *__restrict__ tab, int ntiles,
                                                         int64_t nsb, int step) {
  const int64_t bid = blockIdx.x;
  const int tile = ORDER == 0 ? (int)(bid % ntiles) : (int)(bid / nsb);
  const int64_t sb = ORDER == 0 ? bid / ntiles : bid % nsb;
  // fields that passed their last residual check sit out (uniform per block)
  bool all_done = true;
#pragma unroll
  for (int j = 0; j < NF; ++j) all_done = all_done && batch_field_done(tab[tile * NF + j]);
  if (all_done) return;
  const float2 *d[NF];
  float2 *dn[NF], *r[NF], *e[NF];
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    const BatchField &f = tab[tile * NF + j];
    d[j] = (step & 1) ? f.dB : f.dA;
    dn[j] = (step & 1) ? f.dA : f.dB;
    r[j] = f.r32;
    e[j] = f.e32;
  }
  const BatchField &f0 = tab[tile * NF];
  cheb32_tile<FIRST, NF>(L, f0.CH, U, Dsum, Bsum, DE, d, dn, r, e, f0.cheb[step], sb);
}

// x += e for every field (blockIdx.y = field); with a learned guess the
// field's new history collects every correction as well
__global__ void k_batch_add_e(int64_t n, const BatchField *__restrict__ tab) {
  const BatchField &f = tab[blockIdx.y];
  if (batch_field_done(f)) return;  // its Chebyshev steps were skipped too
  float2 *hn = f.hnew;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 e = f.e32[i];
    const double2 x = f.x[i];
    f.x[i] = make_double2(x.x + (double)e.x, x.y + (double)e.y);
    if (hn) {
      const float2 h = hn[i];
      hn[i] = make_float2(h.x + e.x, h.y + e.y);
    }
  }
}

template <bool FIRST, int NF, int MINB>
static void batch_cheb_nf(int order, dim3 grid, Lat L, const float2 *U, const float2 *Dsum, const float *Bsum,
                          const float2 *DE, const BatchField *tab, int ntiles, int64_t nsb, int step,
                          cudaStream_t st) {
  if (order == 0)
    k_batch_cheb32<FIRST, NF, 0, MINB><<<grid, 192, 0, st>>>(L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step);
  else
    k_batch_cheb32<FIRST, NF, 1, MINB><<<grid, 192, 0, st>>>(L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step);
}

int launch_batch_cheb(int step, int variant, int order, Lat L, const float2 *U, const float2 *Dsum,
                      const float *Bsum, const float2 *DE, const BatchField *tab, int nfields, cudaStream_t st) {
  const int nf_tile = variant == 2 ? 2 : 1;
  if (variant < 0 || variant >= BATCH_CHEB_VARIANTS || nfields % nf_tile != 0 || step < 0 ||
      step >= BATCH_MAX_CHEB)
    return 1;
  const int ntiles = nfields / nf_tile;
  const int64_t nsb = (L.V + 31) / 32;
  const dim3 grid((unsigned)(nsb * ntiles));
  const bool first = step == 0;
  if (variant == 0) {
    if (first) batch_cheb_nf<true, 1, 2>(order, grid, L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step, st);
    else batch_cheb_nf<false, 1, 2>(order, grid, L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step, st);
  } else if (variant == 1) {
    if (first) batch_cheb_nf<true, 1, 3>(order, grid, L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step, st);
    else batch_cheb_nf<false, 1, 3>(order, grid, L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step, st);
  } else {
    if (first) batch_cheb_nf<true, 2, 1>(order, grid, L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step, st);
    else batch_cheb_nf<false, 2, 1>(order, grid, L, U, Dsum, Bsum, DE, tab, ntiles, nsb, step, st);
  }
  return 0;
}
void launch_batch_add_e(int64_t n, const BatchField *tab, int nfields, cudaStream_t st) {
  const dim3 grid((unsigned)std::min<int64_t>((n + 255) / 256, 2048), (unsigned)nfields);
  k_batch_add_e<<<grid, 256, 0, st>>>(n, tab);
}

// x += e (FP64 += FP32), 72 planes
__global__ void k_add_e(int64_t n, double2 *__restrict__ X, const float2 *__restrict__ E) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 e = E[i];
  double2 x = X[i];
  X[i] = make_double2(x.x + (double)e.x, x.y + (double)e.y);
}

void launch_cn_to_f32(int64_t V, const double2 *U, const double2 *DE, const double2 *D, const double *B, float2 *U32,
                      float2 *DE32, float2 *D32, float *B32, cudaStream_t st) {
  k_cn_to_f32<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(V, U, DE, D, B, U32, DE32, D32, B32);
}
void launch_cn_bounds(Lat L, const CnCoef &C, double tau, const double2 *U, const double2 *Dsum, const double *Bsum,
                      const double2 *DE, double *partials, double *out, cudaStream_t st) {
  const int64_t nblk = (L.V + 255) / 256;
  k_cn_bounds<<<(unsigned)nblk, 256, 0, st>>>(L, C, tau, U, Dsum, Bsum, DE, partials);
  k_cn_bounds_final<<<1, 256, 0, st>>>(partials, nblk, out);
}
void launch_cheb32(bool first, Lat L, const CnCoef &C, const float2 *U, const float2 *Dsum, const float *Bsum,
                   const float2 *DE, const float2 *D, float2 *Dn, float2 *R, float2 *E, const ChebCoef &K,
                   cudaStream_t st) {
  const unsigned nb_ = (unsigned)((L.V + 31) / 32);
  if (first)
    k_cheb32<true><<<nb_, 192, 0, st>>>(L, C, U, Dsum, Bsum, DE, D, Dn, R, E, K);
  else
    k_cheb32<false><<<nb_, 192, 0, st>>>(L, C, U, Dsum, Bsum, DE, D, Dn, R, E, K);
}
void launch_add_e(int64_t n, double2 *X, const float2 *E, cudaStream_t st) {
  k_add_e<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, X, E);
}

}  // namespace nrq
