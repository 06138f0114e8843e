// Register-tiled 12-column stencil of the assembled Crank-Nicolson operator
// (used where the TMA-staged stencil of cn_mv3.cu cannot describe the
// lattice with tensor maps, i.e. odd V or V < 64)
// (src/nrqcd.f90:1175-1387 with PETSc's block transposition), applied
// matrix-free: out = in + sum_t alpha_t G_t in for both species at once.
// See cn.cu for the operator; this file holds its stencil kernel.
//
// Work split.  A block covers 32 consecutive sites with 6 warps, one warp per
// (species, output colour c).  A thread owns the output rows (c, s=0,1) of
// all 6 propagator columns of its species (12 complex accumulators).  Per
// neighbour it builds its two rows of the species-specific 6x6 block
//   W = ck (K0^T x 1) + cs0 (X0^T x s_k0^T) + cs1 (X1^T x s_k1^T)
// once (12 complex entries, colour row c) and reuses them from registers for
// the 6 columns: 36 complex multiply-adds per column per neighbour, the
// minimum for a dense 6x6 block.  The three colour warps of a species read
// the same neighbour spinors; those reads hit L1.
#include <type_traits>

#include "nrq_kernels.cuh"

// tuning parameters of the stencil kernel (blocks per SM for the register
// budget, unroll depth of the column loop)
#ifndef NRQ_MV_MINB
#define NRQ_MV_MINB 2
#endif
#ifndef NRQ_MV_UNROLL_COL
#define NRQ_MV_UNROLL_COL 2
#endif

namespace nrq {

constexpr int kMvUnrollCol = NRQ_MV_UNROLL_COL;

// v times entry (s, t) of the transposed reference Pauli matrix s_K^T
// (src/su2.f90:68-79 holds s_2 transposed, so s_2^T = [[0,-i],[i,0]]); with
// K, s and t known at compile time this is a sign flip or a swap
template <int K>
__device__ __forceinline__ cplx sig_mul(int s, int t, cplx v) {
  if (K == 0) return (s != t) ? v : cplx{0.0, 0.0};
  if (K == 1) {
    if (s == 0 && t == 1) return -times_i(v);
    if (s == 1 && t == 0) return times_i(v);
    return {0.0, 0.0};
  }
  if (s != t) return {0.0, 0.0};
  return (s == 0) ? v : -v;
}

__device__ __forceinline__ cplx scal_col(const double *sc, int col12, int slot) {
  return {sc[col12 * SC_STRIDE + slot], sc[col12 * SC_STRIDE + slot + 1]};
}

template <int MODE>
__device__ __forceinline__ void cn_mv2_body(const Lat &L, const CnCoef &C, const double2 *__restrict__ U,
                                            const double2 *__restrict__ Dsum, const double *__restrict__ Bsum,
                                            const double2 *__restrict__ DE, const MvArgs &A, int64_t block,
                                            int64_t partial_row) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;  // 0..5
  const int sp = warp / 3, c = warp % 3;
  const int64_t V = L.V;
  const int64_t x0 = block * 32 + lane;
  const bool active = x0 < V;
  const int64_t x = active ? x0 : 0;
  const int64_t pb = (int64_t)(sp * 36) * V;

  cplx al[6];
  if (MODE == MV_T) {
#pragma unroll
    for (int col = 0; col < 6; ++col) al[col] = scal_col(A.scal, sp * 6 + col, SC_ALPHA);
  }
  // 6-component spinor of column col at site y (MV_T: s = r - alpha v on the fly)
  auto load_w = [&](int64_t y, int col, cplx w[6]) {
    const double2 *p = A.in + pb + (int64_t)(col * 6) * V + y;
#pragma unroll
    for (int r = 0; r < 6; ++r) w[r] = ldg(p + (int64_t)r * V);
    if (MODE == MV_T && A.in2 != nullptr) {
      const double2 *q = A.in2 + pb + (int64_t)(col * 6) * V + y;
#pragma unroll
      for (int r = 0; r < 6; ++r) w[r] = w[r] - al[col] * ldg(q + (int64_t)r * V);
    }
  };

  const cplx ak = C.kin[sp], am = C.mag[sp], ad = C.dar[sp], aso = C.so[sp];
  cplx acc[6][2];
  // ---- diagonal block: [1 + ak dkin] 1 + ad D^T + am B^T, colour row c
  {
    cplx Cd[3];
#pragma unroll
    for (int cp = 0; cp < 3; ++cp) {
      cplx dv = ldg(Dsum + (int64_t)(cp * 3 + c) * V + x);
      double bv = __ldg(Bsum + (int64_t)(cp * 3 + c) * V + x);
      Cd[cp] = ad * dv + bv * am;
    }
    Cd[c] = Cd[c] + C.dkin * ak + cplx{1.0, 0.0};
#pragma unroll
    for (int col = 0; col < 6; ++col) {
      cplx w[6];
      load_w(x, col, w);
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        cplx a_ = Cd[0] * w[s];
        cmac(a_, Cd[1], w[2 + s]);
        cmac(a_, Cd[2], w[4 + s]);
        acc[col][s] = a_;
      }
    }
  }
  const cplx cs0 = times_i(aso);   // eps = +1 permutation (j,k) = (i+1, i+2)
  const cplx cs1 = -times_i(aso);  // eps = -1 permutation (j,k) = (i+2, i+1)
  // one neighbour, direction I and side DIR known at compile time, so the
  // Pauli factors of the block fold to sign flips and swaps
  // (DIR 0: neighbour x+I, blocks from site x, transposed;
  //  DIR 1: neighbour x-I, blocks from site x-I, complex conjugated)
  auto neighbour = [&](auto Ic, auto DIRc) {
    constexpr int I = decltype(Ic)::value, DIR = decltype(DIRc)::value;
    constexpr int K0 = (I + 2) % 3, K1 = (I + 1) % 3;
    const cplx ck = (-0.5 * C.inva2[I]) * ak;
    const int64_t y = nb(L, x, I, DIR == 0 ? +1 : -1);
    const int64_t ms = DIR == 0 ? x : y;
    const double2 *Up = U + (int64_t)(I * 9) * V + ms;
    const double2 *D0 = DE + (int64_t)((I * 2 + 0) * 9) * V + ms;
    const double2 *D1 = DE + (int64_t)((I * 2 + 1) * 9) * V + ms;
    const cplx s0 = DIR == 0 ? cs0 : -cs0, s1 = DIR == 0 ? cs1 : -cs1;
    cplx Wm[2][3][2];
#pragma unroll
    for (int cp = 0; cp < 3; ++cp) {
      const int e = DIR == 0 ? (cp * 3 + c) : (c * 3 + cp);  // M^T[c][cp] = M[cp][c] ; M^*[c][cp]
      cplx u = ldg(Up + (int64_t)e * V), d0 = ldg(D0 + (int64_t)e * V), d1 = ldg(D1 + (int64_t)e * V);
      if (DIR == 1) {
        u = conj(u);
        d0 = conj(d0);
        d1 = conj(d1);
      }
      const cplx ku = ck * u, e0 = s0 * d0, e1 = s1 * d1;
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          cplx v = (s == t) ? ku : cplx{0.0, 0.0};
          v = v + sig_mul<K0>(s, t, e0);
          v = v + sig_mul<K1>(s, t, e1);
          Wm[s][cp][t] = v;
        }
    }
#pragma unroll kMvUnrollCol
    for (int col = 0; col < 6; ++col) {
      cplx w[6];
      load_w(y, col, w);
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int cp = 0; cp < 3; ++cp) {
          cmac(acc[col][s], Wm[s][cp][0], w[2 * cp]);
          cmac(acc[col][s], Wm[s][cp][1], w[2 * cp + 1]);
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

  // ---------------- epilogue by mode; rows (c, s) of the 6 columns
  constexpr int NQ = (MODE == MV_T) ? 3 : ((MODE == MV_RES || MODE == MV_V || MODE == MV_RESC) ? 2 : 0);
  double q[6][3];
#pragma unroll
  for (int col = 0; col < 6; ++col)
#pragma unroll
    for (int k = 0; k < 3; ++k) q[col][k] = 0.0;
  if (active) {
#pragma unroll
    for (int col = 0; col < 6; ++col)
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int64_t o = pb + (int64_t)(col * 6 + 2 * c + s) * V + x;
        const cplx y_ = acc[col][s];
        if (MODE == MV_PLAIN) {
          st(A.out + o, y_);
        } else if (MODE == MV_RHS) {
          st(A.out + o, y_);
          st(A.out2 + o, 2.0 * y_ - ldg(A.in + o));
        } else if (MODE == MV_RES) {
          const cplx b = ldg(A.bvec + o);
          const cplx r = b - y_;
          st(A.out + o, r);
          st(A.out2 + o, r);
          st(A.out3 + o, r);
          q[col][0] += norm2(r);
          q[col][1] += norm2(b);
        } else if (MODE == MV_V) {
          st(A.out + o, y_);
          cplx d = {0.0, 0.0};
          cmac_cj(d, ldg(A.in2 + o), y_);
          q[col][0] += d.re;
          q[col][1] += d.im;
        } else if (MODE == MV_RESC) {
          const cplx b = ldg(A.bvec + o);
          const cplx r = b - y_;
          const cplx dd = r * A.inv_theta[sp];
          A.r32[o] = make_float2((float)r.re, (float)r.im);
          A.d32[o] = make_float2((float)dd.re, (float)dd.im);
          q[col][0] += norm2(r);
          q[col][1] += norm2(b);
        } else {  // MV_T
          st(A.out + o, y_);
          const cplx s_ = A.in2 ? ldg(A.in + o) - al[col] * ldg(A.in2 + o) : ldg(A.in + o);
          cplx d = {0.0, 0.0};
          cmac_cj(d, y_, s_);
          q[col][0] += d.re;
          q[col][1] += d.im;
          q[col][2] += norm2(y_);
        }
      }
  }
  if constexpr (NQ > 0) {
    __shared__ double sh[6][6][3];
#pragma unroll
    for (int col = 0; col < 6; ++col)
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        double v = q[col][k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[warp][col][k] = v;
      }
    __syncthreads();
    if (threadIdx.x < 12 * NQ) {
      const int col12 = threadIdx.x / NQ, k = threadIdx.x % NQ;
      const int spp = col12 / 6, col = col12 % 6;
      const double v = sh[spp * 3 + 0][col][k] + sh[spp * 3 + 1][col][k] + sh[spp * 3 + 2][col][k];
      A.partials[(partial_row * CN_COLS + col12) * NQ + k] = v;
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(192, NRQ_MV_MINB) k_cn_mv2(Lat L, CnCoef C, const double2 *__restrict__ U,
                                                   const double2 *__restrict__ Dsum, const double *__restrict__ Bsum,
                                                   const double2 *__restrict__ DE, MvArgs A) {
  cn_mv2_body<MODE>(L, C, U, Dsum, Bsum, DE, A, blockIdx.x, blockIdx.x);
}

// ------------------------------------------------------------------ batched
// One launch over every field of a batch.  The flattened block index splits
// into (field, site block), field fastest (ORDER 0) or site block fastest
// (ORDER 1); pointers and mass-dependent coefficients come from the device
// table.  MV_RHS: b = A psi, x = 2b - psi.  MV_RESC: r32 = f32(b - A^H x),
// d32 = r32 / theta, with the per-column (r.r, b.b) partials of the field.
template <int MODE, int ORDER>
__global__ void __launch_bounds__(192, NRQ_MV_MINB) k_batch_mv2(Lat L, const double2 *__restrict__ U,
                                                      const double2 *__restrict__ Dsum,
                                                      const double *__restrict__ Bsum,
                                                      const double2 *__restrict__ DE,
                                                      const BatchField *__restrict__ tab, int nfields,
                                                      int64_t nsb, int skip_done) {
  const int64_t bid = blockIdx.x;
  const int fi = ORDER == 0 ? (int)(bid % nfields) : (int)(bid / nsb);
  const int64_t sb = ORDER == 0 ? bid / nfields : bid % nsb;
  const BatchField &f = tab[fi];
  if (MODE == MV_RESC && skip_done && batch_field_done(f)) return;  // uniform per block
  MvArgs a{};
  if (MODE == MV_RHS) {
    a.in = f.psi;
    a.out = f.b;
    a.out2 = f.x;
    cn_mv2_body<MV_RHS>(L, f.CA, U, Dsum, Bsum, DE, a, sb, sb);
  } else {
    a.in = f.x;
    a.bvec = f.b;
    a.r32 = f.r32;
    a.d32 = f.dA;
    a.partials = f.partials;
    a.inv_theta[0] = f.inv_theta[0];
    a.inv_theta[1] = f.inv_theta[1];
    cn_mv2_body<MV_RESC>(L, f.CH, U, Dsum, Bsum, DE, a, sb, sb);
  }
}

template <int MODE>
static void batch_mv_mode(int order, dim3 grid, Lat L, const double2 *U, const double2 *Dsum, const double *Bsum,
                          const double2 *DE, const BatchField *tab, int nfields, int64_t nsb, int skip_done,
                          cudaStream_t st) {
  if (order == 0)
    k_batch_mv2<MODE, 0><<<grid, 192, 0, st>>>(L, U, Dsum, Bsum, DE, tab, nfields, nsb, skip_done);
  else
    k_batch_mv2<MODE, 1><<<grid, 192, 0, st>>>(L, U, Dsum, Bsum, DE, tab, nfields, nsb, skip_done);
}

void launch_batch_mv(int mode, int order, Lat L, const double2 *U, const double2 *Dsum, const double *Bsum,
                     const double2 *DE, const BatchField *tab, int nfields, int skip_done, cudaStream_t st) {
  const int64_t nsb = (L.V + 31) / 32;
  const dim3 grid((unsigned)(nsb * nfields));
  if (mode == MV_RHS)
    batch_mv_mode<MV_RHS>(order, grid, L, U, Dsum, Bsum, DE, tab, nfields, nsb, 0, st);
  else
    batch_mv_mode<MV_RESC>(order, grid, L, U, Dsum, Bsum, DE, tab, nfields, nsb, skip_done, st);
}

void launch_cn_mv(int mode, Lat L, const CnCoef &C, const double2 *U, const double2 *Dsum, const double *Bsum,
                  const double2 *DE, const MvArgs &a, cudaStream_t st) {
  const unsigned nb_ = (unsigned)((L.V + 31) / 32);
  const dim3 blk(192);
  switch (mode) {
    case MV_PLAIN: k_cn_mv2<MV_PLAIN><<<nb_, blk, 0, st>>>(L, C, U, Dsum, Bsum, DE, a); break;
    case MV_RHS: k_cn_mv2<MV_RHS><<<nb_, blk, 0, st>>>(L, C, U, Dsum, Bsum, DE, a); break;
    case MV_RES: k_cn_mv2<MV_RES><<<nb_, blk, 0, st>>>(L, C, U, Dsum, Bsum, DE, a); break;
    case MV_V: k_cn_mv2<MV_V><<<nb_, blk, 0, st>>>(L, C, U, Dsum, Bsum, DE, a); break;
    case MV_RESC: k_cn_mv2<MV_RESC><<<nb_, blk, 0, st>>>(L, C, U, Dsum, Bsum, DE, a); break;
    default: k_cn_mv2<MV_T><<<nb_, blk, 0, st>>>(L, C, U, Dsum, Bsum, DE, a); break;
  }
}

}  // namespace nrq
