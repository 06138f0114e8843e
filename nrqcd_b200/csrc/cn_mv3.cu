// TMA-staged 12-column stencil of the assembled Crank-Nicolson operator
// (src/nrqcd.f90:1175-1387 with PETSc's block transposition; the operator
// is described in cn.cu).  out = in + sum_t alpha_t G_t in for both species.
//
// Persistent kernel, one CTA per SM.  A work unit is 32 consecutive sites
// (x0 = 32u).  Per unit, five stages stream through a three-buffer shared
// memory pipeline, each one a set of 2D TMA tiles 34 sites wide
// (cp.async.bulk.tensor, completion on an mbarrier):
//   stage 0: spinors at x0-1..x0+32 (centre plus both x neighbours),
//            U_x and DE_x at the same sites, Darwin D and magnetic B at x0..x0+31
//   stage 1: spinors at the +y row, U_y and DE_y at the centre sites
//   stage 2: spinors at the -y row, U_y and DE_y at the -y row
//   stage 3: spinors at the +z row, U_z and DE_z at the centre sites
//   stage 4: spinors at the -z row, U_z and DE_z at the -z row
// Thread 0 also acts as the producer: at every stage it first issues the TMA
// loads kBufs-1 stages ahead (after the buffer's previous use is released),
// then consumes its own stage.  Twelve warps, one per (species, output
// colour c, half of the columns), read only shared memory.  A thread owns the rows (c, s = 0, 1) of three
// propagator columns of its species and applies its two rows of the 6x6
// block, built once per neighbour, to its columns.  Lanes whose neighbour is
// not in a stage's tile (periodic wrap) address that neighbour in global
// memory instead: one generic pointer per lane and neighbour selects the
// source, so the inner loop carries no branch.
//
// Every mbarrier wait is bounded (about two seconds of clock64 cycles).  On
// expiry the thread records NRQ_ERR_TIMEOUT in *err and skips the remaining
// work without leaving any barrier unmatched.  The producer drains its
// in-flight copies (again bounded) before the CTA exits.
//
// Single-GPU code: the tiles are read from this GPU's own memory, and no
// load uses cluster multicast.
#include <algorithm>
#include <type_traits>

#include "../../include/nrqcd_b200.h"
#include "nrq_kernels.cuh"
#include "stage.cuh"

namespace nrq {

namespace mv3 {
constexpr int kUnit = 32;        // sites per work unit
constexpr int kTile = 34;        // tile width in sites
constexpr int kStages = 5;       // pipeline stages per unit
constexpr int kBufs = 3;         // shared-memory buffers
constexpr int kConsumerWarps = 12;  // (species, colour, column half)
constexpr int kCols = 3;            // propagator columns per consumer thread
constexpr int kThreads = kConsumerWarps * 32;
// byte offsets inside one buffer (TMA destinations 128-byte aligned)
constexpr int kOffSpin = 0;                          // 72 planes x 34 sites x 16 B = 39168
constexpr int kOffU = 39168;                         // 9 x 34 x 16 = 4896 (padded 4992)
constexpr int kOffDE = kOffU + 4992;                 // 18 x 34 x 16 = 9792 (padded 9856)
constexpr int kOffD = kOffDE + 9856;                 // 9 x 32 x 16 = 4608
constexpr int kOffB = kOffD + 4608;                  // 9 x 32 x 8 = 2304
constexpr int kBufBytes = kOffB + 2304;              // 60928
constexpr uint32_t kTxStage0 = 39168 + 4896 + 9792 + 4608 + 2304;
constexpr uint32_t kTxStage = 39168 + 4896 + 9792;
constexpr int kSmemBytes = kBufs * kBufBytes + 1024; // + alignment slack
}  // namespace mv3

struct Mv3Maps {
  CUtensorMap spin;  // 72 planes x 2V doubles, box {68, 72}
  CUtensorMap U;     // 27 planes x 2V doubles, box {68, 9}
  CUtensorMap DE;    // 54 planes x 2V doubles, box {68, 18}
  CUtensorMap D;     // 9 planes x 2V doubles, box {64, 9}
  CUtensorMap B;     // 9 planes x V doubles, box {32, 9}
};

// (s_K^T)[s][t] * v for the reference Pauli matrices (s_2 held transposed,
// so s_2^T = [[0,-i],[i,0]]); K, s, t resolve at compile time
template <int K>
__device__ __forceinline__ cplx sig_apply(int s, int t, cplx v) {
  if (K == 0) return (s != t) ? v : cplx{0.0, 0.0};
  if (K == 1) {
    if (s == 0 && t == 1) return -times_i(v);
    if (s == 1 && t == 0) return times_i(v);
    return {0.0, 0.0};
  }
  if (s != t) return {0.0, 0.0};
  return (s == 0) ? v : -v;
}

__device__ __forceinline__ cplx sigT3(int k, int s, int t) {
  if (k == 0) return (s != t) ? cplx{1.0, 0.0} : cplx{0.0, 0.0};
  if (k == 1) {
    if (s == 0 && t == 1) return {0.0, -1.0};
    if (s == 1 && t == 0) return {0.0, 1.0};
    return {0.0, 0.0};
  }
  if (s != t) return {0.0, 0.0};
  return (s == 0) ? cplx{1.0, 0.0} : cplx{-1.0, 0.0};
}

// first site of the spinor tile of stage st for unit start x0
__device__ __forceinline__ int64_t stage_spin_start(const Lat &L, int64_t x0, int st) {
  if (st == 0) return x0 - 1;
  const int i = (st + 1) / 2;          // 1,1,2,2
  const int sg = (st & 1) ? +1 : -1;  // stage 1,3: +; 2,4: -
  return nb(L, x0, i, sg);
}
// first site of the colour-matrix tiles of stage st
__device__ __forceinline__ int64_t stage_mat_start(const Lat &L, int64_t x0, int st) {
  if (st == 0 || st == 1 || st == 3) return x0 - 1;
  return stage_spin_start(L, x0, st);
}

template <int MODE>
__global__ void __launch_bounds__(mv3::kThreads, 1)
    k_cn_mv3(Lat L, CnCoef C, const __grid_constant__ Mv3Maps maps, const double2 *__restrict__ U,
             const double2 *__restrict__ DE, MvArgs A, int64_t nunits, int *err) {
  using namespace mv3;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kBufs], empty_bar[kBufs];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t V = L.V;

  if (threadIdx.x == 0) {
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(&full_bar[b], 1);
      mbar_init(&empty_bar[b], kConsumerWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // -------------------------------------------------------------- consumers
  const int sp = warp / 6, c = (warp / 2) % 3, half = warp % 2;
  const int col0 = half * kCols;
  const cplx ak = C.kin[sp], am = C.mag[sp], ad = C.dar[sp], aso = C.so[sp];
  const cplx cs0 = times_i(aso), cs1 = -times_i(aso);
  const int64_t pb = (int64_t)(sp * 36) * V;
  bool dead = false;
  // ---- producer role of thread 0: stage kk = (local unit) * kStages + stage
  const int64_t my_units = (nunits - blockIdx.x + gridDim.x - 1) / gridDim.x;
  const int64_t total = my_units * kStages;
  int64_t issued = 0;
  auto issue = [&](int64_t kk) {
    const int buf = (int)(kk % kBufs);
    const int64_t use = kk / kBufs;
    if (use > 0 && !mbar_wait(&empty_bar[buf], (uint32_t)((use - 1) & 1))) return false;
    const int64_t u = blockIdx.x + (kk / kStages) * gridDim.x;
    const int stg = (int)(kk % kStages);
    const int64_t x0 = u * kUnit;
    unsigned char *bb = smem + buf * kBufBytes;
    const int i = (stg == 0) ? 0 : (stg + 1) / 2;
    mbar_expect_tx(&full_bar[buf], stg == 0 ? kTxStage0 : kTxStage);
    const int64_t ss = stage_spin_start(L, x0, stg), ms = stage_mat_start(L, x0, stg);
    tma_2d(bb + kOffSpin, &maps.spin, (int)(2 * ss), 0, &full_bar[buf]);
    tma_2d(bb + kOffU, &maps.U, (int)(2 * ms), i * 9, &full_bar[buf]);
    tma_2d(bb + kOffDE, &maps.DE, (int)(2 * ms), i * 18, &full_bar[buf]);
    if (stg == 0) {
      tma_2d(bb + kOffD, &maps.D, (int)(2 * x0), 0, &full_bar[buf]);
      tma_2d(bb + kOffB, &maps.B, (int)x0, 0, &full_bar[buf]);
    }
    return true;
  };
  bool prod_dead = false;
  if (threadIdx.x == 0)
    for (; issued < total && issued < kBufs - 1; ++issued) issue(issued);
  int64_t k = 0;
  // begin stage k: issue ahead (thread 0), wait for this stage's tiles
  auto stage_begin = [&](int64_t kk) -> const unsigned char * {
    if (threadIdx.x == 0 && !prod_dead && issued < total) {
      if (issue(issued)) ++issued;
      else {
        prod_dead = true;
        record_timeout(err, 3, 0, -1);
      }
    }
    const int buf = (int)(kk % kBufs);
    if (!dead && !mbar_wait(&full_bar[buf], (uint32_t)((kk / kBufs) & 1))) {
      dead = true;
      record_timeout(err, 3, 0, -1);
    }
    return smem + buf * kBufBytes;
  };
  auto stage_end = [&](int64_t kk) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty_bar[kk % kBufs]);
  };

  for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
    const int64_t x0 = u * kUnit;
    const bool active = x0 + lane < V;
    const int64_t x = active ? x0 + lane : V - 1;
    cplx acc[kCols][2];
#pragma unroll
    for (int j = 0; j < kCols; ++j) acc[j][0] = acc[j][1] = cplx{0.0, 0.0};

    // spinor rows of this thread's columns at site y: generic base + plane stride
    auto spin_base = [&](const unsigned char *b, int64_t ss, int64_t y, int64_t &stride) -> const double2 * {
      const int64_t idx = y - ss;
      if (idx >= 0 && idx < kTile) {
        stride = kTile;
        return (const double2 *)(b + kOffSpin) + (sp * 36 + col0 * 6) * kTile + idx;
      }
      stride = V;
      return A.in + pb + (int64_t)(col0 * 6) * V + y;
    };
    // one neighbour block, direction I (0..2), DIR 0: x+I (matrices at x,
    // transposed), DIR 1: x-I (matrices at x-I, conjugated)
    auto neighbour = [&](auto Ic, auto DIRc, const unsigned char *b, int64_t ss, int64_t ms) {
      constexpr int I = decltype(Ic)::value, DIR = decltype(DIRc)::value;
      constexpr int K0 = (I + 2) % 3, K1 = (I + 1) % 3;
      const int64_t y = nb(L, x, I, DIR == 0 ? +1 : -1);
      const int64_t msite = DIR == 0 ? x : y;
      const int64_t midx = msite - ms;
      const bool mloc = midx >= 0 && midx < kTile;
      const bool mall = __all_sync(0xffffffffu, mloc);
      const uint32_t sUa = smem_u32(b + kOffU) + (uint32_t)(midx * 16), sDa = smem_u32(b + kOffDE) + (uint32_t)(midx * 16);
      const double2 *mU = mloc ? (const double2 *)(b + kOffU) + midx : U + (int64_t)(I * 9) * V + msite;
      const double2 *mD = mloc ? (const double2 *)(b + kOffDE) + midx : DE + (int64_t)(I * 18) * V + msite;
      const int64_t mst = mloc ? kTile : V;
      const cplx ck = (-0.5 * C.inva2[I]) * ak;
      const cplx s0 = DIR == 0 ? cs0 : -cs0, s1 = DIR == 0 ? cs1 : -cs1;
      cplx Wm[2][3][2];
#pragma unroll
      for (int cp = 0; cp < 3; ++cp) {
        const int e = DIR == 0 ? (cp * 3 + c) : (c * 3 + cp);  // M^T vs M^* index
        cplx uu, d0, d1;
        if (mall) {
          uu = lds2(sUa + (uint32_t)(e * kTile * 16));
          d0 = lds2(sDa + (uint32_t)(e * kTile * 16));
          d1 = lds2(sDa + (uint32_t)((9 + e) * kTile * 16));
        } else {
          uu = ld(mU + e * mst);
          d0 = ld(mD + e * mst);
          d1 = ld(mD + (9 + e) * mst);
        }
        if (DIR == 1) {
          uu = conj(uu);
          d0 = conj(d0);
          d1 = conj(d1);
        }
        const cplx ku = ck * uu, e0 = s0 * d0, e1 = s1 * d1;
        // W = ku (1) + e0 s_K0^T + e1 s_K1^T, s^T entries are 0, +-1, +-i
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
          for (int t = 0; t < 2; ++t) {
            cplx v = (s == t) ? ku : cplx{0.0, 0.0};
            v = v + sig_apply<K0>(s, t, e0);
            v = v + sig_apply<K1>(s, t, e1);
            Wm[s][cp][t] = v;
          }
      }
      const int64_t widx = y - ss;
      const bool wloc = widx >= 0 && widx < kTile;
      auto apply = [&](auto load) {
#pragma unroll
        for (int j = 0; j < kCols; ++j) {
          cplx w[6];
#pragma unroll
          for (int r = 0; r < 6; ++r) w[r] = load(j * 6 + r);
#pragma unroll
          for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int cp = 0; cp < 3; ++cp) {
              cmac(acc[j][s], Wm[s][cp][0], w[2 * cp]);
              cmac(acc[j][s], Wm[s][cp][1], w[2 * cp + 1]);
            }
        }
      };
      if (__all_sync(0xffffffffu, wloc)) {  // whole warp in the tile: shared loads
        const uint32_t sb = smem_u32(b + kOffSpin) + (uint32_t)(((sp * 36 + col0 * 6) * kTile + widx) * 16);
        apply([&](int pl) { return lds2(sb + (uint32_t)(pl * kTile * 16)); });
      } else {
        int64_t ws;
        const double2 *wb = spin_base(b, ss, y, ws);
        apply([&](int pl) { return ld(wb + pl * ws); });
      }
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;

    // ---- stage 0: diagonal block, +x, -x
    {
      const unsigned char *b = stage_begin(k);
      if (!dead) {
        const int64_t ss = x0 - 1, ms = x0 - 1;
        const uint32_t sD = smem_u32(b + kOffD), sB = smem_u32(b + kOffB);  // [9][32] each
        cplx Cd[3];
#pragma unroll
        for (int cp = 0; cp < 3; ++cp) {
          cplx dv = lds2(sD + (uint32_t)(((cp * 3 + c) * kUnit + lane) * 16));
          double bv = lds1(sB + (uint32_t)(((cp * 3 + c) * kUnit + lane) * 8));
          Cd[cp] = ad * dv + bv * am;
        }
        Cd[c] = Cd[c] + C.dkin * ak + cplx{1.0, 0.0};
        // centre spinors are always inside the stage-0 tile (index lane + 1)
        const uint32_t wb = smem_u32(b + kOffSpin) + (uint32_t)(((sp * 36 + col0 * 6) * kTile + lane + 1) * 16);
#pragma unroll
        for (int j = 0; j < kCols; ++j) {
          cplx w[6];
#pragma unroll
          for (int r = 0; r < 6; ++r) w[r] = lds2(wb + (uint32_t)((j * 6 + r) * kTile * 16));
#pragma unroll
          for (int s = 0; s < 2; ++s) {
            cplx a_ = Cd[0] * w[s];
            cmac(a_, Cd[1], w[2 + s]);
            cmac(a_, Cd[2], w[4 + s]);
            acc[j][s] = acc[j][s] + a_;
          }
        }
        neighbour(I0{}, I0{}, b, ss, ms);
        neighbour(I0{}, I1{}, b, ss, ms);
      }
      stage_end(k++);
    }
    // ---- stages 1-4: +y, -y, +z, -z
    {
      const unsigned char *b = stage_begin(k);
      if (!dead) neighbour(I1{}, I0{}, b, stage_spin_start(L, x0, 1), x0 - 1);
      stage_end(k++);
    }
    {
      const unsigned char *b = stage_begin(k);
      if (!dead) {
        const int64_t ss = stage_spin_start(L, x0, 2);
        neighbour(I1{}, I1{}, b, ss, ss);
      }
      stage_end(k++);
    }
    {
      const unsigned char *b = stage_begin(k);
      if (!dead) neighbour(I2{}, I0{}, b, stage_spin_start(L, x0, 3), x0 - 1);
      stage_end(k++);
    }
    {
      const unsigned char *b = stage_begin(k);
      if (!dead) {
        const int64_t ss = stage_spin_start(L, x0, 4);
        neighbour(I2{}, I1{}, b, ss, ss);
      }
      stage_end(k++);
    }

    // ------------------------------------------------------------ epilogue
    constexpr int NQ = (MODE == MV_T) ? 3 : ((MODE == MV_RES || MODE == MV_V || MODE == MV_RESC) ? 2 : 0);
    double q[kCols][3];
#pragma unroll
    for (int j = 0; j < kCols; ++j) q[j][0] = q[j][1] = q[j][2] = 0.0;
    if (active && !dead) {
#pragma unroll
      for (int j = 0; j < kCols; ++j)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const int64_t o = pb + (int64_t)((col0 + j) * 6 + 2 * c + s) * V + x;
          const cplx y_ = acc[j][s];
          if (MODE == MV_PLAIN) {
            st(A.out + o, y_);
          } else if (MODE == MV_RHS) {
            st(A.out + o, y_);
            st(A.out2 + o, 2.0 * y_ - ldg(A.in + o));
          } else if (MODE == MV_RES) {
            const cplx bb = ldg(A.bvec + o);
            const cplx r = bb - y_;
            st(A.out + o, r);
            st(A.out2 + o, r);
            st(A.out3 + o, r);
            q[j][0] += norm2(r);
            q[j][1] += norm2(bb);
          } else if (MODE == MV_V) {
            st(A.out + o, y_);
            cplx d = {0.0, 0.0};
            cmac_cj(d, ldg(A.in2 + o), y_);
            q[j][0] += d.re;
            q[j][1] += d.im;
          } else if (MODE == MV_RESC) {
            const cplx bb = ldg(A.bvec + o);
            const cplx r = bb - y_;
            const cplx dd = r * A.inv_theta[sp];
            A.r32[o] = make_float2((float)r.re, (float)r.im);
            A.d32[o] = make_float2((float)dd.re, (float)dd.im);
            q[j][0] += norm2(r);
            q[j][1] += norm2(bb);
          } else {  // MV_T: in = s
            st(A.out + o, y_);
            cplx d = {0.0, 0.0};
            cmac_cj(d, y_, ldg(A.in + o));
            q[j][0] += d.re;
            q[j][1] += d.im;
            q[j][2] += norm2(y_);
          }
        }
    }
    if constexpr (NQ > 0) {
      // one partial row per (unit, colour warp): row = u*3 + c, column col12
#pragma unroll
      for (int j = 0; j < kCols; ++j)
#pragma unroll
        for (int kq = 0; kq < NQ; ++kq) {
          double v = q[j][kq];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
          if (lane == 0) A.partials[((u * 3 + c) * CN_COLS + sp * 6 + col0 + j) * NQ + kq] = v;
        }
    }
  }
  // error path: copies issued ahead of the consumers must land before exit
  if (threadIdx.x == 0 && dead)
    for (int64_t kk = k; kk < issued; ++kk)
      if (!mbar_wait(&full_bar[kk % kBufs], (uint32_t)((kk / kBufs) & 1))) record_timeout(err, 3, 0, -1);
}

// ------------------------------------------------------------------ host
using stage::encode;

int launch_cn_mv3(int mode, Lat L, const CnCoef &C, const double2 *U, const double2 *Dsum, const double *Bsum,
                  const double2 *DE, const MvArgs &a, int *err, int sm_count, cudaStream_t st) {
  using namespace mv3;
  const uint64_t V = (uint64_t)L.V;
  Mv3Maps maps;
  if (!encode(&maps.spin, a.in, 2 * V, 72, 2 * kTile, 72) || !encode(&maps.U, U, 2 * V, 27, 2 * kTile, 9) ||
      !encode(&maps.DE, DE, 2 * V, 54, 2 * kTile, 18) || !encode(&maps.D, Dsum, 2 * V, 9, 2 * kUnit, 9) ||
      !encode(&maps.B, Bsum, V, 9, kUnit, 9))
    return -1;
  const int64_t nunits = (L.V + kUnit - 1) / kUnit;
  const unsigned grid = (unsigned)std::min<int64_t>(nunits, sm_count);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    kern<<<grid, kThreads, kSmemBytes, st>>>(L, C, maps, U, DE, a, nunits, err);
  };
  switch (mode) {
    case MV_PLAIN: go(k_cn_mv3<MV_PLAIN>); break;
    case MV_RHS: go(k_cn_mv3<MV_RHS>); break;
    case MV_RES: go(k_cn_mv3<MV_RES>); break;
    case MV_V: go(k_cn_mv3<MV_V>); break;
    case MV_RESC: go(k_cn_mv3<MV_RESC>); break;
    default: go(k_cn_mv3<MV_T>); break;
  }
  return 0;
}

}  // namespace nrq
