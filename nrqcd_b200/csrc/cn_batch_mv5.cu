// FP64 FMA stencil of the batching form: the right-hand side (MV_RHS: b = A
// psi, x = 2b - psi) and the refinement residual (MV_RESC: r = b - A^H x
// rounded to FP32, d = r / theta, and the per-column (r.r, b.b) partial
// sums) of every field of a batch in one persistent launch, on per-update
// FP64 blocks of every distinct mass (k_cn_blocks5, built with that mass's
// A^H coefficients; A is the same blocks with the neighbour sum negated, as
// in cn_mv5.cu).  The operator is the FP64 FMA stencil's; the schedule and
// the epilogues are k_batch_mv2's (cn_mv.cu).
//
// Work items (field, unit of 32 sites), field fastest (order 0) or unit
// fastest (order 1); a field that converged at its last check sits a
// residual out.  The fields' FP64 propagators and iterates are separate
// allocations that change places every step, so each field has tensor maps
// of its own in device memory (CnBatchMaps: psi and x, each a 34-site tile
// map and a one-site column map), written by the host before every step.
//
// Products.  A thread owns a 3 x 3 tile of one site and species: the three
// output rows of one spin and three of the six columns; per neighbour and
// input row it reads 3 block entries and 3 spinor entries from shared memory
// and does 36 FP64 FMAs.  Pipeline.  Persistent, one CTA per SM: 8 consumer
// warps (warp 4 sp + 2 s + h) and one producer warp.  Ten loads per item, per
// stage and species (stage 0: diagonal matrices, +x and -x; 1: +y; 2: -y; 3:
// +z; 4: -z): a spinor tile (34 sites x 36 planes) and a block tile by TMA,
// into a ring of four buffers completed on mbarriers.  The periodic x
// neighbours that wrap outside a unit's tile arrive as one-site columns with
// stage 0; a lane whose neighbour lies anywhere else outside the tiles reads
// it from global memory.  The epilogue's operand at the own site is loaded
// into registers two stages ahead.  The residual's partial sums of a unit
// are summed over the lanes and the two spin warps of a column (a pair
// barrier, no atomics: the same sums in the same order every launch) into
// one row per (field, unit), the rows k_batch_finalize reads.
//
// Every mbarrier wait is bounded (wait_cycles); on expiry the thread records
// NRQ_ERR_TIMEOUT in *err and skips the remaining work.  The producer never
// has two loads in flight into one buffer and, before it exits, waits
// (bounded) until every load it issued has landed.  Single-GPU code: no load
// uses cluster multicast.
#include <algorithm>
#include <cstring>

#include "../../include/nrqcd_b200.h"
#include "nrq_kernels.cuh"
#include "stage.cuh"

namespace nrq {

namespace bm5 {
constexpr int kUnit = 32;
constexpr int kWarps = 8;
constexpr int kThreads = (kWarps + 1) * 32;
constexpr int kStages = 5;
constexpr int kLoads = 2 * kStages;  // load i is of species i & 1
// an even ring: every buffer holds the loads of one species only
constexpr int kBufs = 4;
constexpr int kTileS = kUnit + 2;                      // x0 - 1 .. x0 + 32
constexpr uint32_t kTileBytes = 36u * kTileS * 16u;    // 19584
constexpr uint32_t kOffW = kTileBytes;
constexpr uint32_t kOffX = 2u * kTileBytes;            // the x-wrap columns
constexpr uint32_t kColBytes = 36u * 16u;              // 576
constexpr uint32_t kColStride = 640u;
constexpr uint32_t kBufBytes = ((kOffX + 3u * kColStride) + 1023u) & ~1023u;  // 41984
constexpr uint32_t kDiagD = 9u * kUnit * 16u;          // 4608
constexpr uint32_t kDiagB = 9u * kUnit * 8u;           // 2304
constexpr uint32_t kDiagStride = 7168u;
constexpr uint32_t kOffDiag = kBufs * kBufBytes;       // 167936
constexpr uint32_t kSmemBytes = kOffDiag + 2u * kDiagStride + 1024u;  // 183296
static_assert(kOffW % 128 == 0 && kOffX % 128 == 0 && kColStride % 128 == 0 && kColStride >= kColBytes &&
                  kBufBytes % 1024 == 0 && kDiagStride % 128 == 0 && kDiagD + kDiagB <= kDiagStride,
              "layout");
static_assert(kSmemBytes + 1024 <= 232448, "shared memory");
static_assert(kBufs % 2 == 0 && kLoads % 2 == 0, "a buffer's uses must all belong to one species");
}  // namespace bm5

struct BatchMv5Maps {
  CUtensorMap W;   // 216 planes per block set x 2V doubles, box {68, 36}
  CUtensorMap W1;  // one site: box {2, 36}
  CUtensorMap D;   // 9 planes x 2V doubles, box {64, 9}
  CUtensorMap B;   // 9 planes x V doubles, box {32, 9}
};

namespace {

struct UnitPosB {
  int x0, cx, cy, cz;
};
__device__ __forceinline__ UnitPosB unit_pos_b(const Lat &L, int x0) {
  const int nx = (int)L.nx, ny = (int)L.ny;
  const int t = x0 / nx, z = t / ny;
  return {x0, x0 - t * nx, t - z * ny, z};
}
__device__ __forceinline__ void neighbours_b(const Lat &L, const UnitPosB &P, int l, int (&nb)[6]) {
  const int nx = (int)L.nx, ny = (int)L.ny, nz = (int)L.nz;
  int x = P.cx + l, y = P.cy, z = P.cz;
  while (x >= nx) {
    x -= nx;
    if (++y == ny) {
      y = 0;
      ++z;
    }
  }
  const int s = P.x0 + l;
  const int row = nx, plane = nx * ny;
  nb[0] = x + 1 < nx ? s + 1 : s - (nx - 1);
  nb[1] = x > 0 ? s - 1 : s + (nx - 1);
  nb[2] = y + 1 < ny ? s + row : s - (ny - 1) * row;
  nb[3] = y > 0 ? s - row : s + (ny - 1) * row;
  nb[4] = z + 1 < nz ? s + plane : s - (nz - 1) * plane;
  nb[5] = z > 0 ? s - plane : s + (nz - 1) * plane;
}
// first site of the spinor tile of a stage (stage 0: x0 - 1; stages 1-4:
// the +y, -y, +z, -z neighbours of x0)
__device__ __forceinline__ int spin_start_b(const Lat &L, const UnitPosB &P, int stg) {
  const int x0 = P.x0;
  if (stg == 0) return x0 - 1;
  const int ny = (int)L.ny, nz = (int)L.nz;
  const int row = (int)L.nx, plane = (int)(L.nx * L.ny);
  switch (stg) {
    case 1: return P.cy + 1 < ny ? x0 + row : x0 - (ny - 1) * row;
    case 2: return P.cy > 0 ? x0 - row : x0 + (ny - 1) * row;
    case 3: return P.cz + 1 < nz ? x0 + plane : x0 - (nz - 1) * plane;
    default: return P.cz > 0 ? x0 - plane : x0 + (nz - 1) * plane;
  }
}
__device__ __forceinline__ int blk_start_b(int x0, int spin_start, int stg) {
  if (stg == 1 || stg == 3) return x0;
  return spin_start;
}
__device__ __forceinline__ void x_wraps_b(const Lat &L, const UnitPosB &P, int &yl, int &yr) {
  const int nx = (int)L.nx, V = (int)L.V, x0 = P.x0;
  yl = yr = -1;
  if (nx < bm5::kTileS) return;
  const int pl = P.cx == 0 ? 0 : nx - P.cx, pr = nx - 1 - P.cx;
  if (pl < bm5::kUnit && x0 + pl < V) yl = x0 + pl + nx - 1;
  if (pr < bm5::kUnit && x0 + pr < V) yr = x0 + pr - (nx - 1);
}

__device__ __forceinline__ double2 lds_d2b(uint32_t a) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ double lds_d1b(uint32_t a) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}

// The thread's tile (rows 2c + s; columns 3h + k) += sum over q of w[c][q]
// psi[q][3h + k].  Forward: w = W(x)[2c+s][q], entry (2c+s)*6 + q; backward:
// w = -conj(W(y)[q][2c+s]), entry q*6 + 2c + s.
template <bool BWD, typename LW, typename LP>
__device__ __forceinline__ void nb_products_b(double (&acc)[3][3][2], int s, int h, LW load_w, LP load_p) {
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double wr[3], wi[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double2 wv = load_w(BWD ? q * 6 + 2 * c + s : (2 * c + s) * 6 + q);
      wr[c] = BWD ? -wv.x : wv.x;
      wi[c] = wv.y;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 p = load_p((3 * h + k) * 6 + q);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc[c][k][0] = fma(wr[c], p.x, fma(-wi[c], p.y, acc[c][k][0]));
        acc[c][k][1] = fma(wr[c], p.y, fma(wi[c], p.x, acc[c][k][1]));
      }
    }
  }
}

}  // namespace

template <int MODE>
__global__ void __launch_bounds__(bm5::kThreads, 1)
    k_batch_mv5(Lat L, const __grid_constant__ BatchMv5Maps maps, const CnBatchMaps *__restrict__ fmaps,
                const double2 *__restrict__ W, const BatchField *__restrict__ tab, int nfields, int nunits, int order,
                int skip_done, int *err, long long wait_cycles) {
  using namespace bm5;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kBufs], empty_bar[kBufs], dfull[2], dempty[2];
  // per unit parity, species and column half: the spin-1 warp's column sums
  __shared__ double red[2][2][2][3][2];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int V = (int)L.V;
  const int nwork = nfields * nunits;
  // the input of the mode: psi (RHS) or the iterate x (RESC)
  constexpr int kIn = MODE == MV_RHS ? 0 : 1;
  const double nb_sign = MODE == MV_RHS ? -1.0 : 1.0;

  if (threadIdx.x == 0) {
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(&full_bar[b], 1);
      mbar_init(&empty_bar[b], 4);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], 1);
      mbar_init(&dempty[b], kWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  auto wait = [&](uint64_t *bar, uint32_t parity) -> bool {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
      if (clock64() - t0 > wait_cycles) return false;
    return true;
  };
  auto item = [&](int w, int &f, int &u) {
    if (order == 0) {
      f = w % nfields;
      u = w / nfields;
    } else {
      f = w / nunits;
      u = w % nunits;
    }
  };
  auto skip = [&](int f) { return MODE == MV_RESC && skip_done && batch_field_done(tab[f]); };

  // ---------------------------------------------------------- producer
  if (warp == kWarps) {
    if (lane == 0) {
      bool ok = true;
      int i = 0, k = 0;
      for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x) {
        int f, u;
        item(w, f, u);
        if (skip(f)) continue;
        const UnitPosB P = unit_pos_b(L, u * kUnit);
        const int x0 = P.x0;
        const CUtensorMap *spin = &fmaps[f].in[kIn].spin, *spin1 = &fmaps[f].in[kIn].spin1;
        const int wrow = tab[f].wblk * 216;
        {
          const int db = k & 1;
          if (k >= 2) {
            const uint32_t dpar = (uint32_t)((k / 2 - 1) & 1);
            if (!wait(&dempty[db], dpar)) {
              record_timeout(err, 7, 2, i);
              ok = false;
            } else if (!mbar_wait(&dfull[db], dpar)) {
              record_timeout(err, 7, 3, i);
              ok = false;
            }
            if (!ok) break;
          }
          unsigned char *dd = smem + kOffDiag + db * kDiagStride;
          mbar_expect_tx(&dfull[db], kDiagD + kDiagB);
          tma_2d(dd, &maps.D, 2 * x0, 0, &dfull[db]);
          tma_2d(dd + kDiagD, &maps.B, x0, 0, &dfull[db]);
        }
        for (int li = 0; li < kLoads && ok; ++li, ++i) {
          const int b = i % kBufs;
          if (i >= kBufs) {
            const uint32_t par = (uint32_t)((i / kBufs - 1) & 1);
            if (!wait(&empty_bar[b], par)) {
              record_timeout(err, 7, 2, i);
              ok = false;
            } else if (!mbar_wait(&full_bar[b], par)) {
              record_timeout(err, 7, 3, i);
              ok = false;
            }
            if (!ok) break;
          }
          const int stg = li >> 1, sp = li & 1;
          const int ss = spin_start_b(L, P, stg);
          const int ws = blk_start_b(x0, ss, stg);
          const int I = stg == 0 ? 0 : (stg + 1) / 2;
          unsigned char *bb = smem + b * kBufBytes;
          int yl = -1, yr = -1;
          if (stg == 0) x_wraps_b(L, P, yl, yr);
          uint32_t tx = 2u * kTileBytes;
          if (stg == 0) tx += (yl >= 0 ? 2u : 0u) * kColBytes + (yr >= 0 ? kColBytes : 0u);
          mbar_expect_tx(&full_bar[b], tx);
          tma_2d(bb, spin, 2 * ss, sp * 36, &full_bar[b]);
          tma_2d(bb + kOffW, &maps.W, 2 * ws, wrow + (I * 2 + sp) * 36, &full_bar[b]);
          if (stg == 0) {
            if (yl >= 0) {
              tma_2d(bb + kOffX, spin1, 2 * yl, sp * 36, &full_bar[b]);
              tma_2d(bb + kOffX + kColStride, &maps.W1, 2 * yl, wrow + sp * 36, &full_bar[b]);
            }
            if (yr >= 0) tma_2d(bb + kOffX + 2 * kColStride, spin1, 2 * yr, sp * 36, &full_bar[b]);
          }
        }
        ++k;
      }
      for (int j = max(0, i - kBufs); j < i; ++j)
        if (!mbar_wait(&full_bar[j % kBufs], (uint32_t)((j / kBufs) & 1))) {
          record_timeout(err, 7, 4, j);
          break;
        }
      for (int j = max(0, k - 2); j < k; ++j)
        if (!mbar_wait(&dfull[j & 1], (uint32_t)((j >> 1) & 1))) {
          record_timeout(err, 7, 4, -1 - j);
          break;
        }
    }
    return;
  }

  // ---------------------------------------------------------- consumers
  const int sp = warp >> 2, s = (warp >> 1) & 1, h = warp & 1;
  const int site_in_unit = lane;
  const int pair_bar = 2 + 2 * sp + h;  // the two spin warps of (species, column half)
  bool dead = false;

  int k = 0;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    int f, u;
    item(w, f, u);
    if (skip(f)) continue;
    const BatchField &F = tab[f];
    const CnCoef &C = MODE == MV_RHS ? F.CA : F.CH;
    const double2 *in = MODE == MV_RHS ? F.psi : F.x;
    const double2 *Wf = W + (int64_t)F.wblk * 216 * V;
    const cplx ak = C.kin[sp], am = C.mag[sp], ad = C.dar[sp];
    const cplx dg = C.dkin * ak + cplx{1.0, 0.0};

    const UnitPosB P = unit_pos_b(L, u * kUnit);
    const int x0 = P.x0;
    const int x = x0 + site_in_unit;
    const bool act = x < V;
    const int xs = act ? x : V - 1;
    int nb[6];
    neighbours_b(L, P, xs - x0, nb);
    int yl = -1, yr = -1;
    x_wraps_b(L, P, yl, yr);
    double acc[3][3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) acc[c][kk][0] = acc[c][kk][1] = 0.0;
    // the epilogue's operand at the own site: psi (RHS) or b (RESC)
    const double2 *epi_src = MODE == MV_RHS ? F.psi : F.b;
    cplx ev[3][3];

#pragma unroll
    for (int stg = 0; stg < kStages; ++stg) {
      const int ld = k * kLoads + stg * 2 + sp;
      const int b = ld % kBufs;
      if (stg == kStages - 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int kk = 0; kk < 3; ++kk)
            ev[c][kk] = ldg(epi_src + (int64_t)(sp * 36 + (3 * h + kk) * 6 + 2 * c + s) * V + xs);
      }
      int role = -1;
      if (!dead && !wait(&full_bar[b], (uint32_t)((ld / kBufs) & 1))) role = 0;
      if (stg == 0 && !dead && role < 0 && !wait(&dfull[k & 1], (uint32_t)((k >> 1) & 1))) role = 1;
      if (__any_sync(0xffffffffu, role >= 0) && !dead) {
        dead = true;
        if (role >= 0) record_timeout(err, 7, role, ld);
      }
      const unsigned char *bb = smem + b * kBufBytes;
      const uint32_t s_tile = smem_u32(bb), s_w = smem_u32(bb + kOffW);
      if (!dead) {
        const int ss = spin_start_b(L, P, stg);
        const int ws = blk_start_b(x0, ss, stg);
        if (stg == 0) {
          const unsigned char *dd = smem + kOffDiag + (k & 1) * kDiagStride;
          const uint32_t s_d = smem_u32(dd) + (uint32_t)(site_in_unit * 16);
          const uint32_t s_b = smem_u32(dd + kDiagD) + (uint32_t)(site_in_unit * 8);
          const uint32_t s_own = s_tile + (uint32_t)((site_in_unit + 1) * 16 + s * kTileS * 16);
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            cplx cd[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const int e = j * 3 + c;
              const double2 dv = lds_d2b(s_d + (uint32_t)(e * kUnit * 16));
              const double bv = lds_d1b(s_b + (uint32_t)(e * kUnit * 8));
              cd[c] = ad * cplx{dv.x, dv.y} + bv * am;
              if (j == c) cd[c] = cd[c] + dg;
              cd[c] = nb_sign * cd[c];
            }
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
              const double2 p = lds_d2b(s_own + (uint32_t)(((3 * h + kk) * 6 + 2 * j) * kTileS * 16));
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                acc[c][kk][0] = fma(cd[c].re, p.x, fma(-cd[c].im, p.y, acc[c][kk][0]));
                acc[c][kk][1] = fma(cd[c].re, p.y, fma(cd[c].im, p.x, acc[c][kk][1]));
              }
            }
          }
        }
#pragma unroll
        for (int hh = 0; hh < (stg == 0 ? 2 : 1); ++hh) {
          const bool bwd = stg == 0 ? (hh == 1) : (stg % 2 == 0);
          const int d = stg == 0 ? hh : stg + 1;
          const int I = d >> 1;
          const int y = nb[d];
          const int m = bwd ? y : xs;
          const bool ps = (unsigned)(y - ss) < (unsigned)kTileS;
          const bool wsh = (unsigned)(m - ws) < (unsigned)kTileS;
          const bool pw = stg == 0 && !ps && y == (bwd ? yl : yr);
          const bool ww = stg == 0 && bwd && !wsh && m == yl;
          if (stg == 0 && __any_sync(0xffffffffu, act && (pw || ww)) &&
              __all_sync(0xffffffffu, ((ps || pw) && (wsh || ww)) || !act)) {
            const uint32_t xc = smem_u32(bb + kOffX);
            const uint32_t wa = ww ? xc + kColStride : s_w + (uint32_t)((m - ws) * 16);
            const uint32_t pa = pw ? xc + (bwd ? 0u : 2u * kColStride) : s_tile + (uint32_t)((y - ss) * 16);
            const uint32_t wst = ww ? 16u : (uint32_t)kTileS * 16u, pst = pw ? 16u : (uint32_t)kTileS * 16u;
            auto lw = [&](int e) { return lds_d2b(wa + (uint32_t)e * wst); };
            auto lp = [&](int e) { return lds_d2b(pa + (uint32_t)e * pst); };
            if (bwd)
              nb_products_b<true>(acc, s, h, lw, lp);
            else
              nb_products_b<false>(acc, s, h, lw, lp);
          } else if (__all_sync(0xffffffffu, (ps && wsh) || !act)) {
            const uint32_t wa = s_w + (uint32_t)((m - ws) * 16), pa = s_tile + (uint32_t)((y - ss) * 16);
            auto lw = [&](int e) { return lds_d2b(wa + (uint32_t)(e * kTileS * 16)); };
            auto lp = [&](int e) { return lds_d2b(pa + (uint32_t)(e * kTileS * 16)); };
            if (bwd)
              nb_products_b<true>(acc, s, h, lw, lp);
            else
              nb_products_b<false>(acc, s, h, lw, lp);
          } else if (act) {
            const double2 *wp = wsh ? (const double2 *)(bb + kOffW) + (m - ws) : Wf + (int64_t)((I * 2 + sp) * 36) * V + m;
            const double2 *pp = ps ? (const double2 *)bb + (y - ss) : in + (int64_t)(sp * 36) * V + y;
            const int64_t wst = wsh ? kTileS : V, pst = ps ? kTileS : V;
            auto lw = [&](int e) { return wp[e * wst]; };
            auto lp = [&](int e) { return pp[e * pst]; };
            if (bwd)
              nb_products_b<true>(acc, s, h, lw, lp);
            else
              nb_products_b<false>(acc, s, h, lw, lp);
          }
        }
      }
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&empty_bar[b]);
        if (stg == 0) mbar_arrive(&dempty[k & 1]);
      }
    }

    // ---------------------------------------------------------- epilogue
    double q[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    if (!dead && act) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
          const int64_t off = (int64_t)(sp * 36 + (3 * h + kk) * 6 + 2 * c + s) * V + x;
          const cplx y_ = {nb_sign * acc[c][kk][0], nb_sign * acc[c][kk][1]};
          if (MODE == MV_RHS) {
            st(F.b + off, y_);
            st(F.x + off, 2.0 * y_ - ev[c][kk]);
          } else {
            const cplx rv = ev[c][kk] - y_;
            const cplx dv = rv * F.inv_theta[sp];
            F.r32[off] = make_float2((float)rv.re, (float)rv.im);
            F.dA[off] = make_float2((float)dv.re, (float)dv.im);
            q[kk][0] += norm2(rv);
            q[kk][1] += norm2(ev[c][kk]);
          }
        }
    }
    if (MODE == MV_RESC) {
      // the unit's partial row: each column over the lanes, then over the
      // two spin warps (spin 1 hands its sums to spin 0 through red[])
#pragma unroll
      for (int kk = 0; kk < 3; ++kk)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) q[kk][j] += __shfl_xor_sync(0xffffffffu, q[kk][j], o);
      if (s == 1 && lane == 0)
#pragma unroll
        for (int kk = 0; kk < 3; ++kk)
#pragma unroll
          for (int j = 0; j < 2; ++j) red[k & 1][sp][h][kk][j] = q[kk][j];
      named_bar_sync(pair_bar, 64);
      if (s == 0 && lane < 6 && !dead) {
        const int kk = lane >> 1, j = lane & 1;
        const int col12 = sp * 6 + 3 * h + kk;
        double v = 0.0;
#pragma unroll
        for (int t = 0; t < 6; ++t)
          if (t == lane) v = q[t >> 1][t & 1];
        F.partials[((int64_t)u * CN_COLS + col12) * 2 + j] = v + red[k & 1][sp][h][kk][j];
      }
    }
    ++k;
  }
}

// ------------------------------------------------------------------ host
bool batch_mv5_applicable(const Lat &L) { return L.V >= bm5::kTileS && L.V <= 0x7fffffffLL && (L.V & 1) == 0; }

bool batch_mv5_field_maps(CnBatchMaps *m, const Lat &L, const double2 *psi, const double2 *x) {
  using namespace bm5;
  const uint64_t V = (uint64_t)L.V;
  memset(m, 0, sizeof(*m));
  const double2 *src[2] = {psi, x};
  for (int k = 0; k < 2; ++k)
    if (!stage::encode(&m->in[k].spin, src[k], 2 * V, 72, 2 * kTileS, 36) ||
        !stage::encode(&m->in[k].spin1, src[k], 2 * V, 72, 2, 36))
      return false;
  return true;
}

int launch_batch_mv5(int mode, int order, Lat L, const double2 *W, int nblk, const double2 *Dsum, const double *Bsum,
                     const CnBatchMaps *fmaps, const BatchField *tab, int nfields, int skip_done, int *err,
                     int sm_count, cudaStream_t st, long long wait_cycles) {
  using namespace bm5;
  if (!batch_mv5_applicable(L) || nfields <= 0 || order < 0 || order > 1 || (mode != MV_RHS && mode != MV_RESC))
    return -1;
  const int64_t nunits = (L.V + kUnit - 1) / kUnit;
  if (nunits * nfields > 0x7fffffffLL) return -1;
  const uint64_t V = (uint64_t)L.V;
  BatchMv5Maps maps;
  memset(&maps, 0, sizeof(maps));
  if (!stage::encode(&maps.W, W, 2 * V, 216ull * nblk, 2 * kTileS, 36) ||
      !stage::encode(&maps.W1, W, 2 * V, 216ull * nblk, 2, 36) || !stage::encode(&maps.D, Dsum, 2 * V, 9, 2 * kUnit, 9) ||
      !stage::encode(&maps.B, Bsum, V, 9, kUnit, 9))
    return -1;
  const unsigned grid = (unsigned)std::min<int64_t>(nunits * nfields, sm_count);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    kern<<<grid, kThreads, kSmemBytes, st>>>(L, maps, fmaps, W, tab, nfields, (int)nunits, order, skip_done, err,
                                            wait_cycles);
  };
  if (mode == MV_RHS)
    go(k_batch_mv5<MV_RHS>);
  else
    go(k_batch_mv5<MV_RESC>);
  return 0;
}

}  // namespace nrq
