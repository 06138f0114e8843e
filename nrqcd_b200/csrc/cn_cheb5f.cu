// FP32 Chebyshev step of the precision forms on cached FP32 blocks:
//   t = A^H d (all 12 columns), then per site and row
//   r <- r - t ; e <- e + d (first step: e = d) ; d' = c1 d + c2 r
// (c1, c2 per species), the step of k_cheb32 (cn_f32.cu) with the operator
// applied as the FP64 FMA stencil applies it (cn_mv5.cu): the forward 6x6
// spin-colour block W_I(x) of every site, direction and species, written by
// k_cn_blocks5 rounded to FP32 (216 planes of V complex, plane (I*2 +
// species)*36 + row*6 + column); the backward block is -W_I(x-I)^H; the
// diagonal from the FP32 copies of the plaquette sums (Dsum, Bsum).
//
// Products.  A thread owns a 3 x 3 tile of one site and species: the three
// output rows of one spin (the three colours) and three of the six columns.
// Per neighbour and input row it reads 3 block entries and 3 spinor entries
// (8-byte shared-memory loads, two wavefronts per warp) and does 36 FP32
// FMAs.  The FP32 pipe has twice the FP64 rate and every load half the
// bytes, so the products take well under the time the blocks and spinors
// need to arrive from HBM: the kernel is bound by its loads.
//
// Pipeline.  Persistent, one CTA per SM: 8 consumer warps (species 0 in
// warps 0-3, species 1 in 4-7; a warp holds one spin and column half of a
// 32-site unit) and one producer warp.  Ten loads per unit, per stage and
// species (stage 0: diagonal matrices, +x and -x; 1: +y; 2: -y; 3: +z; 4:
// -z): a spinor tile and a block tile of 36 sites x 36 planes by TMA, into a
// ring of eight buffers completed on mbarriers.  A TMA copy of FP32 planes
// starts on a 16-byte boundary, i.e. an even site: the stage-0 tiles span
// x0 - 2 .. x0 + 33, the others start at the neighbouring row (nx even), and
// the periodic x neighbours that wrap outside a unit's tile come as two-site
// columns from the even site at or below them.  A lane whose neighbour or
// block lies anywhere else outside the tiles reads it from global memory.
// The epilogue's operands at the own site (d, r, e) are loaded into
// registers two stages ahead.
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

namespace c5f {
constexpr int kUnit = 32;                  // sites per work unit (one per lane)
constexpr int kWarps = 8;                  // consumer warps: (species, spin, column half)
constexpr int kThreads = (kWarps + 1) * 32;
constexpr int kStages = 5;                 // stages per unit
constexpr int kLoads = 2 * kStages;        // loads per unit: (stage, species); load i is of species i & 1
// Ring of load buffers; an even ring gives every buffer the loads of one
// species only, whose warps released the previous use themselves, so a
// consumer never waits on a full barrier more than one phase ahead.
constexpr int kBufs = 8;
constexpr int kTileS = kUnit + 4;          // tile width in sites: x0 - 2 .. x0 + 33
constexpr uint32_t kTileBytes = 36u * kTileS * 8u;     // 10368: 36 planes x 36 sites
constexpr uint32_t kOffW = kTileBytes;                 // block tile (36 entry planes)
// stage 0 only: the x-wrap columns, 36 planes x two sites (16 B) each (the
// spinor and the block at the -x neighbour of the unit's x = 0 site, the
// spinor at the +x neighbour of its x = nx - 1 site)
constexpr uint32_t kOffX = 2u * kTileBytes;            // 20736
constexpr uint32_t kColBytes = 36u * 16u;              // 576
constexpr uint32_t kColStride = 640u;                  // 128-byte aligned column starts
constexpr uint32_t kBufBytes = ((kOffX + 3u * kColStride) + 1023u) & ~1023u;  // 23552
// the unit's diagonal matrices, double-buffered by unit after the ring:
// D (9 planes x 32 sites x 8 B), then B (9 planes x 32 sites x 4 B)
constexpr uint32_t kDiagD = 9u * kUnit * 8u;           // 2304
constexpr uint32_t kDiagB = 9u * kUnit * 4u;           // 1152
constexpr uint32_t kDiagStride = 3584u;
constexpr uint32_t kOffDiag = kBufs * kBufBytes;       // 188416
constexpr uint32_t kSmemBytes = kOffDiag + 2u * kDiagStride + 1024u;  // 196608
static_assert(kOffW % 128 == 0 && kOffX % 128 == 0 && kColStride % 128 == 0 && kColStride >= kColBytes &&
                  kBufBytes % 1024 == 0 && kDiagStride % 128 == 0 && kDiagD % 128 == 0 &&
                  kDiagD + kDiagB <= kDiagStride,
              "layout");
static_assert(kSmemBytes + 1024 <= 232448, "shared memory");
static_assert(kBufs % 2 == 0 && kLoads % 2 == 0, "a buffer's uses must all belong to one species");
}  // namespace c5f

struct Cheb5fMaps {
  CUtensorMap spin;   // 72 planes x 2V floats, box {72, 36}
  CUtensorMap W;      // 216 planes x 2V floats, box {72, 36}
  CUtensorMap spin1;  // the same planes, two sites: box {4, 36}
  CUtensorMap W1;
  CUtensorMap D;      // 9 planes x 2V floats, box {64, 9}
  CUtensorMap B;      // 9 planes x V floats, box {32, 9}
};

namespace {

struct cfl {
  float re, im;
};

struct UnitPos5f {
  int x0, cx, cy, cz;
};
__device__ __forceinline__ UnitPos5f unit_pos5f(const Lat &L, int x0) {
  const int nx = (int)L.nx, ny = (int)L.ny;
  const int t = x0 / nx, z = t / ny;
  return {x0, x0 - t * nx, t - z * ny, z};
}

// Position of work unit u: in blocks of 8 x 8 rows where the lattice allows
// (nx a multiple of 32, ny and nz of 8), so that neighbouring units' +-y and
// +-z tiles come from L2, as in the FP64 FMA stencil (cn_mv5.cu); otherwise
// in site order.
__device__ __forceinline__ UnitPos5f unit_pos5f_of(const Lat &L, int u) {
  const int nx = (int)L.nx, ny = (int)L.ny, nz = (int)L.nz;
  if ((nx & 31) || (ny & 7) || (nz & 7)) return unit_pos5f(L, u * c5f::kUnit);
  const int nxu = nx >> 5;
  int t = u / nxu;
  const int cx = (u - t * nxu) << 5;
  const int yi = t & 7, zi = (t >> 3) & 7;
  t >>= 6;
  const int nby = ny >> 3;
  const int bz = t / nby, by = t - bz * nby;
  const int cy = (by << 3) + yi, cz = (bz << 3) + zi;
  return {cx + nx * (cy + ny * cz), cx, cy, cz};
}

// the six periodic neighbours (+x,-x,+y,-y,+z,-z) of the site l sites after
// the unit's first (V < 2^31), its coordinates by carrying from the unit's
__device__ __forceinline__ void neighbours5f(const Lat &L, const UnitPos5f &P, int l, int (&nb)[6]) {
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

// first site of the spinor tile of stage stg (stage 0: x0 - 2; stages 1-4:
// the +y, -y, +z, -z neighbours of x0, even for even nx)
__device__ __forceinline__ int spin_start5f(const Lat &L, const UnitPos5f &P, int stg) {
  const int x0 = P.x0;
  if (stg == 0) return x0 - 2;
  const int ny = (int)L.ny, nz = (int)L.nz;
  const int row = (int)L.nx, plane = (int)(L.nx * L.ny);
  switch (stg) {
    case 1: return P.cy + 1 < ny ? x0 + row : x0 - (ny - 1) * row;
    case 2: return P.cy > 0 ? x0 - row : x0 + (ny - 1) * row;
    case 3: return P.cz + 1 < nz ? x0 + plane : x0 - (nz - 1) * plane;
    default: return P.cz > 0 ? x0 - plane : x0 + (nz - 1) * plane;
  }
}
// first site of the block tile: forward stages read the unit's own blocks,
// backward stages the neighbours', stage 0 both (the spinor tile's sites)
__device__ __forceinline__ int blk_start5f(int x0, int spin_start, int stg) {
  if (stg == 1 || stg == 3) return x0;
  return spin_start;
}

// Sites of the unit whose x neighbour wraps outside the stage-0 tile (rows
// of at least kTileS sites): yl = the -x neighbour of its x = 0 site, yr =
// the +x neighbour of its x = nx - 1 site; -1 where the unit has none.
__device__ __forceinline__ void x_wraps5f(const Lat &L, const UnitPos5f &P, int &yl, int &yr) {
  const int nx = (int)L.nx, V = (int)L.V, x0 = P.x0;
  yl = yr = -1;
  if (nx < c5f::kTileS) return;
  const int pl = P.cx == 0 ? 0 : nx - P.cx, pr = nx - 1 - P.cx;
  if (pl < c5f::kUnit && x0 + pl < V) yl = x0 + pl + nx - 1;
  if (pr < c5f::kUnit && x0 + pr < V) yr = x0 + pr - (nx - 1);
}

__device__ __forceinline__ float2 lds_f2(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ float lds_f1(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}

// The thread's tile (rows 2c + s, c = 0..2; columns 3h + k) += sum over q
// of w[c][q] psi[q][3h + k].  Forward: w[c][q] = W(x)[2c+s][q], entry
// (2c+s)*6 + q; backward: w[c][q] = -conj(W(y)[q][2c+s]), entry q*6 + 2c + s.
// load_w(e) reads entry e of the block, load_p(e) plane e of the spinor.
template <bool BWD, typename LW, typename LP>
__device__ __forceinline__ void nb_products5f(float (&acc)[3][3][2], int s, int h, LW load_w, LP load_p) {
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    float wr[3], wi[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float2 wv = load_w(BWD ? q * 6 + 2 * c + s : (2 * c + s) * 6 + q);
      wr[c] = BWD ? -wv.x : wv.x;
      wi[c] = wv.y;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float2 p = load_p((3 * h + k) * 6 + q);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc[c][k][0] = fmaf(wr[c], p.x, fmaf(-wi[c], p.y, acc[c][k][0]));
        acc[c][k][1] = fmaf(wr[c], p.y, fmaf(wi[c], p.x, acc[c][k][1]));
      }
    }
  }
}

__device__ __forceinline__ cfl cmulf(cfl a, cfl b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

}  // namespace

// Arguments of one launch: a single field (tab == nullptr: d, r, e, the
// operator's coefficients C and this step's Chebyshev coefficients K), or a
// batch (the device table: per field its vectors, its coefficients at its
// mass, this step's Chebyshev coefficients and its block set wblk).
struct Cheb5fArgs {
  CnCoef C;
  ChebCoef K;
  const float2 *Din;
  float2 *Dn, *R, *E;
  const BatchField *tab;
  int step, order;
  const float2 *Wf;
  float nb_sign;
  int nunits, nfields, nwork;
  int *err;
  long long wait_cycles;
};

// work item w of a launch: (field, unit); a batch orders the items field
// fastest (order 0) or unit fastest (order 1)
template <bool BATCH>
__device__ __forceinline__ void cheb5f_item(const Cheb5fArgs &A, int w, int &f, int &u) {
  if (!BATCH) {
    f = 0;
    u = w;
  } else if (A.order == 0) {
    f = w % A.nfields;
    u = w / A.nfields;
  } else {
    f = w / A.nunits;
    u = w % A.nunits;
  }
}
// a batch field that converged at its last residual check sits the step out
// (the same answer for every thread of the launch)
template <bool BATCH>
__device__ __forceinline__ bool cheb5f_skip(const Cheb5fArgs &A, int f) {
  return BATCH && batch_field_done(A.tab[f]);
}

template <bool FIRST, bool BATCH>
__global__ void __launch_bounds__(c5f::kThreads, 1)
    k_cheb5f(Lat L, const __grid_constant__ Cheb5fArgs A, const __grid_constant__ Cheb5fMaps maps) {
  using namespace c5f;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kBufs], empty_bar[kBufs], dfull[2], dempty[2];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int V = (int)L.V;  // the launcher admits V < 2^31 only
  int *err = A.err;
  const long long wait_cycles = A.wait_cycles;

  if (threadIdx.x == 0) {
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(&full_bar[b], 1);
      mbar_init(&empty_bar[b], 4);  // the four consumer warps of the load's species
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], 1);
      mbar_init(&dempty[b], kWarps);  // every consumer warp
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

  // ---------------------------------------------------------- producer
  if (warp == kWarps) {
    if (lane == 0) {
      bool ok = true;
      int i = 0, k = 0;  // loads issued, items begun
      for (int w = blockIdx.x; w < A.nwork && ok; w += gridDim.x) {
        int f, u;
        cheb5f_item<BATCH>(A, w, f, u);
        if (cheb5f_skip<BATCH>(A, f)) continue;
        const UnitPos5f P = unit_pos5f_of(L, u);
        const int x0 = P.x0;
        const int srow = BATCH ? f * 72 : 0;                   // the field's planes
        const int wrow = BATCH ? A.tab[f].wblk * 216 : 0;      // its block set
        {  // the unit's diagonal matrices, with its first load
          const int db = k & 1;
          if (k >= 2) {
            const uint32_t dpar = (uint32_t)((k / 2 - 1) & 1);
            if (!wait(&dempty[db], dpar)) {
              record_timeout(err, 6, 2, i);
              ok = false;
            } else if (!mbar_wait(&dfull[db], dpar)) {
              record_timeout(err, 6, 3, i);
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
            // every consumer warp of the species released the buffer, and
            // its previous load landed
            if (!wait(&empty_bar[b], par)) {
              record_timeout(err, 6, 2, i);
              ok = false;
            } else if (!mbar_wait(&full_bar[b], par)) {
              record_timeout(err, 6, 3, i);
              ok = false;
            }
            if (!ok) break;
          }
          const int stg = li >> 1, sp = li & 1;
          const int ss = spin_start5f(L, P, stg);
          const int ws = blk_start5f(x0, ss, stg);
          const int I = stg == 0 ? 0 : (stg + 1) / 2;
          unsigned char *bb = smem + b * kBufBytes;
          int yl = -1, yr = -1;
          if (stg == 0) x_wraps5f(L, P, yl, yr);
          uint32_t tx = 2u * kTileBytes;
          if (stg == 0) tx += (yl >= 0 ? 2u : 0u) * kColBytes + (yr >= 0 ? kColBytes : 0u);
          mbar_expect_tx(&full_bar[b], tx);
          tma_2d(bb, &maps.spin, 2 * ss, srow + sp * 36, &full_bar[b]);
          tma_2d(bb + kOffW, &maps.W, 2 * ws, wrow + (I * 2 + sp) * 36, &full_bar[b]);
          if (stg == 0) {  // two-site columns from the even site at or below
            if (yl >= 0) {
              tma_2d(bb + kOffX, &maps.spin1, 2 * (yl & ~1), srow + sp * 36, &full_bar[b]);
              tma_2d(bb + kOffX + kColStride, &maps.W1, 2 * (yl & ~1), wrow + sp * 36, &full_bar[b]);
            }
            if (yr >= 0)
              tma_2d(bb + kOffX + 2 * kColStride, &maps.spin1, 2 * (yr & ~1), srow + sp * 36, &full_bar[b]);
          }
        }
        ++k;
      }
      // every issued load lands before the CTA exits
      for (int j = max(0, i - kBufs); j < i; ++j)
        if (!mbar_wait(&full_bar[j % kBufs], (uint32_t)((j / kBufs) & 1))) {
          record_timeout(err, 6, 4, j);
          break;
        }
      for (int j = max(0, k - 2); j < k; ++j)
        if (!mbar_wait(&dfull[j & 1], (uint32_t)((j >> 1) & 1))) {
          record_timeout(err, 6, 4, -1 - j);
          break;
        }
    }
    return;
  }

  // ---------------------------------------------------------- consumers
  // warp w = 4 sp + 2 s + h: species sp, spin s, column half h; lane = site
  // of the 32-site unit.  The thread owns rows 2c + s (c = 0..2) and columns
  // 3h .. 3h + 2 of its site and species.
  const int sp = warp >> 2, s = (warp >> 1) & 1, h = warp & 1;
  const int site_in_unit = lane;
  const float nb_sign = A.nb_sign;
  bool dead = false;

  int k = 0;  // items begun
  for (int w = blockIdx.x; w < A.nwork; w += gridDim.x) {
    int f, u;
    cheb5f_item<BATCH>(A, w, f, u);
    if (cheb5f_skip<BATCH>(A, f)) continue;
    // the item's field: vectors and coefficients
    const CnCoef &C = BATCH ? A.tab[f].CH : A.C;
    const ChebCoef &K = BATCH ? A.tab[f].cheb[A.step] : A.K;
    const float2 *Din = BATCH ? ((A.step & 1) ? A.tab[f].dB : A.tab[f].dA) : A.Din;
    float2 *Dn = BATCH ? ((A.step & 1) ? A.tab[f].dA : A.tab[f].dB) : A.Dn;
    float2 *R = BATCH ? A.tab[f].r32 : A.R;
    float2 *E = BATCH ? A.tab[f].e32 : A.E;
    const float2 *Wf = A.Wf + (BATCH ? (int64_t)A.tab[f].wblk * 216 * V : 0);
    const cfl ak = {(float)C.kin[sp].re, (float)C.kin[sp].im};
    const cfl am = {(float)C.mag[sp].re, (float)C.mag[sp].im}, ad = {(float)C.dar[sp].re, (float)C.dar[sp].im};
    const cfl dg = {(float)C.dkin * ak.re + 1.f, (float)C.dkin * ak.im};
    const cfl c1 = {(float)K.c1[sp].re, (float)K.c1[sp].im}, c2 = {(float)K.c2[sp].re, (float)K.c2[sp].im};

    const UnitPos5f P = unit_pos5f_of(L, u);
    const int x0 = P.x0;
    const int x = x0 + site_in_unit;
    const bool act = x < V;
    const int xs = act ? x : V - 1;  // a valid site for the addresses of idle lanes
    int nb[6];
    neighbours5f(L, P, xs - x0, nb);
    int yl = -1, yr = -1;
    x_wraps5f(L, P, yl, yr);
    float acc[3][3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) acc[c][kk][0] = acc[c][kk][1] = 0.f;
    float2 ed[3][3], er[3][3], ee[3][3];

#pragma unroll
    for (int stg = 0; stg < kStages; ++stg) {
      const int ld = k * kLoads + stg * 2 + sp;
      const int b = ld % kBufs;
      if (stg == kStages - 2) {
        // the epilogue's operands, loaded into registers two stages ahead
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int kk = 0; kk < 3; ++kk) {
            const int64_t off = (int64_t)(sp * 36 + (3 * h + kk) * 6 + 2 * c + s) * V + xs;
            ed[c][kk] = __ldg(Din + off);
            er[c][kk] = R[off];
            if (!FIRST) ee[c][kk] = E[off];
          }
      }
      int role = -1;
      if (!dead && !wait(&full_bar[b], (uint32_t)((ld / kBufs) & 1))) role = 0;
      // stage 0 also reads the unit's diagonal matrices
      if (stg == 0 && !dead && role < 0 && !wait(&dfull[k & 1], (uint32_t)((k >> 1) & 1))) role = 1;
      // warp-uniform: the products below use warp votes
      if (__any_sync(0xffffffffu, role >= 0) && !dead) {
        dead = true;
        if (role >= 0) record_timeout(err, 6, role, ld);
      }
      const unsigned char *bb = smem + b * kBufBytes;
      const uint32_t s_tile = smem_u32(bb), s_w = smem_u32(bb + kOffW);
      if (!dead) {
        const int ss = spin_start5f(L, P, stg);
        const int ws = blk_start5f(x0, ss, stg);
        if (stg == 0) {
          // diagonal (colour only): row (c, s) takes input rows (j, s);
          // x - ss = site_in_unit + 2 lies inside the tile for every lane
          const unsigned char *dd = smem + kOffDiag + (k & 1) * kDiagStride;
          const uint32_t s_d = smem_u32(dd) + (uint32_t)(site_in_unit * 8);
          const uint32_t s_b = smem_u32(dd + kDiagD) + (uint32_t)(site_in_unit * 4);
          const uint32_t s_own = s_tile + (uint32_t)((site_in_unit + 2) * 8 + s * kTileS * 8);
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            cfl cd[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const int e = j * 3 + c;
              const float2 dv = lds_f2(s_d + (uint32_t)(e * kUnit * 8));
              const float bv = lds_f1(s_b + (uint32_t)(e * kUnit * 4));
              cd[c] = cmulf(ad, cfl{dv.x, dv.y});
              cd[c].re += bv * am.re;
              cd[c].im += bv * am.im;
              if (j == c) {
                cd[c].re += dg.re;
                cd[c].im += dg.im;
              }
              cd[c].re *= nb_sign;  // see the epilogue
              cd[c].im *= nb_sign;
            }
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
              const float2 p = lds_f2(s_own + (uint32_t)(((3 * h + kk) * 6 + 2 * j) * kTileS * 8));
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                acc[c][kk][0] = fmaf(cd[c].re, p.x, fmaf(-cd[c].im, p.y, acc[c][kk][0]));
                acc[c][kk][1] = fmaf(cd[c].re, p.y, fmaf(cd[c].im, p.x, acc[c][kk][1]));
              }
            }
          }
        }
        // neighbours of this stage: stage 0 = +x (forward) and -x (backward)
#pragma unroll
        for (int hh = 0; hh < (stg == 0 ? 2 : 1); ++hh) {
          const bool bwd = stg == 0 ? (hh == 1) : (stg % 2 == 0);
          const int d = stg == 0 ? hh : stg + 1;  // neighbour index in nb[]
          const int I = d >> 1;
          const int y = nb[d];                   // neighbour site
          const int m = bwd ? y : xs;            // site of the forward block
          const bool ps = (unsigned)(y - ss) < (unsigned)kTileS;  // spinor in the tile
          const bool wsh = (unsigned)(m - ws) < (unsigned)kTileS; // block in the tile
          // stage 0: a wrapped x neighbour in the wrap columns
          const bool pw = stg == 0 && !ps && y == (bwd ? yl : yr);
          const bool ww = stg == 0 && bwd && !wsh && m == yl;
          if (stg == 0 && __any_sync(0xffffffffu, act && (pw || ww)) &&
              __all_sync(0xffffffffu, ((ps || pw) && (wsh || ww)) || !act)) {
            // shared memory, a lane's operands in the tile or in a wrap
            // column (per-lane strides; a column holds two sites per plane)
            const uint32_t xc = smem_u32(bb + kOffX);
            const uint32_t wa = ww ? xc + kColStride + (uint32_t)((m & 1) * 8) : s_w + (uint32_t)((m - ws) * 8);
            const uint32_t pa = pw ? xc + (bwd ? 0u : 2u * kColStride) + (uint32_t)((y & 1) * 8)
                                   : s_tile + (uint32_t)((y - ss) * 8);
            const uint32_t wst = ww ? 16u : (uint32_t)kTileS * 8u, pst = pw ? 16u : (uint32_t)kTileS * 8u;
            auto lw = [&](int e) { return lds_f2(wa + (uint32_t)e * wst); };
            auto lp = [&](int e) { return lds_f2(pa + (uint32_t)e * pst); };
            if (bwd)
              nb_products5f<true>(acc, s, h, lw, lp);
            else
              nb_products5f<false>(acc, s, h, lw, lp);
          } else if (__all_sync(0xffffffffu, (ps && wsh) || !act)) {
            // every operand of the warp in shared memory
            const uint32_t wa = s_w + (uint32_t)((m - ws) * 8), pa = s_tile + (uint32_t)((y - ss) * 8);
            auto lw = [&](int e) { return lds_f2(wa + (uint32_t)(e * kTileS * 8)); };
            auto lp = [&](int e) { return lds_f2(pa + (uint32_t)(e * kTileS * 8)); };
            if (bwd)
              nb_products5f<true>(acc, s, h, lw, lp);
            else
              nb_products5f<false>(acc, s, h, lw, lp);
          } else if (act) {
            // some lanes' operands outside the tiles (periodic wraps, tile
            // edges): those lanes read global memory, the others the tiles
            const float2 *wp = wsh ? (const float2 *)(bb + kOffW) + (m - ws) : Wf + (int64_t)((I * 2 + sp) * 36) * V + m;
            const float2 *pp = ps ? (const float2 *)bb + (y - ss) : Din + (int64_t)(sp * 36) * V + y;
            const int64_t wst = wsh ? kTileS : V, pst = ps ? kTileS : V;
            auto lw = [&](int e) { return wp[e * wst]; };
            auto lp = [&](int e) { return pp[e * pst]; };
            if (bwd)
              nb_products5f<true>(acc, s, h, lw, lp);
            else
              nb_products5f<false>(acc, s, h, lw, lp);
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
    if (!dead && act) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
          const int64_t off = (int64_t)(sp * 36 + (3 * h + kk) * 6 + 2 * c + s) * V + x;
          // D in + sgn N in = sgn (sgn D in + N in), sgn = +-1: the diagonal
          // was scaled by sgn and the neighbour sum was not
          const float tr = nb_sign * acc[c][kk][0], ti = nb_sign * acc[c][kk][1];
          const float2 dv = ed[c][kk];
          const float2 r = make_float2(er[c][kk].x - tr, er[c][kk].y - ti);
          R[off] = r;
          E[off] = FIRST ? dv : make_float2(ee[c][kk].x + dv.x, ee[c][kk].y + dv.y);
          const cfl a = cmulf(c1, cfl{dv.x, dv.y}), bq = cmulf(c2, cfl{r.x, r.y});
          Dn[off] = make_float2(a.re + bq.re, a.im + bq.im);
        }
    }
    ++k;
  }
}

// ------------------------------------------------------------------ host
bool cheb5f_applicable(const Lat &L) {
  return L.V >= c5f::kTileS && L.V <= 0x7fffffffLL && (L.V % 4) == 0 && (L.nx % 2) == 0;
}

namespace {
// tensor maps of a launch: the d vectors of nfields fields (72 planes each)
// and nblk block sets (216 planes each)
bool cheb5f_maps(Cheb5fMaps &maps, const Lat &L, const float2 *D, int nfields, const float2 *Wf, int nblk,
                 const float2 *Dsum, const float *Bsum) {
  using namespace c5f;
  const uint64_t V = (uint64_t)L.V;
  constexpr CUtensorMapDataType F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  constexpr CUtensorMapSwizzle NS = CU_TENSOR_MAP_SWIZZLE_NONE;
  memset(&maps, 0, sizeof(maps));
  return stage::encode(&maps.spin, D, 2 * V, 72ull * nfields, 2 * kTileS, 36, NS, F32) &&
         stage::encode(&maps.W, Wf, 2 * V, 216ull * nblk, 2 * kTileS, 36, NS, F32) &&
         stage::encode(&maps.spin1, D, 2 * V, 72ull * nfields, 4, 36, NS, F32) &&
         stage::encode(&maps.W1, Wf, 2 * V, 216ull * nblk, 4, 36, NS, F32) &&
         stage::encode(&maps.D, Dsum, 2 * V, 9, 2 * kUnit, 9, NS, F32) &&
         stage::encode(&maps.B, Bsum, V, 9, kUnit, 9, NS, F32);
}
template <bool BATCH>
void cheb5f_go(bool first, const Lat &L, const Cheb5fArgs &a, const Cheb5fMaps &maps, int sm_count,
               cudaStream_t st) {
  using namespace c5f;
  const unsigned grid = (unsigned)std::min<int64_t>(a.nwork, sm_count);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    kern<<<grid, kThreads, kSmemBytes, st>>>(L, a, maps);
  };
  if (first)
    go(k_cheb5f<true, BATCH>);
  else
    go(k_cheb5f<false, BATCH>);
}
}  // namespace

int launch_cheb5f(bool first, Lat L, const CnCoef &C, double nb_sign, const float2 *Wf, const float2 *Dsum,
                  const float *Bsum, const float2 *D, float2 *Dn, float2 *R, float2 *E, const ChebCoef &K, int *err,
                  int sm_count, cudaStream_t st, long long wait_cycles) {
  using namespace c5f;
  if (!cheb5f_applicable(L)) return -1;
  Cheb5fMaps maps;
  if (!cheb5f_maps(maps, L, D, 1, Wf, 1, Dsum, Bsum)) return -1;
  Cheb5fArgs a{};
  a.C = C;
  a.K = K;
  a.Din = D;
  a.Dn = Dn;
  a.R = R;
  a.E = E;
  a.Wf = Wf;
  a.nb_sign = (float)nb_sign;
  a.nunits = (int)((L.V + kUnit - 1) / kUnit);
  a.nfields = 1;
  a.nwork = a.nunits;
  a.err = err;
  a.wait_cycles = wait_cycles;
  cheb5f_go<false>(first, L, a, maps, sm_count, st);
  return 0;
}

int launch_batch_cheb5f(int step, int order, Lat L, const float2 *Wf, int nblk, const float2 *Dsum,
                        const float *Bsum, const float2 *dA_all, const float2 *dB_all, const BatchField *tab,
                        int nfields, int *err, int sm_count, cudaStream_t st, long long wait_cycles) {
  using namespace c5f;
  if (!cheb5f_applicable(L) || step < 0 || step >= BATCH_MAX_CHEB || nfields <= 0 || order < 0 || order > 1)
    return -1;
  const int64_t nunits = (L.V + kUnit - 1) / kUnit;
  if (nunits * nfields > 0x7fffffffLL) return -1;
  Cheb5fMaps maps;
  if (!cheb5f_maps(maps, L, (step & 1) ? dB_all : dA_all, nfields, Wf, nblk, Dsum, Bsum)) return -1;
  Cheb5fArgs a{};
  a.tab = tab;
  a.step = step;
  a.order = order;
  a.Wf = Wf;
  a.nb_sign = 1.f;
  a.nunits = (int)nunits;
  a.nfields = nfields;
  a.nwork = (int)(nunits * nfields);
  a.err = err;
  a.wait_cycles = wait_cycles;
  cheb5f_go<true>(step == 0, L, a, maps, sm_count, st);
  return 0;
}

}  // namespace nrq
