// FP64 FMA stencil of the assembled Crank-Nicolson operator on cached 6x6
// blocks (src/nrqcd.f90:1175-1387 with PETSc's block transposition; the
// operator is described in cn.cu): out = D in + sum over the 6 neighbours of
// the spin-colour blocks applied to the 6 propagator columns, both species.
//
// Blocks.  Once per update, k_cn_blocks5 writes the forward block of every
// site, direction and species with the operator's coefficients folded in
// (the blocks of the tensor-core stencil, cn_mv4.cu) as 216 planes of V
// complex: plane (I*2 + species)*36 + row*6 + column.  With real Wilson
// coefficients the backward block is -W_I(x-I)^H, read from the forward
// block of x-I, and A^H differs from A by the sign of the neighbour sum.
//
// Products.  A thread owns a 3 x 3 tile of one site and species: the three
// output rows of one spin (the three colours) and three of the six columns,
// 18 doubles in registers.  Per neighbour and input row q it reads 3 block
// entries and 3 spinor entries from shared memory and does 36 FP64 FMAs,
// none of them padding.  On B200 the FP64 FMA pipe and the FP64 tensor pipe
// have the same peak, and the tensor pipe's 16x8 tiles hold 12 x 6 useful
// entries.  A 16-byte shared-memory load costs four wavefronts per warp
// whether or not lanes share addresses, so every warp holds 32 consecutive
// sites of one (species, spin, column half): each load then delivers 512
// distinct bytes without bank conflicts, and the tile size sets the traffic.
//
// Pipeline.  Persistent, one CTA per SM: 8 consumer warps (species 0 in
// warps 0-3, species 1 in 4-7; a warp holds one spin and column half of a
// 32-site unit) and one producer warp.  Ten loads per unit, per stage and species
// (stage 0: diagonal matrices, +x and -x; 1: +y; 2: -y; 3: +z; 4: -z): a
// spinor tile (34 sites x 36 planes) and a block tile (34 sites x 36 entry
// planes) by TMA, into a ring of four shared-memory buffers completed on
// mbarriers; the unit's diagonal matrices go with its first load into one
// of two further buffers.  The producer refills a buffer once the four consumer warps of
// its species released it and its previous load has landed.  The periodic
// x neighbours that wrap outside a unit's tile (one site at each row end)
// arrive as two extra one-site spinor columns and one block column with
// stage 0; a lane whose neighbour or block lies anywhere else outside the
// tiles (rows shorter than the tile) reads it from global memory.  Results go straight to global
// memory; the epilogue's operand at the own site is prefetched into L1 two
// stages before the epilogue reads it; the residual and dot-product
// partial sums stay in registers over all units of the CTA (one partial row
// per CTA).
//
// Every mbarrier wait is bounded (wait_cycles); on expiry the thread records
// NRQ_ERR_TIMEOUT in *err and skips the remaining work.  The producer never
// has two loads in flight into one buffer and, before it exits, waits
// (bounded) until every load it issued has landed.  stall_load >= 0 makes
// the producer stop before that load, so that the consumers' wait for it
// runs out: the host's test of the timeout path (nothing faults; the
// context stays usable).  Single-GPU code: no load uses cluster multicast.
#include <algorithm>
#include <cstring>

#include "../../include/nrqcd_b200.h"
#include "nrq_kernels.cuh"
#include "stage.cuh"

namespace nrq {

namespace mv5 {
constexpr int kUnit = 32;                 // sites per work unit (one per lane)
constexpr int kWarps = 8;                 // consumer warps: (species, spin, column half)
constexpr int kThreads = (kWarps + 1) * 32;
constexpr int kMaxReg = 168;              // three warps on one SM quarter: 3 x 32 x 168 <= 16384
constexpr int kStages = 5;                // stages per unit
constexpr int kLoads = 2 * kStages;       // loads per unit: (stage, species)
// Ring of load buffers.  Loads alternate between the species, and a
// consumer waits on a buffer's full barrier by phase parity, which is only
// sound while it never waits more than one phase ahead of the barrier's
// last completed phase.  With an even ring every use of a buffer belongs to
// one species, whose warps released the previous use themselves; an odd
// ring would let one species wait two phases ahead of a load of the other
// that is still in flight, and pass the wait on a stale parity.
constexpr int kBufs = 4;
constexpr int kTileS = kUnit + 2;         // tile width in sites (x0 - 1 .. x0 + 32)
constexpr uint32_t kTileBytes = 36u * kTileS * 16u;    // 19584: 36 planes x 34 sites
constexpr uint32_t kOffW = kTileBytes;                 // block tile (36 entry planes)
// stage 0 only: the x-wrap columns, 36 planes x 16 B each (the spinor and the
// block at the -x neighbour of the unit's x = 0 site, the spinor at the +x
// neighbour of its x = nx - 1 site)
constexpr uint32_t kOffX = 2u * kTileBytes;            // 39168
constexpr uint32_t kColBytes = 36u * 16u;              // 576
constexpr uint32_t kColStride = 640u;                  // 128-byte aligned column starts
constexpr uint32_t kBufBytes = ((kOffX + 3u * kColStride) + 1023u) & ~1023u;  // 41984
// the unit's diagonal matrices, double-buffered by unit after the ring:
// D (9 planes x 32 sites x 16 B), then B (9 planes x 32 sites x 8 B)
constexpr uint32_t kDiagD = 9u * kUnit * 16u;          // 4608
constexpr uint32_t kDiagB = 9u * kUnit * 8u;           // 2304
constexpr uint32_t kDiagStride = 7168u;
constexpr uint32_t kOffDiag = kBufs * kBufBytes;       // 167936
constexpr uint32_t kSmemBytes = kOffDiag + 2u * kDiagStride + 1024u;           // 183296
static_assert(kOffW % 128 == 0 && kOffX % 128 == 0 && kColStride % 128 == 0 && kColStride >= kColBytes &&
                  kBufBytes % 1024 == 0 && kDiagStride % 128 == 0 && kDiagD + kDiagB <= kDiagStride,
              "layout");
static_assert(kSmemBytes + 1024 <= 232448, "shared memory");
static_assert(kBufs % 2 == 0 && kLoads % 2 == 0, "a buffer's uses must all belong to one species");
static_assert(kMaxReg * 32 * 3 <= 16384, "registers of an SM quarter (three warps)");
}  // namespace mv5

struct Mv5Maps {
  CUtensorMap spin;  // 72 planes x 2V doubles, box {68, 36}
  CUtensorMap W;     // 216 planes x 2V doubles, box {68, 36}
  CUtensorMap spin1; // the same planes, one site: box {2, 36}
  CUtensorMap W1;
  CUtensorMap D;     // 9 planes x 2V doubles, box {64, 9}
  CUtensorMap B;     // 9 planes x V doubles, box {32, 9}
};

// entry (s, t) of s_k^T for the reference Pauli matrices (src/su2.f90:68-79
// holds s_2 transposed, so s_2^T = [[0,-i],[i,0]])
__device__ __forceinline__ cplx pauli_t5(int k, int s, int t) {
  if (k == 0) return (s != t) ? cplx{1.0, 0.0} : cplx{0.0, 0.0};
  if (k == 1) {
    if (s == 0 && t == 1) return {0.0, -1.0};
    if (s == 1 && t == 0) return {0.0, 1.0};
    return {0.0, 0.0};
  }
  if (s != t) return {0.0, 0.0};
  return (s == 0) ? cplx{1.0, 0.0} : cplx{-1.0, 0.0};
}

// One thread per (direction I, species, row g, site): row g of the forward
// block W_I(x) of that species, into planes (I*2 + sp)*36 + g*6 + column.
__global__ void __launch_bounds__(256) k_cn_blocks5(Lat L, CnCoef C, const double2 *__restrict__ U,
                                                    const double2 *__restrict__ DE, double2 *__restrict__ W) {
  const int64_t V = L.V;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 36 * V) return;
  const int64_t x = tid % V;
  const int64_t r = tid / V;  // (I*2 + sp)*6 + g
  const int g = (int)(r % 6);
  const int isp = (int)(r / 6);
  const int I = isp >> 1, sp = isp & 1;
  const int c = g >> 1, s = g & 1;
  const int K0 = (I + 2) % 3, K1 = (I + 1) % 3;
  const cplx ck = (-0.5 * C.inva2[I]) * C.kin[sp];
  const cplx cs0 = times_i(C.so[sp]), cs1 = -times_i(C.so[sp]);
  double2 *row = W + ((int64_t)isp * 36 + g * 6) * V + x;
#pragma unroll
  for (int cp = 0; cp < 3; ++cp) {
    const int e = cp * 3 + c;  // M^T[c][cp] = M[cp][c]
    const cplx u = ldg(U + (int64_t)(I * 9 + e) * V + x);
    const cplx d0 = ldg(DE + (int64_t)((I * 2 + 0) * 9 + e) * V + x);
    const cplx d1 = ldg(DE + (int64_t)((I * 2 + 1) * 9 + e) * V + x);
    const cplx ku = ck * u, e0 = cs0 * d0, e1 = cs1 * d1;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      cplx v = (s == t) ? ku : cplx{0.0, 0.0};
      v = v + pauli_t5(K0, s, t) * e0 + pauli_t5(K1, s, t) * e1;
      st(row + (int64_t)(2 * cp + t) * V, v);
    }
  }
}

namespace {

// Coordinates of a unit's first site, from two integer divisions per unit;
// everything else the pipeline needs follows from them by additions.
struct UnitPos {
  int x0, cx, cy, cz;
};
__device__ __forceinline__ UnitPos unit_pos(const Lat &L, int x0) {
  const int nx = (int)L.nx, ny = (int)L.ny;
  const int t = x0 / nx, z = t / ny;
  return {x0, x0 - t * nx, t - z * ny, z};
}

// the six periodic neighbours (+x,-x,+y,-y,+z,-z) of the site l sites after
// the unit's first (V < 2^31); its coordinates by carrying from the unit's
__device__ __forceinline__ void neighbours5(const Lat &L, const UnitPos &P, int l, int (&nb)[6]) {
  const int nx = (int)L.nx, ny = (int)L.ny, nz = (int)L.nz;
  int x = P.cx + l, y = P.cy, z = P.cz;
  while (x >= nx) {  // at most kUnit / nx + 1 rows
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

// first site of the spinor tile of stage stg of the unit (stage 0:
// x0 - 1; stages 1-4: the +y, -y, +z, -z neighbours of x0)
__device__ __forceinline__ int spin_start5(const Lat &L, const UnitPos &P, int stg) {
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
// first site of the block tile of a stage: forward stages read the blocks
// of the unit itself, backward stages those of the neighbours, stage 0 both
// (x0 - 1 .. x0 + 32, the spinor tile's sites)
__device__ __forceinline__ int blk_start5(int x0, int spin_start, int stg) {
  if (stg == 1 || stg == 3) return x0;
  return spin_start;
}

// Sites of the unit whose x neighbour wraps outside the stage-0 tile (rows
// of at least kUnit + 2 sites: one x = 0 and one x = nx - 1 site per unit at
// most): yl = the -x neighbour of its x = 0 site, yr = the +x neighbour of
// its x = nx - 1 site; -1 where the unit has no such site.
__device__ __forceinline__ void x_wraps5(const Lat &L, const UnitPos &P, int &yl, int &yr) {
  const int nx = (int)L.nx, V = (int)L.V, x0 = P.x0;
  yl = yr = -1;
  if (nx < mv5::kTileS) return;
  const int pl = P.cx == 0 ? 0 : nx - P.cx, pr = nx - 1 - P.cx;
  if (pl < mv5::kUnit && x0 + pl < V) yl = x0 + pl + nx - 1;
  if (pr < mv5::kUnit && x0 + pr < V) yr = x0 + pr - (nx - 1);
}

// 16-byte and 8-byte loads from shared-memory addresses (ld.shared)
__device__ __forceinline__ double2 lds_d2(uint32_t a) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ double lds_d1(uint32_t a) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}

// The thread's tile (rows 2c + s, c = 0..2; columns 3h + k, k = 0..2) +=
// sum over q of w[c][q] psi[q][3h + k].  Forward: w[c][q] = W(x)[2c+s][q],
// entry (2c+s)*6 + q; backward: w[c][q] = -conj(W(y)[q][2c+s]), entry
// q*6 + 2c + s.  load_w(e) reads entry e of the
// block, load_p(e) plane e of the spinor (species planes), from the shared
// tiles or global memory.
template <bool BWD, typename LW, typename LP>
__device__ __forceinline__ void nb_products(double (&acc)[3][3][2], int s, int h, LW load_w, LP load_p) {
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
__global__ void __maxnreg__(mv5::kMaxReg)
    k_cn_mv5(Lat L, CnCoef C, double nb_sign, const __grid_constant__ Mv5Maps maps, const double2 *__restrict__ W,
             MvArgs A, int nunits, int *err, long long wait_cycles, int stall_load) {
  using namespace mv5;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kBufs], empty_bar[kBufs], dfull[2], dempty[2];
  __shared__ volatile int s_issued;  // loads the producer issued (diagnostics of an expired wait)
  __shared__ double red[kWarps][3][3];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int V = (int)L.V;  // the launcher admits V < 2^31 only

  if (threadIdx.x == 0) {
    s_issued = 0;
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

  const int my_units = (nunits - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int total = my_units * kLoads;

  // bounded wait with this launch's limit
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
      const int stop = stall_load >= 0 ? min(stall_load, total) : total;
      bool ok = true;
      int i = 0, ndiag = 0;
      UnitPos P{0, 0, 0, 0};
      for (; i < stop && ok; ++i) {
        const int b = i % kBufs;
        if (i >= kBufs) {
          const uint32_t par = (uint32_t)((i / kBufs - 1) & 1);
          // every consumer warp of the species released the buffer, and its
          // previous load landed
          if (!wait(&empty_bar[b], par)) {
            record_timeout(err, 5, 2, i);
            ok = false;
          } else if (!mbar_wait(&full_bar[b], par)) {
            record_timeout(err, 5, 3, i);
            ok = false;
          }
          if (!ok) break;
        }
        const int li = i % kLoads, stg = li >> 1, sp = li & 1;
        if (li == 0) P = unit_pos(L, ((int)blockIdx.x + (i / kLoads) * (int)gridDim.x) * kUnit);
        const int x0 = P.x0;
        if (li == 0) {  // the unit's diagonal matrices, with its first load
          const int k = i / kLoads, db = k & 1;
          if (k >= 2) {
            const uint32_t dpar = (uint32_t)((k / 2 - 1) & 1);
            if (!wait(&dempty[db], dpar)) {
              record_timeout(err, 5, 2, i);
              ok = false;
            } else if (!mbar_wait(&dfull[db], dpar)) {
              record_timeout(err, 5, 3, i);
              ok = false;
            }
            if (!ok) break;
          }
          unsigned char *dd = smem + kOffDiag + db * kDiagStride;
          mbar_expect_tx(&dfull[db], kDiagD + kDiagB);
          tma_2d(dd, &maps.D, 2 * x0, 0, &dfull[db]);
          tma_2d(dd + kDiagD, &maps.B, x0, 0, &dfull[db]);
          ++ndiag;
        }
        const int ss = spin_start5(L, P, stg);
        const int ws = blk_start5(x0, ss, stg);
        const int I = stg == 0 ? 0 : (stg + 1) / 2;
        unsigned char *bb = smem + b * kBufBytes;
        int yl = -1, yr = -1;
        if (stg == 0) x_wraps5(L, P, yl, yr);
        uint32_t tx = 2u * kTileBytes;
        if (stg == 0) tx += (yl >= 0 ? 2u : 0u) * kColBytes + (yr >= 0 ? kColBytes : 0u);
        mbar_expect_tx(&full_bar[b], tx);
        tma_2d(bb, &maps.spin, 2 * ss, sp * 36, &full_bar[b]);
        tma_2d(bb + kOffW, &maps.W, 2 * ws, (I * 2 + sp) * 36, &full_bar[b]);
        if (stg == 0) {
          if (yl >= 0) {
            tma_2d(bb + kOffX, &maps.spin1, 2 * yl, sp * 36, &full_bar[b]);
            tma_2d(bb + kOffX + kColStride, &maps.W1, 2 * yl, sp * 36, &full_bar[b]);
          }
          if (yr >= 0) tma_2d(bb + kOffX + 2 * kColStride, &maps.spin1, 2 * yr, sp * 36, &full_bar[b]);
        }
        s_issued = i + 1;
      }
      // every issued load lands before the CTA exits: loads before the last
      // kBufs were waited for above
      for (int k = max(0, i - kBufs); k < i; ++k)
        if (!mbar_wait(&full_bar[k % kBufs], (uint32_t)((k / kBufs) & 1))) {
          record_timeout(err, 5, 4, k);
          break;
        }
      for (int k = max(0, ndiag - 2); k < ndiag; ++k)
        if (!mbar_wait(&dfull[k & 1], (uint32_t)((k >> 1) & 1))) {
          record_timeout(err, 5, 4, -1 - k);
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
  constexpr int NQ = (MODE == MV_T) ? 3 : ((MODE == MV_RES || MODE == MV_V || MODE == MV_RESC) ? 2 : 0);
  double qs[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) qs[k][0] = qs[k][1] = qs[k][2] = 0.0;
  const cplx ak = C.kin[sp], am = C.mag[sp], ad = C.dar[sp];
  const cplx dg = C.dkin * ak + cplx{1.0, 0.0};
  bool dead = false;

  for (int u = 0; u < my_units; ++u) {
    const UnitPos P = unit_pos(L, ((int)blockIdx.x + u * (int)gridDim.x) * kUnit);
    const int x0 = P.x0;
    const int x = x0 + site_in_unit;
    const bool act = x < V;
    const int xs = act ? x : V - 1;  // a valid site for the addresses of idle lanes
    int nb[6];
    neighbours5(L, P, xs - x0, nb);
    int yl = -1, yr = -1;
    x_wraps5(L, P, yl, yr);
    double acc[3][3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[c][k][0] = acc[c][k][1] = 0.0;
    // the epilogue's operand at the own site: b for the residuals, rh for V,
    // the input itself for RHS and T
    const double2 *epi_src = (MODE == MV_V) ? A.in2 : (MODE == MV_RES || MODE == MV_RESC) ? A.bvec : A.in;

#pragma unroll
    for (int stg = 0; stg < kStages; ++stg) {
      const int ld = u * kLoads + stg * 2 + sp;
      const int b = ld % kBufs;
      if (stg == kStages - 2 && MODE != MV_PLAIN) {
        // brought into L1 two stages ahead (no registers held), read there
        // in the epilogue
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int k = 0; k < 3; ++k)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(epi_src + (int64_t)(sp * 36 + (3 * h + k) * 6 + 2 * c + s) * V +
                                                          xs));
      }
      int role = -1;
      if (!dead && !wait(&full_bar[b], (uint32_t)((ld / kBufs) & 1))) role = 0;
      // stage 0 also reads the unit's diagonal matrices
      if (stg == 0 && !dead && role < 0 && !wait(&dfull[u & 1], (uint32_t)((u >> 1) & 1))) role = 1;
      // warp-uniform: the products below use warp votes
      if (__any_sync(0xffffffffu, role >= 0) && !dead) {
        dead = true;
        if (role >= 0) {
          record_timeout(err, 5, role, ld);
          if (err[3] == (int)blockIdx.x && err[2] == ld) {  // this thread's record: add the detail
            const uint64_t word = role == 0 ? *(volatile uint64_t *)&full_bar[b] : *(volatile uint64_t *)&dfull[u & 1];
            err[4] = s_issued + 1;
            err[5] = (int)(uint32_t)word;
            err[6] = (int)(uint32_t)(word >> 32);
            err[7] = role == 0 ? (ld / kBufs) & 1 : (u >> 1) & 1;
          }
        }
      }
      const unsigned char *bb = smem + b * kBufBytes;
      const uint32_t s_tile = smem_u32(bb), s_w = smem_u32(bb + kOffW);
      if (!dead) {
        const int ss = spin_start5(L, P, stg);
        const int ws = blk_start5(x0, ss, stg);
        if (stg == 0) {
          // diagonal (colour only): row (c, s) takes input rows (j, s);
          // x - ss = site_in_unit + 1 lies inside the tile for every lane
          const unsigned char *dd = smem + kOffDiag + (u & 1) * kDiagStride;
          const uint32_t s_d = smem_u32(dd) + (uint32_t)(site_in_unit * 16);
          const uint32_t s_b = smem_u32(dd + kDiagD) + (uint32_t)(site_in_unit * 8);
          const uint32_t s_own = s_tile + (uint32_t)((site_in_unit + 1) * 16 + s * kTileS * 16);
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            cplx cd[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const int e = j * 3 + c;
              const double2 dv = lds_d2(s_d + (uint32_t)(e * kUnit * 16));
              const double bv = lds_d1(s_b + (uint32_t)(e * kUnit * 8));
              cd[c] = ad * cplx{dv.x, dv.y} + bv * am;
              if (j == c) cd[c] = cd[c] + dg;
              cd[c] = nb_sign * cd[c];  // see the epilogue
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              const double2 p = lds_d2(s_own + (uint32_t)(((3 * h + k) * 6 + 2 * j) * kTileS * 16));
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                acc[c][k][0] = fma(cd[c].re, p.x, fma(-cd[c].im, p.y, acc[c][k][0]));
                acc[c][k][1] = fma(cd[c].re, p.y, fma(cd[c].im, p.x, acc[c][k][1]));
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
            // column (per-lane strides)
            const uint32_t xc = smem_u32(bb + kOffX);
            const uint32_t wa = ww ? xc + kColStride : s_w + (uint32_t)((m - ws) * 16);
            const uint32_t pa = pw ? xc + (bwd ? 0u : 2u * kColStride) : s_tile + (uint32_t)((y - ss) * 16);
            const uint32_t wst = ww ? 16u : (uint32_t)kTileS * 16u, pst = pw ? 16u : (uint32_t)kTileS * 16u;
            auto lw = [&](int e) { return lds_d2(wa + (uint32_t)e * wst); };
            auto lp = [&](int e) { return lds_d2(pa + (uint32_t)e * pst); };
            if (bwd)
              nb_products<true>(acc, s, h, lw, lp);
            else
              nb_products<false>(acc, s, h, lw, lp);
          } else if (__all_sync(0xffffffffu, (ps && wsh) || !act)) {
            // every operand of the warp in shared memory
            const uint32_t wa = s_w + (uint32_t)((m - ws) * 16), pa = s_tile + (uint32_t)((y - ss) * 16);
            auto lw = [&](int e) { return lds_d2(wa + (uint32_t)(e * kTileS * 16)); };
            auto lp = [&](int e) { return lds_d2(pa + (uint32_t)(e * kTileS * 16)); };
            if (bwd)
              nb_products<true>(acc, s, h, lw, lp);
            else
              nb_products<false>(acc, s, h, lw, lp);
          } else if (act) {
            // some lanes' operands outside the tiles (periodic wraps, tile
            // edges): those lanes read global memory, the others the tiles
            const double2 *wp = wsh ? (const double2 *)(bb + kOffW) + (m - ws)
                                    : W + (int64_t)((I * 2 + sp) * 36) * V + m;
            const double2 *pp = ps ? (const double2 *)bb + (y - ss) : A.in + (int64_t)(sp * 36) * V + y;
            const int64_t wst = wsh ? kTileS : V, pst = ps ? kTileS : V;
            auto lw = [&](int e) { return wp[e * wst]; };
            auto lp = [&](int e) { return pp[e * pst]; };
            if (bwd)
              nb_products<true>(acc, s, h, lw, lp);
            else
              nb_products<false>(acc, s, h, lw, lp);
          }
        }
      }
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&empty_bar[b]);
        if (stg == 0) mbar_arrive(&dempty[u & 1]);
      }
    }

    // ---------------------------------------------------------- epilogue
    if (!dead && act) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int64_t off = (int64_t)(sp * 36 + (3 * h + k) * 6 + 2 * c + s) * V + x;
          // D in + sgn N in = sgn (sgn D in + N in), sgn = +-1: the diagonal
          // was scaled by sgn and the neighbour sum was not
          const cplx y_ = {nb_sign * acc[c][k][0], nb_sign * acc[c][k][1]};
          const cplx ev = MODE == MV_PLAIN ? cplx{0.0, 0.0} : ldg(epi_src + off);
          if (MODE == MV_PLAIN) {
            st(A.out + off, y_);
          } else if (MODE == MV_RHS) {
            st(A.out + off, y_);
            st(A.out2 + off, 2.0 * y_ - ev);
          } else if (MODE == MV_RES) {
            const cplx rv = ev - y_;
            st(A.out + off, rv);
            st(A.out2 + off, rv);
            st(A.out3 + off, rv);
            qs[k][0] += norm2(rv);
            qs[k][1] += norm2(ev);
          } else if (MODE == MV_V) {
            st(A.out + off, y_);
            cplx dd = {0.0, 0.0};
            cmac_cj(dd, ev, y_);
            qs[k][0] += dd.re;
            qs[k][1] += dd.im;
          } else if (MODE == MV_RESC) {
            const cplx rv = ev - y_;
            const cplx dv = rv * A.inv_theta[sp];
            A.r32[off] = make_float2((float)rv.re, (float)rv.im);
            A.d32[off] = make_float2((float)dv.re, (float)dv.im);
            qs[k][0] += norm2(rv);
            qs[k][1] += norm2(ev);
          } else {  // MV_T: in = s
            st(A.out + off, y_);
            cplx dd = {0.0, 0.0};
            cmac_cj(dd, y_, ev);
            qs[k][0] += dd.re;
            qs[k][1] += dd.im;
            qs[k][2] += norm2(y_);
          }
        }
    }
  }

  // one partial row per CTA: each column summed over the warp's lanes, then
  // over the two spin warps of its species and half in a fixed order
  if constexpr (NQ > 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int kk = 0; kk < NQ; ++kk) {
        double v = qs[k][kk];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k][kk] = v;
      }
    named_bar_sync(1, kWarps * 32);
    if (threadIdx.x < CN_COLS * NQ) {
      const int col12 = threadIdx.x / NQ, kk = threadIdx.x % NQ;
      const int spc = col12 / 6, n = col12 % 6, hc = n / 3, k = n % 3;
      // warps 4 spc + 2 s + hc for s = 0, 1
      A.partials[((int64_t)blockIdx.x * CN_COLS + col12) * NQ + kk] =
          red[4 * spc + hc][k][kk] + red[4 * spc + 2 + hc][k][kk];
    }
  }
}

// ------------------------------------------------------------------ host
void launch_cn_blocks5(Lat L, const CnCoef &C, const double2 *U, const double2 *DE, double2 *W, cudaStream_t st) {
  const int64_t n = 36 * L.V;
  const unsigned grid = (unsigned)((n + 255) / 256);
  k_cn_blocks5<<<grid, 256, 0, st>>>(L, C, U, DE, W);
}

int64_t cn_mv5_units(int64_t V) { return (V + mv5::kUnit - 1) / mv5::kUnit; }
int64_t cn_mv5_rows(int64_t V, int sm_count) { return std::min<int64_t>(cn_mv5_units(V), sm_count); }
int64_t cn_mv5_block_entries(int64_t V) { return 216 * V; }

int launch_cn_mv5(int mode, Lat L, const CnCoef &C, double nb_sign, const double2 *W, const double2 *Dsum,
                  const double *Bsum, const MvArgs &a, int *err, int sm_count, cudaStream_t st,
                  long long wait_cycles, int stall_load) {
  using namespace mv5;
  const uint64_t V = (uint64_t)L.V;
  // B tiles start at x0 = 32 u (16-byte aligned rows need an even V as well)
  if (L.V < kTileS || L.V > 0x7fffffffLL || (L.V & 1)) return -1;
  Mv5Maps maps;
  memset(&maps, 0, sizeof(maps));
  if (!stage::encode(&maps.spin, a.in, 2 * V, 72, 2 * kTileS, 36) ||
      !stage::encode(&maps.W, W, 2 * V, 216, 2 * kTileS, 36) ||
      !stage::encode(&maps.spin1, a.in, 2 * V, 72, 2, 36) || !stage::encode(&maps.W1, W, 2 * V, 216, 2, 36) ||
      !stage::encode(&maps.D, Dsum, 2 * V, 9, 2 * kUnit, 9) || !stage::encode(&maps.B, Bsum, V, 9, kUnit, 9))
    return -1;
  const int nunits = (int)cn_mv5_units(L.V);
  const unsigned grid = (unsigned)cn_mv5_rows(L.V, sm_count);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    kern<<<grid, kThreads, kSmemBytes, st>>>(L, C, nb_sign, maps, W, a, nunits, err, wait_cycles, stall_load);
  };
  switch (mode) {
    case MV_PLAIN: go(k_cn_mv5<MV_PLAIN>); break;
    case MV_RHS: go(k_cn_mv5<MV_RHS>); break;
    case MV_RES: go(k_cn_mv5<MV_RES>); break;
    case MV_V: go(k_cn_mv5<MV_V>); break;
    case MV_RESC: go(k_cn_mv5<MV_RESC>); break;
    default: go(k_cn_mv5<MV_T>); break;
  }
  return 0;
}

}  // namespace nrq
