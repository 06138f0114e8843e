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
// Products.  Four threads share the 6x6 product of one site, species and
// neighbour: thread (kh, h) accumulates all six output rows of columns
// 3h .. 3h+2 over the input rows q = 3kh .. 3kh+2, 36 doubles in registers.
// Per input row it reads 6 block entries and 3 spinor entries from shared
// memory and does 72 FP64 FMAs, none of them padding: 108 16-byte loads per
// site, species and neighbour, against 144 for four 3x3 tiles over all six
// input rows.  On B200 the FP64 FMA pipe and the FP64 tensor pipe have the
// same peak, and the tensor pipe's 16x8 tiles hold 12 x 6 useful entries.  A
// 16-byte shared-memory load costs four wavefronts per warp whether or not
// lanes share addresses, so every warp holds 32 consecutive sites of one
// (row half, species, column half): each load then delivers 512 distinct
// bytes without bank conflicts, and the loads per site set the traffic.
// After a unit's last stage the two row-half warps of a (species, column
// half) sum their partial tiles through tensor memory (each keeps three of
// the six rows; exchange_halves), which takes no shared memory.
//
// Pipeline.  Persistent, one CTA per SM: 8 consumer warps (warp 4kh + 2sp +
// h) and a producer warpgroup, whose first warp issues the loads and which
// hands its registers to the consumers (setmaxnreg: 232 per consumer thread,
// which the 36 accumulators and the epilogue's operands need).  Ten loads per
// unit, per stage and species (stage 0: diagonal matrices, +x and -x; 1: +y;
// 2: -y; 3: +z; 4: -z): a spinor tile (34 sites x 36 planes) and a block tile
// (34 sites x 36 entry planes) by TMA, into a ring of five shared-memory
// buffers completed on mbarriers, one full barrier per buffer and species;
// the unit's diagonal matrices go with its first load into one of two
// further buffers.  The producer refills a buffer once the four consumer
// warps of its species released it and its previous load has landed.  The
// periodic x neighbours that wrap outside a unit's tile (one site at each
// row end) arrive as two extra one-site spinor columns and one block column
// with stage 0; a lane whose neighbour or block lies anywhere else outside
// the tiles (rows shorter than the tile) reads it from global memory.
// Results go straight to global memory; the epilogue's operand at the own
// site is loaded into registers two stages before the epilogue (the ring
// takes nearly all of the shared memory, so L1 is too small to hold it);
// the residual and dot-product partial sums stay in registers over all
// units of the CTA (one partial row per CTA).
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
#include "tc.cuh"

namespace nrq {

namespace mv5 {
constexpr int kUnit = 32;                 // sites per work unit (one per lane)
constexpr int kWarps = 8;                 // consumer warps: (species, spin, column half)
// the producer warpgroup (warps 8-11: warp 8 loads, 9-11 leave) gives its
// registers to the two consumer warpgroups (setmaxnreg)
constexpr int kThreads = (kWarps + 4) * 32;
constexpr int kMaxReg = 168;              // at launch: 12 warps x 32 x 168 = 64512 registers
constexpr int kProdReg = 40, kConsReg = 232;
constexpr int kStages = 5;                // stages per unit
constexpr int kLoads = 2 * kStages;       // loads per unit: (stage, species)
// Ring of load buffers.  Loads alternate between the species (load i is of
// species i & 1), and a consumer waits on a full barrier by phase parity,
// which is only sound while it never waits more than one phase ahead of the
// barrier's last completed phase.  Each buffer therefore has one full
// barrier per species, completed only by that species' loads: the k-th load
// of a species into a buffer is load i with i / kPer = k, and its consumers
// released the (k-1)-th themselves.  With an odd ring the uses of a buffer
// alternate species; a single full barrier per buffer would then let one
// species wait two phases ahead of a load of the other still in flight and
// pass the wait on a stale parity.  The empty barriers have one waiter, the
// producer, which takes every use of a buffer in order.
constexpr int kBufs = 5;
constexpr int kPer = (kBufs % 2) ? 2 * kBufs : kBufs;  // loads between two uses of one (buffer, species)
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
constexpr uint32_t kOffDiag = kBufs * kBufBytes;       // 209920
constexpr uint32_t kSmemBytes = kOffDiag + 2u * kDiagStride + 1024u;           // 225280
constexpr uint32_t kTmemCols = 128;  // the exchange: columns 0-35 and 64-99 of every lane
static_assert(kOffW % 128 == 0 && kOffX % 128 == 0 && kColStride % 128 == 0 && kColStride >= kColBytes &&
                  kBufBytes % 1024 == 0 && kDiagStride % 128 == 0 && kDiagD + kDiagB <= kDiagStride,
              "layout");
static_assert(kSmemBytes + 1024 <= 232448, "shared memory");
static_assert(kLoads % 2 == 0, "load i is of species i & 1");
static_assert(kMaxReg * kThreads <= 65536 && kMaxReg * 32 * 3 <= 16384, "registers at launch");
static_assert(kProdReg * 128 + kConsReg * 256 <= kMaxReg * kThreads && (2 * kConsReg + kProdReg) * 32 <= 16384,
              "the split draws only on the launch's registers and fits each SM quarter");
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

// One thread per (direction I, colour row c, site): rows g = 2c + s of the
// forward blocks W_I(x) of both species, column 2cp + t, into plane
// (I*2 + sp)*36 + g*6 + column, in FP64 (W) and/or rounded to FP32 (Wf, the
// FP32 Chebyshev stencil's blocks).  The entries (cp, c) of the link and
// the two derived matrices belong to this c alone, so every input is read
// once, and every store is coalesced over the warp's consecutive sites.
template <bool F64, bool F32>
__global__ void __launch_bounds__(256) k_cn_blocks5(Lat L, CnCoef C, const double2 *__restrict__ U,
                                                    const double2 *__restrict__ DE, double2 *__restrict__ W,
                                                    float2 *__restrict__ Wf) {
  const int64_t V = L.V;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 9 * V) return;
  const int64_t x = tid % V;
  const int r = (int)(tid / V);  // I*3 + c
  const int I = r / 3, c = r % 3;
  const int K0 = (I + 2) % 3, K1 = (I + 1) % 3;
  cplx u[3], d0[3], d1[3];
#pragma unroll
  for (int cp = 0; cp < 3; ++cp) {
    const int e = cp * 3 + c;  // M^T[c][cp] = M[cp][c]
    u[cp] = ldg(U + (int64_t)(I * 9 + e) * V + x);
    d0[cp] = ldg(DE + (int64_t)((I * 2 + 0) * 9 + e) * V + x);
    d1[cp] = ldg(DE + (int64_t)((I * 2 + 1) * 9 + e) * V + x);
  }
#pragma unroll
  for (int sp = 0; sp < 2; ++sp) {
    const cplx ck = (-0.5 * C.inva2[I]) * C.kin[sp];
    const cplx cs0 = times_i(C.so[sp]), cs1 = -times_i(C.so[sp]);
#pragma unroll
    for (int cp = 0; cp < 3; ++cp) {
      const cplx ku = ck * u[cp], e0 = cs0 * d0[cp], e1 = cs1 * d1[cp];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int g = 2 * c + s;
        const int64_t row = ((int64_t)(I * 2 + sp) * 36 + g * 6) * V + x;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          cplx v = (s == t) ? ku : cplx{0.0, 0.0};
          v = v + pauli_t5(K0, s, t) * e0 + pauli_t5(K1, s, t) * e1;
          if (F64) st(W + row + (int64_t)(2 * cp + t) * V, v);
          if (F32) Wf[row + (int64_t)(2 * cp + t) * V] = make_float2((float)v.re, (float)v.im);
        }
      }
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

// Position of work unit u (32 consecutive sites along x).  Where every row
// holds whole units (nx a multiple of 32) and ny, nz are multiples of 8, the
// units are taken in blocks of 8 x 8 rows (x fastest, then y and z within
// the block, then the blocks), so that the +-y and +-z tiles a unit shares
// with its neighbours are read within a few hundred units of each other,
// while L2 still holds them, at any lattice size (in site order the +-z
// tiles are a whole plane of units apart: 127 MB of loads at 128^3);
// otherwise in site order.
__device__ __forceinline__ UnitPos unit_pos_of(const Lat &L, int u) {
  const int nx = (int)L.nx, ny = (int)L.ny, nz = (int)L.nz;
  if ((nx & 31) || (ny & 7) || (nz & 7)) return unit_pos(L, u * mv5::kUnit);
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

// The thread's partial tile (rows r = 0..5; columns 3h + k, k = 0..2) +=
// sum over its three input rows q = 3 kh + qq of w[r][q] psi[q][3h + k].
// Forward: w[r][q] = W(x)[r][q], entry r*6 + q; backward: w[r][q] =
// -conj(W(y)[q][r]), entry q*6 + r.  load_w(e) reads entry e + (3 kh,
// backward 18 kh) of the block and load_p(e) plane e + 18 h + 3 kh of the
// spinor (species planes), from the shared tiles or global memory: the
// callers fold the thread's offsets into their base addresses, so that e
// is a constant of the unrolled loops.
template <bool BWD, typename LW, typename LP>
__device__ __forceinline__ void nb_products(double (&acc)[6][3][2], LW load_w, LP load_p) {
#pragma unroll
  for (int qq = 0; qq < 3; ++qq) {
    double wr[6], wi[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      const double2 wv = load_w(BWD ? qq * 6 + r : r * 6 + qq);
      wr[r] = BWD ? -wv.x : wv.x;
      wi[r] = wv.y;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 p = load_p(k * 6 + qq);
#pragma unroll
      for (int r = 0; r < 6; ++r) {
        acc[r][k][0] = fma(wr[r], p.x, fma(-wi[r], p.y, acc[r][k][0]));
        acc[r][k][1] = fma(wr[r], p.y, fma(wi[r], p.x, acc[r][k][1]));
      }
    }
  }
}

// The diagonal (colour only) of the thread's input rows q = 3 KH + qq: row
// 2c + (q & 1) takes cd[c][q >> 1] psi[q], cd from the unit's D and B tiles.
template <int KH>
__device__ __forceinline__ void diag_products(double (&acc)[6][3][2], int h, uint32_t s_d, uint32_t s_b,
                                              uint32_t s_own, cplx ad, cplx am, cplx dg, double nb_sign) {
#pragma unroll
  for (int qq = 0; qq < 3; ++qq) {
    constexpr int kTile = mv5::kTileS * 16;
    const int q = 3 * KH + qq, j = q >> 1, sq = q & 1;
    cplx cd[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int e = j * 3 + c;
      const double2 dv = lds_d2(s_d + (uint32_t)(e * mv5::kUnit * 16));
      const double bv = lds_d1(s_b + (uint32_t)(e * mv5::kUnit * 8));
      cd[c] = ad * cplx{dv.x, dv.y} + bv * am;
      if (j == c) cd[c] = cd[c] + dg;
      cd[c] = nb_sign * cd[c];  // see the epilogue
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 p = lds_d2(s_own + (uint32_t)(((3 * h + k) * 6 + q) * kTile));
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc[2 * c + sq][k][0] = fma(cd[c].re, p.x, fma(-cd[c].im, p.y, acc[2 * c + sq][k][0]));
        acc[2 * c + sq][k][1] = fma(cd[c].re, p.y, fma(cd[c].im, p.x, acc[2 * c + sq][k][1]));
      }
    }
  }
}

// Tensor memory as the scratch of the exchange: 36 columns of 32 bits per
// lane (nine complex doubles), the lane quarter of the warp.
__device__ __forceinline__ void tmem_st36(uint32_t taddr, const uint32_t (&w)[36]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr), "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(w[8]), "r"(w[9]), "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]), "r"(w[14]), "r"(w[15]), "r"(w[16]), "r"(w[17]), "r"(w[18]), "r"(w[19]), "r"(w[20]), "r"(w[21]), "r"(w[22]), "r"(w[23]), "r"(w[24]), "r"(w[25]), "r"(w[26]), "r"(w[27]), "r"(w[28]), "r"(w[29]), "r"(w[30]), "r"(w[31]) : "memory");
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr + 32u), "r"(w[32]),
               "r"(w[33]), "r"(w[34]), "r"(w[35])
               : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld36(uint32_t taddr, uint32_t (&w)[36]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];" : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7]), "=r"(w[8]), "=r"(w[9]), "=r"(w[10]), "=r"(w[11]), "=r"(w[12]), "=r"(w[13]), "=r"(w[14]), "=r"(w[15]), "=r"(w[16]), "=r"(w[17]), "=r"(w[18]), "=r"(w[19]), "=r"(w[20]), "=r"(w[21]), "=r"(w[22]), "=r"(w[23]), "=r"(w[24]), "=r"(w[25]), "=r"(w[26]), "=r"(w[27]), "=r"(w[28]), "=r"(w[29]), "=r"(w[30]), "=r"(w[31]) : "r"(taddr) : "memory");
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(w[32]), "=r"(w[33]), "=r"(w[34]), "=r"(w[35])
               : "r"(taddr + 32u)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// The two warps of a (species, column half) hold partial tiles over the two
// halves of the input rows; warp kh keeps output rows 3 kh .. 3 kh + 2.  Both
// share a tensor-memory lane quarter (warp & 3): each writes the other's
// three rows into its own 36 columns (64 kh ..), and after the pair's
// barrier reads the partner's columns and adds them to its rows.
template <int KH>
__device__ __forceinline__ void exchange_halves(const double (&acc)[6][3][2], double (&res)[3][3][2],
                                                uint32_t tbase, int warp, int bar_id) {
  const uint32_t quarter = tbase + ((uint32_t)(32 * (warp & 3)) << 16);
  uint32_t w[36];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const double v = acc[3 * (1 - KH) + i][k][ri];
        w[(i * 3 + k) * 4 + 2 * ri] = (uint32_t)__double2loint(v);
        w[(i * 3 + k) * 4 + 2 * ri + 1] = (uint32_t)__double2hiint(v);
      }
  tmem_st36(quarter + 64u * KH, w);
  tc::fence_before_sync();
  named_bar_sync(bar_id, 64);
  tc::fence_after_sync();
  tmem_ld36(quarter + 64u * (1 - KH), w);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int ri = 0; ri < 2; ++ri)
        res[i][k][ri] = acc[3 * KH + i][k][ri] +
                        __hiloint2double((int)w[(i * 3 + k) * 4 + 2 * ri + 1], (int)w[(i * 3 + k) * 4 + 2 * ri]);
  tc::fence_before_sync();
  named_bar_sync(bar_id, 64);  // the columns are free for the next unit
  tc::fence_after_sync();
}

}  // namespace

// Sum of six doubles over the warp by halving exchanges (8 shuffles where
// six butterflies take 30): after the exchange across lane bit 4 each half
// of the warp carries three of the values, across bit 3 two (the third
// padded), across bit 2 one, then bits 1 and 0 finish the sum.  Lane L ends
// with value 3 (L >> 4) + 2 ((L >> 3) & 1) + ((L >> 2) & 1) (index 3 of a
// half is the padding); warp_sum6_slot gives that index, or -1.
__device__ __forceinline__ double warp_sum6(const double v[6], int lane) {
  const bool b4 = (lane >> 4) & 1, b3 = (lane >> 3) & 1, b2 = (lane >> 2) & 1;
  double w[4];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double mine = b4 ? v[j + 3] : v[j], other = b4 ? v[j] : v[j + 3];
    w[j] = mine + __shfl_xor_sync(0xffffffffu, other, 16);
  }
  w[3] = 0.0;
  double y[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const double mine = b3 ? w[j + 2] : w[j], other = b3 ? w[j] : w[j + 2];
    y[j] = mine + __shfl_xor_sync(0xffffffffu, other, 8);
  }
  double z = (b2 ? y[1] : y[0]) + __shfl_xor_sync(0xffffffffu, b2 ? y[0] : y[1], 4);
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}
__device__ __forceinline__ int warp_sum6_slot(int lane) {
  if (lane & 3) return -1;
  const int idx = 2 * ((lane >> 3) & 1) + ((lane >> 2) & 1);
  return idx < 3 ? 3 * (lane >> 4) + idx : -1;
}

template <int MODE>
__global__ void __maxnreg__(mv5::kMaxReg)
    k_cn_mv5(Lat L, CnCoef C, double nb_sign, const __grid_constant__ Mv5Maps maps, const double2 *__restrict__ W,
             MvArgs A, int nunits, int *err, long long wait_cycles, int stall_load) {
  using namespace mv5;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kBufs][2], empty_bar[kBufs], dfull[2], dempty[2];
  __shared__ volatile int s_issued;  // loads the producer issued (diagnostics of an expired wait)
  __shared__ uint32_t s_tmem;        // the exchange's tensor-memory columns
  __shared__ double red[kWarps][3][MODE == MV_T2 ? 5 : MODE == MV_RES2 ? 4 : 3];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int V = (int)L.V;  // the launcher admits V < 2^31 only

  if (threadIdx.x == 0) {
    s_issued = 0;
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(&full_bar[b][0], 1);
      mbar_init(&full_bar[b][1], 1);
      mbar_init(&empty_bar[b], 4);  // the four consumer warps of the load's species
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], 1);
      mbar_init(&dempty[b], kWarps);  // every consumer warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(&s_tmem, kTmemCols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = s_tmem;

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
  if (warp >= kWarps) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kProdReg));
    if (warp == kWarps && lane == 0) {
      const int stop = stall_load >= 0 ? min(stall_load, total) : total;
      bool ok = true;
      int i = 0, ndiag = 0;
      UnitPos P{0, 0, 0, 0};
      for (; i < stop && ok; ++i) {
        const int b = i % kBufs;
        if (i >= kBufs) {
          const uint32_t par = (uint32_t)((i / kBufs - 1) & 1);
          const int j = i - kBufs;  // the buffer's previous load
          // every consumer warp of the species released the buffer, and its
          // previous load landed
          if (!wait(&empty_bar[b], par)) {
            record_timeout(err, 5, 2, i);
            ok = false;
          } else if (!mbar_wait(&full_bar[b][j & 1], (uint32_t)((j / kPer) & 1))) {
            record_timeout(err, 5, 3, i);
            ok = false;
          }
          if (!ok) break;
        }
        const int li = i % kLoads, stg = li >> 1, sp = li & 1;
        if (li == 0) P = unit_pos_of(L, (int)blockIdx.x + (i / kLoads) * (int)gridDim.x);
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
        uint64_t *fb = &full_bar[b][sp];
        mbar_expect_tx(fb, tx);
        tma_2d(bb, &maps.spin, 2 * ss, sp * 36, fb);
        tma_2d(bb + kOffW, &maps.W, 2 * ws, (I * 2 + sp) * 36, fb);
        if (stg == 0) {
          if (yl >= 0) {
            tma_2d(bb + kOffX, &maps.spin1, 2 * yl, sp * 36, fb);
            tma_2d(bb + kOffX + kColStride, &maps.W1, 2 * yl, sp * 36, fb);
          }
          if (yr >= 0) tma_2d(bb + kOffX + 2 * kColStride, &maps.spin1, 2 * yr, sp * 36, fb);
        }
        s_issued = i + 1;
      }
      // every issued load lands before the CTA exits: loads before the last
      // kBufs were waited for above
      for (int k = max(0, i - kBufs); k < i; ++k)
        if (!mbar_wait(&full_bar[k % kBufs][k & 1], (uint32_t)((k / kPer) & 1))) {
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
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kConsReg));

  // ---------------------------------------------------------- consumers
  // warp w = 4 kh + 2 sp + h: input-row half kh, species sp, column half h;
  // lane = site of the 32-site unit.  The thread accumulates all six output
  // rows of columns 3h .. 3h + 2 over input rows 3 kh .. 3 kh + 2 of its site
  // and species; after the unit's last stage it keeps rows 3 kh .. 3 kh + 2
  // of the sum (exchange_halves with warp w ^ 4).
  const int kh = warp >> 2, sp = (warp >> 1) & 1, h = warp & 1;
  const int pair_bar = 2 + (warp & 3);  // named barrier of the warp pair (ids 2-5)
  // the thread's first spinor plane and block entries (see nb_products)
  const int pofs = 18 * h + 3 * kh, wofs_f = 3 * kh, wofs_b = 18 * kh;
  const int site_in_unit = lane;
  constexpr int NQ = MODE == MV_T2 ? 5 : MODE == MV_RES2 ? 4 : (MODE == MV_T) ? 3
                   : ((MODE == MV_RES || MODE == MV_V || MODE == MV_V2 || MODE == MV_RESC) ? 2 : 0);
  // the products with the FP32 shadow residual (MV_T2: rh.t, MV_RES2:
  // rh.r) are summed over the warp after every unit into the warp's own
  // slots XQ, XQ + 1 of red, which keeps them out of the registers of the
  // stage loop; the other sums (NR per column) stay in registers
  constexpr int XQ = MODE == MV_T2 ? 3 : MODE == MV_RES2 ? 2 : -1;
  constexpr int NR = XQ >= 0 ? XQ : NQ;
  constexpr bool kShadow = MODE == MV_T2 || MODE == MV_V2;  // reads sh32
  double qs[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) qs[k][0] = qs[k][1] = qs[k][2] = 0.0;
  // the lane that ends with value j of the per-unit sums (re and im of the
  // three columns) owns its slot of red, which it clears here
  if (XQ >= 0 && warp_sum6_slot(lane) >= 0) {
    const int j = warp_sum6_slot(lane);
    red[warp][j >> 1][XQ + (j & 1)] = 0.0;
  }
  const cplx ak = C.kin[sp], am = C.mag[sp], ad = C.dar[sp];
  const cplx dg = C.dkin * ak + cplx{1.0, 0.0};
  bool dead = false;

  for (int u = 0; u < my_units; ++u) {
    const UnitPos P = unit_pos_of(L, (int)blockIdx.x + u * (int)gridDim.x);
    const int x0 = P.x0;
    const int x = x0 + site_in_unit;
    const bool act = x < V;
    const int xs = act ? x : V - 1;  // a valid site for the addresses of idle lanes
    int nb[6];
    neighbours5(L, P, xs - x0, nb);
    int yl = -1, yr = -1;
    x_wraps5(L, P, yl, yr);
    double acc[6][3][2];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[r][k][0] = acc[r][k][1] = 0.0;
    // the epilogue's operand at the own site: b for the residuals, rh for V,
    // the input itself for RHS and T; the FP32 shadow residual for V2, T2
    const double2 *epi_src =
        (MODE == MV_V) ? A.in2 : (MODE == MV_RES || MODE == MV_RES2 || MODE == MV_RESC) ? A.bvec : A.in;
    cplx ev[3][3];
    float2 eh[3][3];

#pragma unroll
    for (int stg = 0; stg < kStages; ++stg) {
      const int ld = u * kLoads + stg * 2 + sp;
      const int b = ld % kBufs;
      if (stg == kStages - 2 && MODE != MV_PLAIN) {
        // the epilogue's operands, loaded into registers two stages ahead
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int64_t o = (int64_t)(sp * 36 + (3 * h + k) * 6 + 3 * kh + i) * V + xs;
            if (MODE != MV_V2) ev[i][k] = ldg(epi_src + o);
            if (kShadow) eh[i][k] = __ldg(A.sh32 + o);
          }
      }
      int role = -1;
      if (!dead && !wait(&full_bar[b][sp], (uint32_t)((ld / kPer) & 1))) role = 0;
      // stage 0 also reads the unit's diagonal matrices
      if (stg == 0 && !dead && role < 0 && !wait(&dfull[u & 1], (uint32_t)((u >> 1) & 1))) role = 1;
      // warp-uniform: the products below use warp votes
      if (__any_sync(0xffffffffu, role >= 0) && !dead) {
        dead = true;
        if (role >= 0) {
          record_timeout(err, 5, role, ld);
          if (err[3] == (int)blockIdx.x && err[2] == ld) {  // this thread's record: add the detail
            const uint64_t word =
                role == 0 ? *(volatile uint64_t *)&full_bar[b][sp] : *(volatile uint64_t *)&dfull[u & 1];
            err[4] = s_issued + 1;
            err[5] = (int)(uint32_t)word;
            err[6] = (int)(uint32_t)(word >> 32);
            err[7] = role == 0 ? (ld / kPer) & 1 : (u >> 1) & 1;
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
          const uint32_t s_own = s_tile + (uint32_t)((site_in_unit + 1) * 16);
          if (kh == 0)
            diag_products<0>(acc, h, s_d, s_b, s_own, ad, am, dg, nb_sign);
          else
            diag_products<1>(acc, h, s_d, s_b, s_own, ad, am, dg, nb_sign);
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
            const uint32_t wst = ww ? 16u : (uint32_t)kTileS * 16u, pst = pw ? 16u : (uint32_t)kTileS * 16u;
            const uint32_t wa = (ww ? xc + kColStride : s_w + (uint32_t)((m - ws) * 16)) +
                                (uint32_t)(bwd ? wofs_b : wofs_f) * wst;
            const uint32_t pa =
                (pw ? xc + (bwd ? 0u : 2u * kColStride) : s_tile + (uint32_t)((y - ss) * 16)) + (uint32_t)pofs * pst;
            auto lw = [&](int e) { return lds_d2(wa + (uint32_t)e * wst); };
            auto lp = [&](int e) { return lds_d2(pa + (uint32_t)e * pst); };
            if (bwd)
              nb_products<true>(acc, lw, lp);
            else
              nb_products<false>(acc, lw, lp);
          } else if (__all_sync(0xffffffffu, (ps && wsh) || !act)) {
            // every operand of the warp in shared memory
            constexpr uint32_t kPl = kTileS * 16u;  // plane stride of the tiles
            const uint32_t wa = s_w + (uint32_t)((m - ws) * 16) + (uint32_t)(bwd ? wofs_b : wofs_f) * kPl;
            const uint32_t pa = s_tile + (uint32_t)((y - ss) * 16) + (uint32_t)pofs * kPl;
            auto lw = [&](int e) { return lds_d2(wa + (uint32_t)e * kPl); };
            auto lp = [&](int e) { return lds_d2(pa + (uint32_t)e * kPl); };
            if (bwd)
              nb_products<true>(acc, lw, lp);
            else
              nb_products<false>(acc, lw, lp);
          } else if (act) {
            // some lanes' operands outside the tiles (periodic wraps, tile
            // edges): those lanes read global memory, the others the tiles
            const int64_t wst = wsh ? kTileS : V, pst = ps ? kTileS : V;
            const double2 *wp = (wsh ? (const double2 *)(bb + kOffW) + (m - ws)
                                     : W + (int64_t)((I * 2 + sp) * 36) * V + m) +
                                (bwd ? wofs_b : wofs_f) * wst;
            const double2 *pp = (ps ? (const double2 *)bb + (y - ss) : A.in + (int64_t)(sp * 36) * V + y) + pofs * pst;
            auto lw = [&](int e) { return wp[e * wst]; };
            auto lp = [&](int e) { return pp[e * pst]; };
            if (bwd)
              nb_products<true>(acc, lw, lp);
            else
              nb_products<false>(acc, lw, lp);
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
    // every warp of the pair takes both barriers of the exchange, dead or
    // not, active lanes or not
    cplx ht[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};  // this unit's product with the shadow, per column
    double res[3][3][2];
    if (kh == 0)
      exchange_halves<0>(acc, res, tbase, warp, pair_bar);
    else
      exchange_halves<1>(acc, res, tbase, warp, pair_bar);
    if (!dead && act) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int64_t off = (int64_t)(sp * 36 + (3 * h + k) * 6 + 3 * kh + i) * V + x;
          // D in + sgn N in = sgn (sgn D in + N in), sgn = +-1: the diagonal
          // was scaled by sgn and the neighbour sum was not
          const cplx y_ = {nb_sign * res[i][k][0], nb_sign * res[i][k][1]};
          const cplx ev_ = ev[i][k];
          if (MODE == MV_PLAIN) {
            st(A.out + off, y_);
          } else if (MODE == MV_RHS) {
            st(A.out + off, y_);
            st(A.out2 + off, 2.0 * y_ - ev_);
          } else if (MODE == MV_RES) {
            const cplx rv = ev_ - y_;
            st(A.out + off, rv);
            st(A.out2 + off, rv);
            st(A.out3 + off, rv);
            qs[k][0] += norm2(rv);
            qs[k][1] += norm2(ev_);
          } else if (MODE == MV_RES2) {
            const cplx rv = ev_ - y_;
            const float2 f = make_float2((float)rv.re, (float)rv.im);
            st(A.out + off, rv);
            A.sh32[off] = f;
            st(A.out3 + off, rv);
            qs[k][0] += norm2(rv);
            qs[k][1] += norm2(ev_);
            cmac_cj(ht[k], cplx{(double)f.x, (double)f.y}, rv);
          } else if (MODE == MV_V) {
            st(A.out + off, y_);
            cplx dd = {0.0, 0.0};
            cmac_cj(dd, ev_, y_);
            qs[k][0] += dd.re;
            qs[k][1] += dd.im;
          } else if (MODE == MV_V2) {
            st(A.out + off, y_);
            cplx dd = {0.0, 0.0};
            cmac_cj(dd, cplx{(double)eh[i][k].x, (double)eh[i][k].y}, y_);
            qs[k][0] += dd.re;
            qs[k][1] += dd.im;
          } else if (MODE == MV_RESC) {
            const cplx rv = ev_ - y_;
            const cplx dv = rv * A.inv_theta[sp];
            A.r32[off] = make_float2((float)rv.re, (float)rv.im);
            A.d32[off] = make_float2((float)dv.re, (float)dv.im);
            qs[k][0] += norm2(rv);
            qs[k][1] += norm2(ev_);
          } else {  // MV_T, MV_T2: in = s
            st(A.out + off, y_);
            cplx dd = {0.0, 0.0};
            cmac_cj(dd, y_, ev_);
            qs[k][0] += dd.re;
            qs[k][1] += dd.im;
            qs[k][2] += norm2(y_);
            if (MODE == MV_T2) cmac_cj(ht[k], cplx{(double)eh[i][k].x, (double)eh[i][k].y}, y_);
          }
        }
    }
    if (XQ >= 0) {
      const double hv[6] = {ht[0].re, ht[0].im, ht[1].re, ht[1].im, ht[2].re, ht[2].im};
      const double z = warp_sum6(hv, lane);
      const int j = warp_sum6_slot(lane);  // recomputed: a register held across the stages spills
      if (j >= 0) red[warp][j >> 1][XQ + (j & 1)] += z;
    }
  }

  // every consumer warp is done with the tensor memory before warp 0 frees it
  tc::fence_before_sync();
  named_bar_sync(1, kWarps * 32);
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tbase, kTmemCols);

  // one partial row per CTA: each column summed over the warp's lanes, then
  // over the two row-half warps of its species and column half in a fixed
  // order
  if constexpr (NQ > 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int kk = 0; kk < NR; ++kk) {  // the shadow products are in red already
        double v = qs[k][kk];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k][kk] = v;
      }
    named_bar_sync(1, kWarps * 32);
    if (threadIdx.x < CN_COLS * NQ) {
      const int col12 = threadIdx.x / NQ, kk = threadIdx.x % NQ;
      const int spc = col12 / 6, n = col12 % 6, hc = n / 3, k = n % 3;
      // warps 4 kh + 2 spc + hc for kh = 0, 1
      A.partials[((int64_t)blockIdx.x * CN_COLS + col12) * NQ + kk] =
          red[2 * spc + hc][k][kk] + red[4 + 2 * spc + hc][k][kk];
    }
  }
}

// The same stencil over every field of a batch (the batching form's
// right-hand side and refinement residual; k_batch_mv2 in cn_mv.cu is the
// register-tiled alternative): work items (field, unit), field fastest
// (order 0) or unit fastest (order 1).  MV_RHS reads psi (b = A psi, x = 2b
// - psi), MV_RESC the iterate x (r = b - A^H x rounded to FP32, d = r /
// theta), each from the field's own tensor maps (fmaps), both on the field's
// block set (wblk: blocks built with that mass's A^H coefficients, so A is
// the neighbour sum negated).  A field that converged sits a residual out
// (skip_done).  The residual's partial sums form one row per (field, unit),
// the rows launch_batch_finalize reads, summed in a fixed order.
template <int MODE>
__global__ void __maxnreg__(mv5::kMaxReg)
    k_batch_mv5(Lat L, const __grid_constant__ Mv5Maps maps, const double2 *__restrict__ W, int nunits, int *err,
                long long wait_cycles, const BatchField *__restrict__ tab, const CnBatchMaps *__restrict__ fmaps,
                int nfields, int order, int skip_done) {
  using namespace mv5;
  static_assert(MODE == MV_RHS || MODE == MV_RESC, "batch modes");
  const int nwork = nfields * nunits;
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
  constexpr int kIn = MODE == MV_RHS ? 0 : 1;  // the field's input: psi or x
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kBufs][2], empty_bar[kBufs], dfull[2], dempty[2];
  __shared__ volatile int s_issued;  // loads the producer issued (diagnostics of an expired wait)
  __shared__ uint32_t s_tmem;        // the exchange's tensor-memory columns
  __shared__ double redb[2][2][2][3][2];  // per item parity, species, column half, column, sum
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int V = (int)L.V;  // the launcher admits V < 2^31 only

  if (threadIdx.x == 0) {
    s_issued = 0;
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(&full_bar[b][0], 1);
      mbar_init(&full_bar[b][1], 1);
      mbar_init(&empty_bar[b], 4);  // the four consumer warps of the load's species
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], 1);
      mbar_init(&dempty[b], kWarps);  // every consumer warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(&s_tmem, kTmemCols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = s_tmem;


  // bounded wait with this launch's limit
  auto wait = [&](uint64_t *bar, uint32_t parity) -> bool {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
      if (clock64() - t0 > wait_cycles) return false;
    return true;
  };

  // ---------------------------------------------------------- producer
  if (warp >= kWarps) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kProdReg));
    if (warp == kWarps && lane == 0) {
      bool ok = true;
      int i = 0, ndiag = 0, k = 0;  // loads issued, diagonal loads issued, items begun
      for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x) {
        int f, u;
        item(w, f, u);
        if (skip(f)) continue;
        const UnitPos P = unit_pos_of(L, u);
        const int x0 = P.x0;
        const CUtensorMap *spin = &fmaps[f].in[kIn].spin, *spin1 = &fmaps[f].in[kIn].spin1;
        const int wrow = tab[f].wblk * 216;
        {  // the unit's diagonal matrices, with its first load
          const int db = k & 1;
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
        for (int li = 0; li < kLoads && ok; ++li, ++i) {
          const int b = i % kBufs;
          if (i >= kBufs) {
            const uint32_t par = (uint32_t)((i / kBufs - 1) & 1);
            const int j = i - kBufs;  // the buffer's previous load
            // every consumer warp of the species released the buffer, and
            // its previous load landed
            if (!wait(&empty_bar[b], par)) {
              record_timeout(err, 5, 2, i);
              ok = false;
            } else if (!mbar_wait(&full_bar[b][j & 1], (uint32_t)((j / kPer) & 1))) {
              record_timeout(err, 5, 3, i);
              ok = false;
            }
            if (!ok) break;
          }
          const int stg = li >> 1, sp = li & 1;
          const int ss = spin_start5(L, P, stg);
          const int ws = blk_start5(x0, ss, stg);
          const int I = stg == 0 ? 0 : (stg + 1) / 2;
          unsigned char *bb = smem + b * kBufBytes;
          int yl = -1, yr = -1;
          if (stg == 0) x_wraps5(L, P, yl, yr);
          uint32_t tx = 2u * kTileBytes;
          if (stg == 0) tx += (yl >= 0 ? 2u : 0u) * kColBytes + (yr >= 0 ? kColBytes : 0u);
          uint64_t *fb = &full_bar[b][sp];
          mbar_expect_tx(fb, tx);
          tma_2d(bb, spin, 2 * ss, sp * 36, fb);
          tma_2d(bb + kOffW, &maps.W, 2 * ws, wrow + (I * 2 + sp) * 36, fb);
          if (stg == 0) {
            if (yl >= 0) {
              tma_2d(bb + kOffX, spin1, 2 * yl, sp * 36, fb);
              tma_2d(bb + kOffX + kColStride, &maps.W1, 2 * yl, wrow + sp * 36, fb);
            }
            if (yr >= 0) tma_2d(bb + kOffX + 2 * kColStride, spin1, 2 * yr, sp * 36, fb);
          }
          s_issued = i + 1;
        }
        ++k;
      }
      // every issued load lands before the CTA exits: loads before the last
      // kBufs were waited for above
      for (int k = max(0, i - kBufs); k < i; ++k)
        if (!mbar_wait(&full_bar[k % kBufs][k & 1], (uint32_t)((k / kPer) & 1))) {
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
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kConsReg));

  // ---------------------------------------------------------- consumers
  // warp w = 4 kh + 2 sp + h: input-row half kh, species sp, column half h;
  // lane = site of the 32-site unit.  The thread accumulates all six output
  // rows of columns 3h .. 3h + 2 over input rows 3 kh .. 3 kh + 2 of its site
  // and species; after the unit's last stage it keeps rows 3 kh .. 3 kh + 2
  // of the sum (exchange_halves with warp w ^ 4).
  const int kh = warp >> 2, sp = (warp >> 1) & 1, h = warp & 1;
  const int pair_bar = 2 + (warp & 3);  // named barrier of the warp pair (ids 2-5)
  // the thread's first spinor plane and block entries (see nb_products)
  const int pofs = 18 * h + 3 * kh, wofs_f = 3 * kh, wofs_b = 18 * kh;
  const int site_in_unit = lane;
  bool dead = false;

  int it = 0;  // items begun
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    int f, u;
    item(w, f, u);
    if (skip(f)) continue;
    // the item's operator, input and block set (the field's own)
    const BatchField *F = tab + f;
    const CnCoef &Ci = MODE == MV_RHS ? F->CA : F->CH;
    const double nb_sign = MODE == MV_RHS ? -1.0 : 1.0;
    const double2 *in = MODE == MV_RHS ? F->psi : F->x;
    const double2 *Wb = W + (int64_t)F->wblk * 216 * V;
    const cplx ak = Ci.kin[sp], am = Ci.mag[sp], ad = Ci.dar[sp];
    const cplx dg = Ci.dkin * ak + cplx{1.0, 0.0};
    const UnitPos P = unit_pos_of(L, u);
    const int x0 = P.x0;
    const int x = x0 + site_in_unit;
    const bool act = x < V;
    const int xs = act ? x : V - 1;  // a valid site for the addresses of idle lanes
    int nb[6];
    neighbours5(L, P, xs - x0, nb);
    int yl = -1, yr = -1;
    x_wraps5(L, P, yl, yr);
    double acc[6][3][2];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[r][k][0] = acc[r][k][1] = 0.0;
    // the epilogue's operand at the own site: b for the residuals, rh for V,
    // the input itself for RHS and T
    const double2 *epi_src = MODE == MV_RHS ? F->psi : F->b;
    cplx ev[3][3];

#pragma unroll
    for (int stg = 0; stg < kStages; ++stg) {
      const int ld = it * kLoads + stg * 2 + sp;
      const int b = ld % kBufs;
      if (stg == kStages - 2) {
        // the epilogue's operand, loaded into registers two stages ahead
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int k = 0; k < 3; ++k) ev[i][k] = ldg(epi_src + (int64_t)(sp * 36 + (3 * h + k) * 6 + 3 * kh + i) * V + xs);
      }
      int role = -1;
      if (!dead && !wait(&full_bar[b][sp], (uint32_t)((ld / kPer) & 1))) role = 0;
      // stage 0 also reads the unit's diagonal matrices
      if (stg == 0 && !dead && role < 0 && !wait(&dfull[it & 1], (uint32_t)((it >> 1) & 1))) role = 1;
      // warp-uniform: the products below use warp votes
      if (__any_sync(0xffffffffu, role >= 0) && !dead) {
        dead = true;
        if (role >= 0) {
          record_timeout(err, 5, role, ld);
          if (err[3] == (int)blockIdx.x && err[2] == ld) {  // this thread's record: add the detail
            const uint64_t word =
                role == 0 ? *(volatile uint64_t *)&full_bar[b][sp] : *(volatile uint64_t *)&dfull[it & 1];
            err[4] = s_issued + 1;
            err[5] = (int)(uint32_t)word;
            err[6] = (int)(uint32_t)(word >> 32);
            err[7] = role == 0 ? (ld / kPer) & 1 : (it >> 1) & 1;
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
          const unsigned char *dd = smem + kOffDiag + (it & 1) * kDiagStride;
          const uint32_t s_d = smem_u32(dd) + (uint32_t)(site_in_unit * 16);
          const uint32_t s_b = smem_u32(dd + kDiagD) + (uint32_t)(site_in_unit * 8);
          const uint32_t s_own = s_tile + (uint32_t)((site_in_unit + 1) * 16);
          if (kh == 0)
            diag_products<0>(acc, h, s_d, s_b, s_own, ad, am, dg, nb_sign);
          else
            diag_products<1>(acc, h, s_d, s_b, s_own, ad, am, dg, nb_sign);
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
            const uint32_t wst = ww ? 16u : (uint32_t)kTileS * 16u, pst = pw ? 16u : (uint32_t)kTileS * 16u;
            const uint32_t wa = (ww ? xc + kColStride : s_w + (uint32_t)((m - ws) * 16)) +
                                (uint32_t)(bwd ? wofs_b : wofs_f) * wst;
            const uint32_t pa =
                (pw ? xc + (bwd ? 0u : 2u * kColStride) : s_tile + (uint32_t)((y - ss) * 16)) + (uint32_t)pofs * pst;
            auto lw = [&](int e) { return lds_d2(wa + (uint32_t)e * wst); };
            auto lp = [&](int e) { return lds_d2(pa + (uint32_t)e * pst); };
            if (bwd)
              nb_products<true>(acc, lw, lp);
            else
              nb_products<false>(acc, lw, lp);
          } else if (__all_sync(0xffffffffu, (ps && wsh) || !act)) {
            // every operand of the warp in shared memory
            constexpr uint32_t kPl = kTileS * 16u;  // plane stride of the tiles
            const uint32_t wa = s_w + (uint32_t)((m - ws) * 16) + (uint32_t)(bwd ? wofs_b : wofs_f) * kPl;
            const uint32_t pa = s_tile + (uint32_t)((y - ss) * 16) + (uint32_t)pofs * kPl;
            auto lw = [&](int e) { return lds_d2(wa + (uint32_t)e * kPl); };
            auto lp = [&](int e) { return lds_d2(pa + (uint32_t)e * kPl); };
            if (bwd)
              nb_products<true>(acc, lw, lp);
            else
              nb_products<false>(acc, lw, lp);
          } else if (act) {
            // some lanes' operands outside the tiles (periodic wraps, tile
            // edges): those lanes read global memory, the others the tiles
            const int64_t wst = wsh ? kTileS : V, pst = ps ? kTileS : V;
            const double2 *wp = (wsh ? (const double2 *)(bb + kOffW) + (m - ws)
                                     : Wb + (int64_t)((I * 2 + sp) * 36) * V + m) +
                                (bwd ? wofs_b : wofs_f) * wst;
            const double2 *pp = (ps ? (const double2 *)bb + (y - ss) : in + (int64_t)(sp * 36) * V + y) + pofs * pst;
            auto lw = [&](int e) { return wp[e * wst]; };
            auto lp = [&](int e) { return pp[e * pst]; };
            if (bwd)
              nb_products<true>(acc, lw, lp);
            else
              nb_products<false>(acc, lw, lp);
          }
        }
      }
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&empty_bar[b]);
        if (stg == 0) mbar_arrive(&dempty[it & 1]);
      }
    }

    // ---------------------------------------------------------- epilogue
    // every warp of the pair takes both barriers of the exchange, dead or
    // not, active lanes or not
    double res[3][3][2];
    if (kh == 0)
      exchange_halves<0>(acc, res, tbase, warp, pair_bar);
    else
      exchange_halves<1>(acc, res, tbase, warp, pair_bar);
    double qb[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};  // the residual: this item's sums
    if (!dead && act) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int64_t off = (int64_t)(sp * 36 + (3 * h + k) * 6 + 3 * kh + i) * V + x;
          // D in + sgn N in = sgn (sgn D in + N in), sgn = +-1: the diagonal
          // was scaled by sgn and the neighbour sum was not
          const cplx y_ = {nb_sign * res[i][k][0], nb_sign * res[i][k][1]};
          const cplx ev_ = ev[i][k];
          if (MODE == MV_RHS) {
            st(F->b + off, y_);
            st(F->x + off, 2.0 * y_ - ev_);
          } else {
            const cplx rv = ev_ - y_;
            const cplx dv = rv * F->inv_theta[sp];
            F->r32[off] = make_float2((float)rv.re, (float)rv.im);
            F->dA[off] = make_float2((float)dv.re, (float)dv.im);
            qb[k][0] += norm2(rv);
            qb[k][1] += norm2(ev_);
          }
        }
    }
    if (MODE == MV_RESC) {
      // the item's partial row: each column over the lanes, then over the
      // warp pair (the row half kh = 1 hands its sums to kh = 0)
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) qb[k][j] += __shfl_xor_sync(0xffffffffu, qb[k][j], o);
      if (kh == 1 && lane == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int j = 0; j < 2; ++j) redb[it & 1][sp][h][k][j] = qb[k][j];
      named_bar_sync(pair_bar, 64);
      if (kh == 0 && lane < 6 && !dead) {
        double v = 0.0;
#pragma unroll
        for (int t = 0; t < 6; ++t)
          if (t == lane) v = qb[t >> 1][t & 1];
        const int k = lane >> 1, j = lane & 1;
        F->partials[((int64_t)u * CN_COLS + sp * 6 + 3 * h + k) * 2 + j] = v + redb[it & 1][sp][h][k][j];
      }
    }
    ++it;
  }

  // every consumer warp is done with the tensor memory before warp 0 frees it
  tc::fence_before_sync();
  named_bar_sync(1, kWarps * 32);
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tbase, kTmemCols);
}

// ------------------------------------------------------------------ host
void launch_cn_blocks5(Lat L, const CnCoef &C, const double2 *U, const double2 *DE, double2 *W, float2 *Wf,
                       cudaStream_t st) {
  const int64_t n = 9 * L.V;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (W && Wf)
    k_cn_blocks5<true, true><<<grid, 256, 0, st>>>(L, C, U, DE, W, Wf);
  else if (W)
    k_cn_blocks5<true, false><<<grid, 256, 0, st>>>(L, C, U, DE, W, Wf);
  else if (Wf)
    k_cn_blocks5<false, true><<<grid, 256, 0, st>>>(L, C, U, DE, W, Wf);
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
    case MV_T2: go(k_cn_mv5<MV_T2>); break;
    case MV_RES2: go(k_cn_mv5<MV_RES2>); break;
    case MV_V2: go(k_cn_mv5<MV_V2>); break;
    default: go(k_cn_mv5<MV_T>); break;
  }
  return 0;
}


bool batch_mv5_applicable(const Lat &L) { return L.V >= mv5::kTileS && L.V <= 0x7fffffffLL && (L.V & 1) == 0; }

bool batch_mv5_field_maps(CnBatchMaps *m, const Lat &L, const double2 *psi, const double2 *x) {
  using namespace mv5;
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
  using namespace mv5;
  if (!batch_mv5_applicable(L) || nfields <= 0 || order < 0 || order > 1 || (mode != MV_RHS && mode != MV_RESC))
    return -1;
  const int64_t nunits = cn_mv5_units(L.V);
  if (nunits * nfields > 0x7fffffffLL) return -1;
  const uint64_t V = (uint64_t)L.V;
  Mv5Maps maps;  // the fields' spinor maps come from fmaps
  memset(&maps, 0, sizeof(maps));
  if (!stage::encode(&maps.W, W, 2 * V, 216ull * nblk, 2 * kTileS, 36) ||
      !stage::encode(&maps.W1, W, 2 * V, 216ull * nblk, 2, 36) || !stage::encode(&maps.D, Dsum, 2 * V, 9, 2 * kUnit, 9) ||
      !stage::encode(&maps.B, Bsum, V, 9, kUnit, 9))
    return -1;
  const unsigned grid = (unsigned)std::min<int64_t>(nunits * nfields, sm_count);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    kern<<<grid, kThreads, kSmemBytes, st>>>(L, maps, W, (int)nunits, err, wait_cycles, tab, fmaps, nfields, order,
                                            skip_done);
  };
  if (mode == MV_RHS)
    go(k_batch_mv5<MV_RHS>);
  else
    go(k_batch_mv5<MV_RESC>);
  return 0;
}

}  // namespace nrq
