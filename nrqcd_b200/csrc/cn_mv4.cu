// Tensor-core FP64 stencil of the assembled Crank-Nicolson operator
// (src/nrqcd.f90:1175-1387 with PETSc's block transposition; the operator
// is described in cn.cu).  out = D in + sum over the 6 neighbours of the
// 6x6 spin-colour blocks applied to the 6 propagator columns, both species.
//
// Blocks.  Once per update, k_cn_blocks writes the forward block of every
// site, direction and species (the operator's coefficients folded in):
//   W_I(x) = ck (U_I(x)^T x 1) + cs0 (DE_I0(x)^T x s_K0^T) + cs1 (DE_I1(x)^T x s_K1^T)
// With real Wilson coefficients every alpha_t is imaginary and every G_t
// hermitian, so the backward block is W_back(x) = -W_I(x-I)^H; the kernel
// reads it from the forward block of x-I (index transposed, signs flipped)
// and needs no second copy.  A^H differs from A only by conj(alpha_t) =
// -alpha_t: one set of blocks serves both with a sign on the neighbour sum.
//
// Products.  Per site, species and neighbour, out(6 x 6 cols) += W(6x6) in:
// as a real GEMM, M = 16 (re rows 0-5, im rows 8-13 of the 6 output rows),
// N = 8 (6 columns), K = 12 (re/im of the 6 input rows), three
// mma.sync.m16n8k4 FP64 steps.  A lane's A fragment is one complex entry of
// W (x1 or xi), its B fragment the real or imaginary part of one spinor
// entry, its C fragment two complex outputs.  The FP64 tensor pipe has the
// DFMA peak on B200 but one instruction carries 512 FMAs, which frees issue
// slots for the loads the register-tiled stencils stall on.
//
// Pipeline.  Persistent, one CTA per SM: 16 consumer warps (one site of the
// unit each) and one producer warp.  A work unit is 16 sites (x0 = 16u);
// five stages per unit, stage s in shared-memory buffer s (TMA tiles for the
// spinors, bulk copies for the blocks, completion on mbarriers): stage 0 =
// diagonal, +x, -x; 1 = +y; 2 = -y; 3 = +z; 4 = -z.  The producer issues
// each buffer's next stage as soon as every consumer released it.  A site
// whose neighbour (periodic wrap) or neighbour block lies outside the stage's
// tiles reads it from global memory (warp-uniform).  Results go through an
// epilogue tile in buffer 4 (128-byte swizzle): each warp writes its site's
// column, the producer stores the tile with TMA once all warps released the
// buffer.  The residual and dot-product partial sums stay in registers over
// all units of the CTA: one partial row per CTA.
//
// Every mbarrier wait is bounded (about two seconds); on expiry the thread
// records NRQ_ERR_TIMEOUT in *err and skips the remaining work without
// leaving a barrier unmatched; the producer waits (bounded) for its copies in
// flight before the CTA exits.  Single-GPU code: no load uses cluster
// multicast.
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "../../include/nrqcd_b200.h"
#include "nrq_kernels.cuh"
#include "stage.cuh"

// sites per consumer warp of the tensor-core stencil (1: 16 consumer warps
// with two MMA chains each; 2: 8 consumer warps with four)
#ifndef NRQ_MV4_SPW
#define NRQ_MV4_SPW 1
#endif
// K = 12 of a block product as one m16n8k8 and one m16n8k4 MMA (1), or as
// three m16n8k4 MMAs (0)
#ifndef NRQ_MV4_K8
#define NRQ_MV4_K8 1
#endif

namespace nrq {

namespace mv4 {
constexpr int kUnit = 16;                 // sites per work unit
constexpr int kTileS = 19;                // spinor tile width in sites (odd stride in 16-byte words)
constexpr int kStages = 5;                // stages per unit; stage s always uses buffer s
constexpr int kSPW = NRQ_MV4_SPW;         // sites per consumer warp
constexpr int kWarps = kUnit / kSPW;      // consumer warps
constexpr int kThreads = (kWarps + 1) * 32;  // + one producer warp
// registers per thread: the SM quarter that hosts the most warps of the CTA
// (ceil((kWarps + 1) / 4)) holds 16384 registers
constexpr int kMaxReg = kSPW == 1 ? 96 : 168;
static_assert(kUnit % kSPW == 0 && ((kWarps + 4) / 4) * 32 * kMaxReg <= 16384, "warp layout");
constexpr int kBlk = 36;                  // complex entries of one 6x6 block
constexpr int kBlkBytes = kBlk * 16;      // 576
constexpr int kWMax = kUnit + 1;          // blocks per species and stage (stage 0: x0-1 .. x0+15)
constexpr int kWSpecies0 = kWMax * kBlkBytes;  // 9792: species stride of stage 0's block tile
constexpr int kWSpecies = kUnit * kBlkBytes;   // 9216: species stride of stages 1-4
constexpr uint32_t kSpinBytes = 72 * kTileS * 16;  // 21888
// Buffer layout (byte offsets from the 1024-aligned base).  Buffer 4 first:
// spinors, blocks, then the epilogue tile (operand b or rh in, the result
// out; two 128-byte-swizzled halves of 8 sites x 72 planes, 1024-aligned).
// Buffer 0: spinors, blocks, Darwin and magnetic matrices.  Buffers 1-3:
// spinors and blocks.
constexpr int kEpiHalf = 72 * 128;                     // 9216
constexpr int kBuf4 = 0, kOffEpi = 40960;              // buffer 4: spin 0, blocks 22528, epilogue 40960
constexpr int kBuf0 = kOffEpi + 2 * kEpiHalf;          // 59392
constexpr int kOffD = kSpinBytes + 2 * kWSpecies0;     // buffer 0: 41472 (9 x 16 x 16 = 2304)
constexpr int kOffB = kOffD + 2304;                    // 43776 (9 x 16 x 8 = 1152)
constexpr int kBuf1 = kBuf0 + kOffB + 1152;            // 104320
constexpr int kBufPlain = kSpinBytes + 2 * kUnit * kBlkBytes;  // 40320: buffers 1-3
constexpr int kSmemBytes = kBuf1 + 3 * kBufPlain + 1024;       // 226304 + alignment slack
__host__ __device__ constexpr int buf_off(int s) {
  return s == 4 ? kBuf4 : s == 0 ? kBuf0 : kBuf1 + (s - 1) * kBufPlain;
}
__host__ __device__ constexpr int w_off(int s) { return s == 4 ? 22528 : (int)kSpinBytes; }
__host__ __device__ constexpr int w_species(int s) { return s == 0 ? kWSpecies0 : kWSpecies; }
static_assert(kBuf0 % 128 == 0 && kBuf1 % 128 == 0 && kBufPlain % 128 == 0 && kOffD % 128 == 0 &&
                  kOffB % 128 == 0 && kOffEpi % 1024 == 0 && 22528 >= (int)kSpinBytes &&
                  22528 + 2 * kWSpecies <= kOffEpi && kBufPlain == (int)kSpinBytes + 2 * kWSpecies &&
                  kBuf0 + kOffB + 1152 <= kBuf1 && kBuf1 + 3 * kBufPlain + 1024 <= kSmemBytes,
              "buffer layout");
}  // namespace mv4

struct Mv4Maps {
  CUtensorMap spin;    // 72 planes x 2V doubles, box {38, 72}
  CUtensorMap D;       // 9 planes x 2V doubles, box {32, 9}
  CUtensorMap B;       // 9 planes x V doubles, box {16, 9}
  CUtensorMap epi_in;  // epilogue operand (b or rh), box {16, 72}, 128-byte swizzle
  CUtensorMap out[3];  // results stored from the epilogue tile, same boxes
};

// entry (s, t) of s_k^T for the reference Pauli matrices (src/su2.f90:68-79
// holds s_2 transposed, so s_2^T = [[0,-i],[i,0]])
__device__ __forceinline__ cplx pauli_t(int k, int s, int t) {
  if (k == 0) return (s != t) ? cplx{1.0, 0.0} : cplx{0.0, 0.0};
  if (k == 1) {
    if (s == 0 && t == 1) return {0.0, -1.0};
    if (s == 1 && t == 0) return {0.0, 1.0};
    return {0.0, 0.0};
  }
  if (s != t) return {0.0, 0.0};
  return (s == 0) ? cplx{1.0, 0.0} : cplx{-1.0, 0.0};
}

// storage slot of entry (row g, column q) inside a 6x6 block: the entries a
// lane group reads in one MMA step (q in {2j, 2j+1}, all rows) are adjacent
__host__ __device__ __forceinline__ int blk_slot(int g, int q) { return ((q >> 1) * 6 + g) * 2 + (q & 1); }

// One thread per (direction I, species, site, output row g): row g of the
// forward block W_I(x) of that species.  Layout: block (I*2 + sp)*V + x.
__global__ void __launch_bounds__(256) k_cn_blocks(Lat L, CnCoef C, const double2 *__restrict__ U,
                                                   const double2 *__restrict__ DE, double2 *__restrict__ W) {
  const int64_t V = L.V;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 36 * V) return;
  const int g = (int)(tid % 6);
  const int64_t r = tid / 6;  // (I*2 + sp)*V + x
  const int64_t x = r % V;
  const int isp = (int)(r / V);
  const int I = isp >> 1, sp = isp & 1;
  const int c = g >> 1, s = g & 1;
  const int K0 = (I + 2) % 3, K1 = (I + 1) % 3;
  const cplx ck = (-0.5 * C.inva2[I]) * C.kin[sp];
  const cplx cs0 = times_i(C.so[sp]), cs1 = -times_i(C.so[sp]);
  double2 *blk = W + r * mv4::kBlk;
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
      v = v + pauli_t(K0, s, t) * e0 + pauli_t(K1, s, t) * e1;
      st(blk + blk_slot(g, 2 * cp + t), v);
    }
  }
}

// D(16x8) += A(16x4) B(4x8), FP64 tensor cores
__device__ __forceinline__ void dmma(double (&d)[4], double a0, double a1, double b0) {
  asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}
// D(16x8) += A(16x8) B(8x8): the two k4 steps j, j+1 in one instruction
// (a0, a1 the A fragment of step j, a2, a3 that of step j+1; b0, b1 the B
// fragments of the two steps)
__device__ __forceinline__ void dmma8(double (&d)[4], double a0, double a1, double a2, double a3, double b0,
                                      double b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}
// sign flip by an XOR on the high word (m = 0 or the sign bit)
__device__ __forceinline__ double flip(double v, unsigned m) {
  return __hiloint2double(__double2hiint(v) ^ (int)m, __double2loint(v));
}
constexpr unsigned kSign = 0x80000000u;
// shared-memory load at a register address plus a compile-time offset
template <int OFF>
__device__ __forceinline__ double lds_at(uint32_t a) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1+%2];" : "=d"(v) : "r"(a), "n"(OFF));
  return v;
}

// 32-bit coordinates and neighbours (the stencil runs for V < 2^31 only)
__device__ __forceinline__ void coords32(const Lat &L, uint32_t s, uint32_t &x, uint32_t &y, uint32_t &z) {
  const uint32_t nx = (uint32_t)L.nx, ny = (uint32_t)L.ny;
  const uint32_t t = s / nx;
  x = s - t * nx;
  z = t / ny;
  y = t - z * ny;
}
__device__ __forceinline__ int nb32(const Lat &L, uint32_t s, int d, int sgn) {
  uint32_t x, y, z;
  coords32(L, s, x, y, z);
  const uint32_t nx = (uint32_t)L.nx, ny = (uint32_t)L.ny, nz = (uint32_t)L.nz;
  if (d == 0) x = sgn > 0 ? (x + 1 == nx ? 0 : x + 1) : (x == 0 ? nx - 1 : x - 1);
  else if (d == 1) y = sgn > 0 ? (y + 1 == ny ? 0 : y + 1) : (y == 0 ? ny - 1 : y - 1);
  else z = sgn > 0 ? (z + 1 == nz ? 0 : z + 1) : (z == 0 ? nz - 1 : z - 1);
  return (int)((z * ny + y) * nx + x);
}
// first sites of the spinor tiles of the five stages of the unit at x0
// (stage 0: x0 - 1; stages 1-4: the +y, -y, +z, -z neighbours of x0), from
// one coordinate decomposition
__device__ __forceinline__ void mv4_spin_starts(const Lat &L, int x0, int ss[5]) {
  uint32_t cx, cy, cz;
  coords32(L, (uint32_t)x0, cx, cy, cz);
  (void)cx;
  const int ny = (int)L.ny, nz = (int)L.nz, row = (int)L.nx, plane = (int)(L.nx * L.ny);
  ss[0] = x0 - 1;
  ss[1] = (int)cy + 1 < ny ? x0 + row : x0 - (ny - 1) * row;
  ss[2] = cy > 0 ? x0 - row : x0 + (ny - 1) * row;
  ss[3] = (int)cz + 1 < nz ? x0 + plane : x0 - (nz - 1) * plane;
  ss[4] = cz > 0 ? x0 - plane : x0 + (nz - 1) * plane;
}
// first block of the block tiles of stage st (forward stages: the unit
// itself; backward stages: the unit's neighbours; stage 0 covers both)
__device__ __forceinline__ int mv4_blk_start(int x0, int spin_start, int st) {
  if (st == 0) return x0 > 0 ? x0 - 1 : 0;
  if (st == 1 || st == 3) return x0;
  return spin_start;
}
__device__ __forceinline__ int mv4_blk_count(int V, int start, int st) {
  const int want = st == 0 ? mv4::kWMax : mv4::kUnit;
  return min(want, V - start);
}

// Operands of step J of a neighbour with every operand in the stage's
// shared tiles: wa0/wa1 = the lane's A-fragment addresses (block of species
// 0), sb = its B-fragment address (species 0); the step and the species add
// compile-time offsets.
template <bool BWD, int SA, int J>
__device__ __forceinline__ void nb_fast_load(double (&a0)[2], double (&a1)[2], double (&b0)[2], uint32_t wa0,
                                             uint32_t wa1, uint32_t sb) {
  constexpr int oA = J * (BWD ? 64 : 192), sA = SA;
  constexpr int oB = J * 2 * mv4::kTileS * 16, sB = 36 * mv4::kTileS * 16;
  a0[0] = lds_at<oA>(wa0);
  a0[1] = lds_at<oA + sA>(wa0);
  a1[0] = lds_at<oA>(wa1);
  a1[1] = lds_at<oA + sA>(wa1);
  b0[0] = lds_at<oB>(sb);
  b0[1] = lds_at<oB + sB>(sb);
}
// a whole neighbour of the warp's N sites: all operands loaded, then 6N
// MMAs in 2N independent chains (site x species); SA = species stride of the
// block tile
template <bool BWD, int SA, int N>
__device__ __forceinline__ void nb_fast(double (&acc)[N][2][4], const uint32_t (&wa0)[N], const uint32_t (&wa1)[N],
                                        const uint32_t (&sb)[N], unsigned m0, unsigned m1) {
  double a0[3][N][2], a1[3][N][2], b0[3][N][2];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    nb_fast_load<BWD, SA, 0>(a0[0][i], a1[0][i], b0[0][i], wa0[i], wa1[i], sb[i]);
    nb_fast_load<BWD, SA, 1>(a0[1][i], a1[1][i], b0[1][i], wa0[i], wa1[i], sb[i]);
    nb_fast_load<BWD, SA, 2>(a0[2][i], a1[2][i], b0[2][i], wa0[i], wa1[i], sb[i]);
  }
#if NRQ_MV4_K8
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int sp = 0; sp < 2; ++sp)
      dmma8(acc[i][sp], flip(a0[0][i][sp], m0), flip(a1[0][i][sp], m1), flip(a0[1][i][sp], m0),
            flip(a1[1][i][sp], m1), b0[0][i][sp], b0[1][i][sp]);
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int sp = 0; sp < 2; ++sp) dmma(acc[i][sp], flip(a0[2][i][sp], m0), flip(a1[2][i][sp], m1), b0[2][i][sp]);
#else
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int sp = 0; sp < 2; ++sp)
        dmma(acc[i][sp], flip(a0[j][i][sp], m0), flip(a1[j][i][sp], m1), b0[j][i][sp]);
#endif
}

// results of a mode stored from the epilogue tiles (RES: r, rh and p are the
// same values; RESC: the FP32 r and r/theta, two FP32 tiles in buffer 4's
// block region) and whether an epilogue operand arrives in the FP64 tile (b
// for RES and RESC, rh for V, the input itself for T and RHS)
__host__ __device__ constexpr int mv4_tile_outputs(int mode) {
  return mode == MV_RES ? 3 : (mode == MV_RESC ? 2 : 1);
}
__host__ __device__ constexpr bool mv4_tile_input(int mode) { return mode != MV_PLAIN; }
// byte offset of (plane p, site l) in the epilogue tile: two halves of 8
// sites, rows of 128 bytes, 16-byte chunks swizzled with the row (the
// 128-byte swizzle of the tensor maps; the tile is 1024-aligned)
__device__ __forceinline__ uint32_t epi_off(int p, int l) {
  return (uint32_t)((l >> 3) * mv4::kEpiHalf + p * 128 + (((l & 7) ^ (p & 7)) << 4));
}
// byte offset of (plane p, site l) in an FP32 result tile: rows of 16 sites
// x 8 bytes, 16-byte chunks swizzled with the row (1024-aligned tile)
__device__ __forceinline__ uint32_t epi32_off(int p, int l) {
  return (uint32_t)(p * 128 + ((((l >> 1) ^ (p & 7))) << 4) + ((l & 1) << 3));
}
constexpr int kOffF32 = 22528;  // FP32 result tiles of RESC in buffer 4 (its block region, after stage 4)

template <int MODE>
__global__ void __maxnreg__(mv4::kMaxReg)
    k_cn_mv4(Lat L, CnCoef C, double nb_sign, const __grid_constant__ Mv4Maps maps, const double2 *__restrict__ W,
             const double2 *__restrict__ Dsum, const double *__restrict__ Bsum, MvArgs A, int64_t nunits, int *err) {
  using namespace mv4;
  constexpr int kNOut = mv4_tile_outputs(MODE);
  constexpr bool kIn = mv4_tile_input(MODE);
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages];
  // per-warp partial sums of the CTA (one partial row per CTA, at the end)
  __shared__ double red[kWarps][CN_COLS][3];
  // per warp and unit: neighbours (+x,-x,+y,-y,+z,-z) of its sites (entries
  // 6i .. 6i+5 for site i) and the spinor tile starts of stages 1-4 (last 4)
  constexpr int kNbt = 6 * kSPW + 4;
  __shared__ int nbt[kWarps][kNbt];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t V = L.V;
  const int V32 = (int)V;  // the launcher admits V < 2^31 only

  if (threadIdx.x == 0) {
    for (int b = 0; b < kStages; ++b) {
      mbar_init(&full_bar[b], 1);
      mbar_init(&empty_bar[b], kWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // ---- producer: lane 0 of warp kWarps issues the stages of this CTA's
  // units in order, as far ahead as the buffers allow.  Before refilling
  // buffer 4 it stores the previous unit's results from the epilogue tile.
  const int nu = (int)nunits;
  const int my_units = (nu - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int total = my_units * kStages;
  int issued = 0;
  int p_unit = (int)blockIdx.x, p_stg = 0;
  uint32_t p_par = 0;                // empty-barrier parity of the previous use of a buffer
  int pss[5] = {0, 0, 0, 0, 0};      // tile starts of p_unit
  auto store_results = [&](int x0) {
    if (MODE == MV_RESC) {
#pragma unroll
      for (int o = 0; o < 2; ++o) tma_store_2d(&maps.out[o], 2 * x0, 0, smem + kBuf4 + kOffF32 + o * kEpiHalf);
    } else {
#pragma unroll
      for (int o = 0; o < kNOut; ++o)
#pragma unroll
        for (int hf = 0; hf < 2; ++hf)
          tma_store_2d(&maps.out[o], 2 * x0 + 16 * hf, 0, smem + kBuf4 + kOffEpi + hf * kEpiHalf);
    }
    bulk_commit();
  };
  auto issue = [&]() {
    const int stg = p_stg;
    if (issued >= kStages && !mbar_wait(&empty_bar[stg], p_par)) return false;
    const int x0 = p_unit * kUnit;
    if (stg == 0) mv4_spin_starts(L, x0, pss);
    unsigned char *bb = smem + buf_off(stg);
    if (stg == kStages - 1 && kNOut > 0 && issued >= kStages) {
      // the previous unit's results must leave the tile before new operands land in it
      store_results(x0 - (int)gridDim.x * kUnit);
      bulk_wait_read_all();
    }
    const int I = (stg == 0) ? 0 : (stg + 1) / 2;
    // stage start without a dynamically indexed (local-memory) array
    const int sst = stg == 0 ? pss[0] : stg == 1 ? pss[1] : stg == 2 ? pss[2] : stg == 3 ? pss[3] : pss[4];
    const int ws = mv4_blk_start(x0, sst, stg);
    const int wn = mv4_blk_count(V32, ws, stg);
    uint32_t tx = kSpinBytes + 2u * (uint32_t)wn * kBlkBytes;
    if (stg == 0) tx += 2304 + 1152;
    if (stg == kStages - 1 && kIn) tx += 2 * kEpiHalf;
    mbar_expect_tx(&full_bar[stg], tx);
    tma_2d(bb, &maps.spin, 2 * sst, 0, &full_bar[stg]);
#pragma unroll
    for (int sp = 0; sp < 2; ++sp)
      bulk_1d(bb + w_off(stg) + sp * w_species(stg), W + ((int64_t)(I * 2 + sp) * V + ws) * kBlk,
              (uint32_t)wn * kBlkBytes, &full_bar[stg]);
    if (stg == 0) {
      tma_2d(bb + kOffD, &maps.D, 2 * x0, 0, &full_bar[stg]);
      tma_2d(bb + kOffB, &maps.B, x0, 0, &full_bar[stg]);
    }
    if (stg == kStages - 1 && kIn) {
      tma_2d(bb + kOffEpi, &maps.epi_in, 2 * x0, 0, &full_bar[stg]);
      tma_2d(bb + kOffEpi + kEpiHalf, &maps.epi_in, 2 * x0 + 16, 0, &full_bar[stg]);
    }
    if (++p_stg == kStages) {
      p_stg = 0;
      p_unit += (int)gridDim.x;
      if (issued >= kStages) p_par ^= 1u;
    }
    return true;
  };
  bool dead = false;
  if (warp == kWarps) {
    if (lane == 0) {
      bool ok = true;
      for (; issued < total && ok; ++issued) ok = issue();
      if (ok && kNOut > 0 && my_units > 0) {
        // the last unit's results: every warp released buffer 4 after its epilogue
        ok = mbar_wait(&empty_bar[kStages - 1], (uint32_t)((my_units - 1) & 1));
        if (ok) store_results(((int)blockIdx.x + (my_units - 1) * (int)gridDim.x) * kUnit);
      }
      if (!ok) record_timeout(err, 4, 0, -1);
      bulk_wait_all();
      // error path: copies issued ahead of the consumers must land before
      // exit (the last use of each buffer; earlier uses were consumed)
      if (!ok)
        for (int kk = issued > kStages ? issued - kStages : 0; kk < issued; ++kk)
          if (!mbar_wait(&full_bar[kk % kStages], (uint32_t)((kk / kStages) & 1))) break;
    }
  }
  uint32_t c_par = 0;  // consumers: full-barrier parity of the current unit
  auto stage_begin = [&](int stg) -> const unsigned char * {
    if (!dead && !mbar_wait(&full_bar[stg], c_par)) {
      dead = true;
      record_timeout(err, 4, 0, -1);
    }
    return smem + buf_off(stg);
  };
  auto stage_end = [&](int stg) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty_bar[stg]);
  };

  // ---- lane roles in the MMA fragments
  const int g = lane >> 2, kq = lane & 3;
  const int gc = g < 6 ? g : 5;       // rows 6, 7 are padding (any finite data)
  const int part = kq & 1, h = kq >> 1;
  const bool out_lane = g < 6 && kq < 3;  // owns output rows g, columns 2kq, 2kq+1
  const unsigned nbm = nb_sign < 0.0 ? kSign : 0u;
  // A fragments: component byte offsets and sign masks (forward, backward)
  const uint32_t ca0 = (uint32_t)part * 8u, ca1 = (uint32_t)(1 - part) * 8u;
  const unsigned mf0 = (part ? kSign : 0u) ^ nbm, mf1 = nbm;
  const unsigned mb0 = kSign ^ nbm, mb1 = (part ? kSign : 0u) ^ nbm;
  // lane byte offsets of step 0, species 0: A inside a block (forward and
  // backward = transposed entry), B inside a spinor tile column
  const uint32_t offAf = (uint32_t)(2 * gc + h) * 16u, offAb = (uint32_t)((gc >> 1) * 12 + 2 * h + (gc & 1)) * 16u;
  const uint32_t offB = (uint32_t)((gc * 6 + h) * kTileS * 16) + (uint32_t)part * 8u;

  double acc[kSPW][2][4];  // [site][species][C fragment] of the warp's sites

  // general path of one neighbour of one site: block and spinor each in the
  // stage's shared tiles or in global memory (periodic wraps, tile edges)
  auto nb_general = [&](double (&ac)[2][4], bool bwd, int wspec, bool wsh, uint32_t wsa, const double2 *wg, bool ssh,
                        uint32_t ssa, const double2 *sg) {
#pragma unroll
    for (int sp = 0; sp < 2; ++sp) {
      double a0[3], a1[3], b0[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int q = 2 * j + h;
        const int sl = bwd ? blk_slot(q, gc) : blk_slot(gc, q);
        const int pl = gc * 6 + q;  // spinor plane in the species: column n = gc, row q
        if (wsh) {
          const uint32_t ea = wsa + (uint32_t)(sp * wspec + sl * 16);
          a0[j] = lds1(ea + ca0);
          a1[j] = lds1(ea + ca1);
        } else {
          const double *ep = (const double *)(wg + (int64_t)sp * V * kBlk + sl);
          a0[j] = __ldg(ep + part);
          a1[j] = __ldg(ep + 1 - part);
        }
        if (ssh)
          b0[j] = lds1(ssa + (uint32_t)(((sp * 36 + pl) * kTileS) * 16) + (uint32_t)part * 8u);
        else
          b0[j] = __ldg((const double *)(sg + (int64_t)(sp * 36 + pl) * V) + part);
      }
      const unsigned g0 = bwd ? mb0 : mf0, g1 = bwd ? mb1 : mf1;
#if NRQ_MV4_K8
      dmma8(ac[sp], flip(a0[0], g0), flip(a1[0], g1), flip(a0[1], g0), flip(a1[1], g1), b0[0], b0[1]);
      dmma(ac[sp], flip(a0[2], g0), flip(a1[2], g1), b0[2]);
#else
#pragma unroll
      for (int j = 0; j < 3; ++j) dmma(ac[sp], flip(a0[j], g0), flip(a1[j], g1), b0[j]);
#endif
    }
  };
  // one neighbour (direction I, forward or backward) of the warp's sites:
  // m[i] = site of the forward block, y[i] = neighbour site; the tiles start
  // at block ws (wn blocks) and spinor site ss.  All operands in the tiles:
  // the fast path for every site at once; otherwise site by site.
  auto neighbour = [&](auto BWDc, auto SAc, int I, uint32_t sw, uint32_t sspin, int ws, int wn, int ss,
                       const int (&m)[kSPW], const int (&y)[kSPW], const bool (&act)[kSPW]) {
    constexpr bool BWD = decltype(BWDc)::value;
    constexpr int SA = decltype(SAc)::value;
    int wi[kSPW], si[kSPW];
    bool fast = true;
#pragma unroll
    for (int i = 0; i < kSPW; ++i) {
      wi[i] = m[i] - ws;
      si[i] = y[i] - ss;
      fast = fast && act[i] && (unsigned)wi[i] < (unsigned)wn && (unsigned)si[i] < (unsigned)kTileS;
    }
    if (fast) {
      uint32_t wa0[kSPW], wa1[kSPW], sb[kSPW];
#pragma unroll
      for (int i = 0; i < kSPW; ++i) {
        const uint32_t blk = sw + (uint32_t)wi[i] * kBlkBytes + (BWD ? offAb : offAf);
        wa0[i] = blk + ca0;
        wa1[i] = blk + ca1;
        sb[i] = sspin + (uint32_t)si[i] * 16u + offB;
      }
      nb_fast<BWD, SA, kSPW>(acc, wa0, wa1, sb, BWD ? mb0 : mf0, BWD ? mb1 : mf1);
    } else {
#pragma unroll
      for (int i = 0; i < kSPW; ++i) {
        if (!act[i]) continue;
        const bool wsh = (unsigned)wi[i] < (unsigned)wn, ssh = (unsigned)si[i] < (unsigned)kTileS;
        nb_general(acc[i], BWD, SA, wsh, sw + (uint32_t)((wsh ? wi[i] : 0) * kBlkBytes),
                   W + ((int64_t)(I * 2) * V + m[i]) * kBlk, ssh, sspin + (uint32_t)((ssh ? si[i] : 0) * 16),
                   A.in + y[i]);
      }
    }
  };
  using S0 = std::integral_constant<int, kWSpecies0>;
  using S1 = std::integral_constant<int, kWSpecies>;
  using F = std::integral_constant<bool, false>;
  using T = std::integral_constant<bool, true>;

  constexpr int NQ = (MODE == MV_T) ? 3 : ((MODE == MV_RES || MODE == MV_V || MODE == MV_RESC) ? 2 : 0);
  // the lane's partial sums over every unit of this CTA: [species][column e][quantity]
  double qs[2][2][3];
#pragma unroll
  for (int sp = 0; sp < 2; ++sp)
#pragma unroll
    for (int e = 0; e < 2; ++e) qs[sp][e][0] = qs[sp][e][1] = qs[sp][e][2] = 0.0;

  for (int u = (int)blockIdx.x; u < nu && warp < kWarps; u += (int)gridDim.x) {
    const int x0 = u * kUnit;
    int xs[kSPW];
    bool act[kSPW];
#pragma unroll
    for (int i = 0; i < kSPW; ++i) {
      xs[i] = x0 + warp * kSPW + i;
      act[i] = xs[i] < V32;
    }
    // neighbour table, one entry per lane (the previous unit's reads ended
    // at its last stage_end): lanes 0 .. 6 kSPW - 1 the sites' neighbours,
    // the next 4 lanes the tile starts of stages 1-4
    if (lane < kNbt) {
      int v = 0;
      if (lane < 6 * kSPW) {
        const int xi = x0 + warp * kSPW + lane / 6, d = lane % 6;
        if (xi < V32) v = nb32(L, (uint32_t)xi, d >> 1, (d & 1) ? -1 : +1);
      } else {
        const int st = lane - 6 * kSPW + 1;  // 1..4
        v = nb32(L, (uint32_t)x0, (st + 1) >> 1, (st & 1) ? +1 : -1);
      }
      nbt[warp][lane] = v;
    }
    __syncwarp();
    const int *nbw = nbt[warp];
#pragma unroll
    for (int i = 0; i < kSPW; ++i)
#pragma unroll
      for (int sp = 0; sp < 2; ++sp)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][sp][e] = 0.0;

    // ---------------------------------------------------------- stage 0
    {
      const unsigned char *b = stage_begin(0);
      if (!dead && act[0]) {
        const int ss = x0 - 1, ws = mv4_blk_start(x0, ss, 0);
        const int wn = mv4_blk_count(V32, ws, 0);
        const uint32_t sspin = smem_u32(b), sw = smem_u32(b + w_off(0));
        const uint32_t sD = smem_u32(b + kOffD), sB = smem_u32(b + kOffB);
        // diagonal block (colour only): A = delta_st Cd_c[cp], centre spinor
#pragma unroll
        for (int i = 0; i < kSPW; ++i) {
          if (!act[i]) continue;
          const int l = warp * kSPW + i;
          const int c = gc >> 1, s = gc & 1;
          cplx dv[3];
          double bv[3];
#pragma unroll
          for (int j = 0; j < 3; ++j) {  // j = cp, input spin t = h
            const int e = j * 3 + c;
            dv[j] = lds2(sD + (uint32_t)((e * kUnit + l) * 16));
            bv[j] = lds1(sB + (uint32_t)((e * kUnit + l) * 8));
          }
          const uint32_t sbc = sspin + (uint32_t)(l + 1) * 16u + offB;
#pragma unroll
          for (int sp = 0; sp < 2; ++sp) {
            const cplx ak = C.kin[sp], am = C.mag[sp], ad = C.dar[sp];
            const cplx dg = C.dkin * ak + cplx{1.0, 0.0};
            const uint32_t sbs = sbc + (uint32_t)(sp * 36 * kTileS * 16);
            double b0[3];
            b0[0] = lds_at<0>(sbs);
            b0[1] = lds_at<2 * kTileS * 16>(sbs);
            b0[2] = lds_at<4 * kTileS * 16>(sbs);
            double da0[3], da1[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              cplx cd = ad * dv[j] + bv[j] * am;
              if (j == c) cd = cd + dg;
              if (s != h) cd = cplx{0.0, 0.0};
              da0[j] = part ? -cd.im : cd.re;
              da1[j] = part ? cd.re : cd.im;
            }
#if NRQ_MV4_K8
            dmma8(acc[i][sp], da0[0], da1[0], da0[1], da1[1], b0[0], b0[1]);
            dmma(acc[i][sp], da0[2], da1[2], b0[2]);
#else
#pragma unroll
            for (int j = 0; j < 3; ++j) dmma(acc[i][sp], da0[j], da1[j], b0[j]);
#endif
          }
        }
        // +x: block at x (forward), spinor at x+1; -x: block and spinor at x-1
        int yp[kSPW], ym[kSPW];
#pragma unroll
        for (int i = 0; i < kSPW; ++i) {
          yp[i] = nbw[6 * i + 0];
          ym[i] = nbw[6 * i + 1];
        }
        neighbour(F{}, S0{}, 0, sw, sspin, ws, wn, ss, xs, yp, act);
        neighbour(T{}, S0{}, 0, sw, sspin, ws, wn, ss, ym, ym, act);
      }
      stage_end(0);
    }
    // ------------------------------------------------------- stages 1-4
#pragma unroll
    for (int stg = 1; stg < kStages; ++stg) {
      const unsigned char *b = stage_begin(stg);
      if (!dead && act[0]) {
        const int I = (stg + 1) / 2;
        const int ss = nbw[6 * kSPW - 1 + stg], ws = mv4_blk_start(x0, ss, stg);
        const int wn = mv4_blk_count(V32, ws, stg);
        const uint32_t sspin = smem_u32(b), sw = smem_u32(b + w_off(stg));
        int y[kSPW];
#pragma unroll
        for (int i = 0; i < kSPW; ++i) y[i] = nbw[6 * i + 2 * I + ((stg & 1) ? 0 : 1)];
        if (stg & 1)
          neighbour(F{}, S1{}, I, sw, sspin, ws, wn, ss, xs, y, act);
        else
          neighbour(T{}, S1{}, I, sw, sspin, ws, wn, ss, y, y, act);
      }
      if (stg < kStages - 1) stage_end(stg);
    }

    // ------------------------------------------------------------ epilogue
    // (buffer 4 is released after it: the producer then stores the tiles).
    // RESC writes into buffer 4's block region: every consumer warp must have
    // finished stage 4's products first.
    if (MODE == MV_RESC) named_bar_sync(1, kWarps * 32);
    if (!dead && out_lane) {
      const uint32_t epi = smem_u32(smem + kBuf4 + kOffEpi);
#pragma unroll
      for (int i = 0; i < kSPW; ++i) {
        if (!act[i]) continue;
        const int x = xs[i];
#pragma unroll
        for (int sp = 0; sp < 2; ++sp)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int pl = sp * 36 + (2 * kq + e) * 6 + g;
            const uint32_t ea = epi + epi_off(pl, warp * kSPW + i);
            const cplx y_ = {acc[i][sp][e], acc[i][sp][2 + e]};
            const cplx pv = kIn ? lds2(ea) : cplx{0.0, 0.0};
            if (MODE == MV_PLAIN) {
              sts2(ea, y_.re, y_.im);
            } else if (MODE == MV_RHS) {
              sts2(ea, y_.re, y_.im);
              st(A.out2 + (int64_t)pl * V + x, 2.0 * y_ - pv);
            } else if (MODE == MV_RES) {
              const cplx r = pv - y_;
              sts2(ea, r.re, r.im);
              qs[sp][e][0] += norm2(r);
              qs[sp][e][1] += norm2(pv);
            } else if (MODE == MV_V) {
              sts2(ea, y_.re, y_.im);
              cplx dd = {0.0, 0.0};
              cmac_cj(dd, pv, y_);
              qs[sp][e][0] += dd.re;
              qs[sp][e][1] += dd.im;
            } else if (MODE == MV_RESC) {
              const uint32_t fa = smem_u32(smem + kBuf4 + kOffF32) + epi32_off(pl, warp * kSPW + i);
              const cplx r = pv - y_;
              const cplx dd = r * A.inv_theta[sp];
              sts2f(fa, (float)r.re, (float)r.im);
              sts2f(fa + kEpiHalf, (float)dd.re, (float)dd.im);
              qs[sp][e][0] += norm2(r);
              qs[sp][e][1] += norm2(pv);
            } else {  // MV_T: in = s
              sts2(ea, y_.re, y_.im);
              cplx dd = {0.0, 0.0};
              cmac_cj(dd, y_, pv);
              qs[sp][e][0] += dd.re;
              qs[sp][e][1] += dd.im;
              qs[sp][e][2] += norm2(y_);
            }
          }
      }
    }
    if (kNOut > 0) fence_proxy_async_smem();
    stage_end(kStages - 1);
    c_par ^= 1u;
  }
  // one partial row per CTA: sum over the rows g (lane bits 2-4), then over
  // the warps in a fixed order
  if constexpr (NQ > 0) {
    if (warp < kWarps) {
#pragma unroll
      for (int sp = 0; sp < 2; ++sp)
#pragma unroll
        for (int e = 0; e < 2; ++e)
#pragma unroll
          for (int kk = 0; kk < NQ; ++kk) {
            double v = qs[sp][e][kk];
            v += __shfl_xor_sync(0xffffffffu, v, 4);
            v += __shfl_xor_sync(0xffffffffu, v, 8);
            v += __shfl_xor_sync(0xffffffffu, v, 16);
            if (lane < 3) red[warp][sp * 6 + 2 * lane + e][kk] = v;
          }
    }
    __syncthreads();
    if (threadIdx.x < CN_COLS * NQ) {
      const int col12 = threadIdx.x / NQ, kk = threadIdx.x % NQ;
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) v += red[w][col12][kk];
      A.partials[((int64_t)blockIdx.x * CN_COLS + col12) * NQ + kk] = v;
    }
  }
}

// ------------------------------------------------------------------ host
void launch_cn_blocks(Lat L, const CnCoef &C, const double2 *U, const double2 *DE, double2 *W, cudaStream_t st) {
  const int64_t n = 36 * L.V;
  const unsigned grid = (unsigned)((n + 255) / 256);
  k_cn_blocks<<<grid, 256, 0, st>>>(L, C, U, DE, W);
}

int64_t cn_mv4_units(int64_t V) { return (V + mv4::kUnit - 1) / mv4::kUnit; }
int64_t cn_mv4_rows(int64_t V, int sm_count) { return std::min<int64_t>(cn_mv4_units(V), sm_count); }

int launch_cn_mv4(int mode, Lat L, const CnCoef &C, double nb_sign, const double2 *W, const double2 *Dsum,
                  const double *Bsum, const MvArgs &a, int *err, int sm_count, cudaStream_t st) {
  using namespace mv4;
  const uint64_t V = (uint64_t)L.V;
  if (L.V < kWMax || L.V > 0x7fffffffLL) return -1;
  Mv4Maps maps;
  memset(&maps, 0, sizeof(maps));
  if (!stage::encode(&maps.spin, a.in, 2 * V, 72, 2 * kTileS, 72) ||
      !stage::encode(&maps.D, Dsum, 2 * V, 9, 2 * kUnit, 9) || !stage::encode(&maps.B, Bsum, V, 9, kUnit, 9))
    return -1;
  // epilogue tile: operand in, results out (halves of 8 sites, 128-byte swizzle)
  const auto sw128 = CU_TENSOR_MAP_SWIZZLE_128B;
  const void *epi_src = (mode == MV_V) ? (const void *)a.in2
                        : (mode == MV_RES || mode == MV_RESC) ? (const void *)a.bvec : (const void *)a.in;
  if (mv4_tile_input(mode) && !stage::encode(&maps.epi_in, epi_src, 2 * V, 72, 16, 72, sw128)) return -1;
  if (mode == MV_RESC) {  // FP32 tiles: 16 sites x 2 floats per row
    const void *outs[2] = {a.r32, a.d32};
    for (int o = 0; o < 2; ++o)
      if (!stage::encode(&maps.out[o], outs[o], 2 * V, 72, 32, 72, sw128, CU_TENSOR_MAP_DATA_TYPE_FLOAT32)) return -1;
  } else {
    const void *outs[3] = {a.out, a.out2, a.out3};
    for (int o = 0; o < mv4_tile_outputs(mode); ++o)
      if (!stage::encode(&maps.out[o], outs[o], 2 * V, 72, 16, 72, sw128)) return -1;
  }
  const int64_t nunits = cn_mv4_units(L.V);
  const unsigned grid = (unsigned)cn_mv4_rows(L.V, sm_count);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    kern<<<grid, kThreads, kSmemBytes, st>>>(L, C, nb_sign, maps, W, Dsum, Bsum, a, nunits, err);
  };
  switch (mode) {
    case MV_PLAIN: go(k_cn_mv4<MV_PLAIN>); break;
    case MV_RHS: go(k_cn_mv4<MV_RHS>); break;
    case MV_RES: go(k_cn_mv4<MV_RES>); break;
    case MV_V: go(k_cn_mv4<MV_V>); break;
    case MV_RESC: go(k_cn_mv4<MV_RESC>); break;
    default: go(k_cn_mv4<MV_T>); break;
  }
  return 0;
}

}  // namespace nrq
