// FP64 FMA stencil of the assembled Crank-Nicolson operator on cached 6x6
// blocks (src/nrqcd.f90:1175-1387 with PETSc's block transposition; the
// operator is described in cn.cu): out = D in + sum over the 6 neighbours of
// the spin-colour blocks applied to the 6 propagator columns, both species.
//
// Blocks.  Once per update, k_cn_blocks5 writes the forward block of every
// site, direction and species with the operator's coefficients folded in
// (the blocks of the tensor-core stencil, cn_mv4.cu), row-major with a
// stride of 37 entries per block (the 37th is zero) so that the reads of
// one warp spread over the shared-memory banks.  With real Wilson
// coefficients the backward block is -W_I(x-I)^H, read from the forward
// block of x-I, and A^H differs from A by the sign of the neighbour sum.
//
// Products.  Six threads share a site and species: each owns two output
// rows (the two spins of one colour) and three of the six columns, 12
// doubles in registers.  Per neighbour and input row q a thread reads 2
// block entries and 3 spinor entries and does 24 FP64 FMAs, none of them
// padding.  Five consecutive sites of one species fill a warp (30 lanes, 2
// idle); the threads of a site that share rows or columns read the same
// shared-memory words, which shared memory broadcasts.  On B200 the FP64 FMA pipe
// and the FP64 tensor pipe have the same peak, and the tensor pipe's 16x8
// tiles carry 12 x 6 useful entries; these products need 56 % of its work.
//
// Pipeline.  Persistent, one CTA per SM: 8 consumer warps (species 0 in
// warps 0-3, species 1 in 4-7, a unit of 20 sites) and one producer warp.
// Five loads per unit (stage 0: diagonal matrices, -x and +x; 1: +y; 2: -y;
// 3: +z; 4: -z), each a spinor tile (TMA, 22 sites x 72 planes) and a block
// tile (bulk copies), into a ring of four shared-memory buffers completed on
// mbarriers.  The producer refills a buffer once every consumer warp
// released it and its previous load has completed.  A warp whose sites need
// a neighbour or block outside the stage's tiles (periodic wraps, tile
// edges) reads that neighbour from global memory.  Results, and the
// operands of the epilogue at the own site, go straight to and from global
// memory; the residual and dot-product partial sums stay in registers over
// all units of the CTA (one partial row per CTA).
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
constexpr int kUnit = 20;                 // sites per work unit
constexpr int kGroups = 5;                // (site, species) groups per warp, 6 row threads each
constexpr int kWarps = 8;                 // consumer warps: 4 per species
constexpr int kThreads = (kWarps + 1) * 32;
constexpr int kMaxReg = 168;              // 3 warps of one SM quarter x 32 x 168 <= 16384
constexpr int kStages = 5;                // loads per unit
constexpr int kBufs = 4;                  // ring of stage buffers
constexpr int kTileS = 22;                // spinor tile width in sites (x0 - 1 .. x0 + 20)
constexpr int kBlk = 37;                  // complex entries per stored block (36 + 1 zero)
constexpr int kBlkBytes = kBlk * 16;      // 592
constexpr int kWMax = kUnit + 1;          // blocks per species of stage 0 (x0 - 1 .. x0 + 19)
constexpr uint32_t kSpinBytes = 72u * kTileS * 16u;              // 25344
constexpr uint32_t kOffW = kSpinBytes;                           // block tile: species 0, then 1
constexpr uint32_t kWSpecies = (uint32_t)kWMax * kBlkBytes;      // 12432
constexpr uint32_t up128(uint32_t v) { return (v + 127u) & ~127u; }
constexpr uint32_t kOffD = up128(kOffW + 2u * kWSpecies);        // 50304: D, 9 planes x 20 sites x 16 B
constexpr uint32_t kOffB = up128(kOffD + 9u * kUnit * 16u);      // 53248: B, 9 planes x 20 sites x 8 B
constexpr uint32_t kBufBytes = ((kOffB + 9u * kUnit * 8u) + 1023u) & ~1023u;  // 55296
constexpr uint32_t kSmemBytes = kBufs * kBufBytes + 1024u;       // 222208
static_assert(kWarps * kGroups == 2 * kUnit, "warp layout");
static_assert(kOffW % 128 == 0 && kOffD % 128 == 0 && kOffB % 128 == 0 && kBufBytes % 1024 == 0, "layout");
static_assert(kSmemBytes <= 232448, "shared memory");
}  // namespace mv5

struct Mv5Maps {
  CUtensorMap spin;  // 72 planes x 2V doubles, box {44, 72}
  CUtensorMap D;     // 9 planes x 2V doubles, box {40, 9}
  CUtensorMap B;     // 9 planes x V doubles, box {20, 9}
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

// One thread per (direction I, species, site, row g): row g of the forward
// block W_I(x) of that species, row-major, block (I*2 + sp)*V + x of kBlk
// entries (entry 36 of row 5's thread set to zero).
__global__ void __launch_bounds__(256) k_cn_blocks5(Lat L, CnCoef C, const double2 *__restrict__ U,
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
  double2 *blk = W + r * mv5::kBlk;
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
      st(blk + g * 6 + 2 * cp + t, v);
    }
  }
  if (g == 5) st(blk + 36, cplx{0.0, 0.0});
}

namespace {

// coordinates and the six periodic neighbours (+x,-x,+y,-y,+z,-z) of site s
// (the stencil runs for V < 2^31 only)
__device__ __forceinline__ void neighbours5(const Lat &L, int s, int (&nb)[6]) {
  const int nx = (int)L.nx, ny = (int)L.ny, nz = (int)L.nz;
  const int t = s / nx, x = s - t * nx, z = t / ny, y = t - z * ny;
  const int row = nx, plane = nx * ny;
  nb[0] = x + 1 < nx ? s + 1 : s - (nx - 1);
  nb[1] = x > 0 ? s - 1 : s + (nx - 1);
  nb[2] = y + 1 < ny ? s + row : s - (ny - 1) * row;
  nb[3] = y > 0 ? s - row : s + (ny - 1) * row;
  nb[4] = z + 1 < nz ? s + plane : s - (nz - 1) * plane;
  nb[5] = z > 0 ? s - plane : s + (nz - 1) * plane;
}

// first site of the spinor tile of load `stg` of the unit at x0
// (stage 0: x0 - 1; stages 1-4: the +y, -y, +z, -z neighbours of x0)
__device__ __forceinline__ int spin_start5(const Lat &L, int x0, int stg) {
  if (stg == 0) return x0 - 1;
  const int nx = (int)L.nx, ny = (int)L.ny, nz = (int)L.nz;
  const int t = x0 / nx, z = t / ny, y = t - z * ny;
  const int row = nx, plane = nx * ny;
  switch (stg) {
    case 1: return y + 1 < ny ? x0 + row : x0 - (ny - 1) * row;
    case 2: return y > 0 ? x0 - row : x0 + (ny - 1) * row;
    case 3: return z + 1 < nz ? x0 + plane : x0 - (nz - 1) * plane;
    default: return z > 0 ? x0 - plane : x0 + (nz - 1) * plane;
  }
}
// first block and block count of the block tile of a load (forward stages:
// the unit itself; backward stages: its neighbours; stage 0 both)
__device__ __forceinline__ int blk_start5(int x0, int spin_start, int stg) {
  if (stg == 0) return x0 > 0 ? x0 - 1 : 0;
  if (stg == 1 || stg == 3) return x0;
  return spin_start;
}
__device__ __forceinline__ int blk_count5(int V, int start, int stg) {
  return min(stg == 0 ? mv5::kWMax : mv5::kUnit, V - start);
}

// The thread's 2 x 3 output tile (rows 2c + s of colour c, columns 3h + k)
// += sum over q of w[s][q] psi[q][3h + k], all of it in registers.  Forward:
// w[s][q] = sgn W(x)[2c+s][q], at w + (s*6 + q) (row-major block, w at row
// 2c); backward: w[s][q] = -sgn conj(W(y)[q][2c+s]), at w + (q*6 + s) (w at
// column 2c).  psi[q][3h + k] at psi + (k*6 + q) * pstride (psi at plane
// 18 h of the species).
template <bool BWD>
__device__ __forceinline__ void nb_products(double (&acc)[2][3][2], const double2 *w, const double2 *psi,
                                            int pstride, double sgn) {
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double wr[2], wi[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double2 wv = w[BWD ? q * 6 + s : s * 6 + q];
      wr[s] = BWD ? -sgn * wv.x : sgn * wv.x;
      wi[s] = sgn * wv.y;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 p = psi[(k * 6 + q) * pstride];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        acc[s][k][0] = fma(wr[s], p.x, fma(-wi[s], p.y, acc[s][k][0]));
        acc[s][k][1] = fma(wr[s], p.y, fma(wi[s], p.x, acc[s][k][1]));
      }
    }
  }
}

// 16-byte load from a shared-memory address (ld.shared, never generic)
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

// nb_products with both operands in the stage's shared tiles (shared-space
// byte addresses; every offset below is a compile-time constant)
template <bool BWD>
__device__ __forceinline__ void nb_products_smem(double (&acc)[2][3][2], uint32_t w, uint32_t psi, double sgn) {
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double wr[2], wi[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double2 wv = lds_d2(w + (uint32_t)((BWD ? q * 6 + s : s * 6 + q) * 16));
      wr[s] = BWD ? -sgn * wv.x : sgn * wv.x;
      wi[s] = sgn * wv.y;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2 p = lds_d2(psi + (uint32_t)((k * 6 + q) * mv5::kTileS * 16));
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        acc[s][k][0] = fma(wr[s], p.x, fma(-wi[s], p.y, acc[s][k][0]));
        acc[s][k][1] = fma(wr[s], p.y, fma(wi[s], p.x, acc[s][k][1]));
      }
    }
  }
}

}  // namespace

template <int MODE>
__global__ void __maxnreg__(mv5::kMaxReg)
    k_cn_mv5(Lat L, CnCoef C, double nb_sign, const __grid_constant__ Mv5Maps maps, const double2 *__restrict__ W,
             const double2 *__restrict__ Dsum, const double *__restrict__ Bsum, MvArgs A, int nunits, int *err,
             long long wait_cycles, int stall_load) {
  using namespace mv5;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kBufs], empty_bar[kBufs];
  __shared__ double red[kWarps][6][3];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int V = (int)L.V;  // the launcher admits V < 2^31 only

  if (threadIdx.x == 0) {
    for (int b = 0; b < kBufs; ++b) {
      mbar_init(&full_bar[b], 1);
      mbar_init(&empty_bar[b], kWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const int my_units = (nunits - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int total = my_units * kStages;

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
      int i = 0;
      for (; i < stop && ok; ++i) {
        const int b = i % kBufs;
        if (i >= kBufs) {
          const uint32_t par = (uint32_t)((i / kBufs - 1) & 1);
          // every consumer warp released the buffer, and its previous load landed
          ok = wait(&empty_bar[b], par) && mbar_wait(&full_bar[b], par);
          if (!ok) break;
        }
        const int stg = i % kStages;
        const int x0 = ((int)blockIdx.x + (i / kStages) * (int)gridDim.x) * kUnit;
        const int ss = spin_start5(L, x0, stg);
        const int ws = blk_start5(x0, ss, stg);
        const int wn = blk_count5(V, ws, stg);
        const int I = stg == 0 ? 0 : (stg + 1) / 2;
        unsigned char *bb = smem + b * kBufBytes;
        uint32_t tx = kSpinBytes + 2u * (uint32_t)wn * kBlkBytes;
        if (stg == 0) tx += 9u * kUnit * 16u + 9u * kUnit * 8u;
        mbar_expect_tx(&full_bar[b], tx);
        tma_2d(bb, &maps.spin, 2 * ss, 0, &full_bar[b]);
#pragma unroll
        for (int sp = 0; sp < 2; ++sp)
          bulk_1d(bb + kOffW + sp * kWSpecies, W + ((int64_t)(I * 2 + sp) * V + ws) * kBlk,
                  (uint32_t)wn * kBlkBytes, &full_bar[b]);
        if (stg == 0) {
          tma_2d(bb + kOffD, &maps.D, 2 * x0, 0, &full_bar[b]);
          tma_2d(bb + kOffB, &maps.B, x0, 0, &full_bar[b]);
        }
      }
      if (!ok) atomicExch(err, NRQ_ERR_TIMEOUT);
      // every issued load lands before the CTA exits: loads before the last
      // kBufs were waited for above
      for (int k = max(0, i - kBufs); k < i; ++k)
        if (!mbar_wait(&full_bar[k % kBufs], (uint32_t)((k / kBufs) & 1))) {
          atomicExch(err, NRQ_ERR_TIMEOUT);
          break;
        }
    }
    return;
  }

  // ---------------------------------------------------------- consumers
  // lane = 6 g + j: site group g (5 per warp, lanes 30-31 idle), colour
  // c = j % 3 and column half h = j / 3; the thread owns rows 2c, 2c + 1
  // (spins 0, 1 of colour c) and columns 3h .. 3h + 2 of its site and species
  const int sp = warp >> 2;                 // species of this warp
  const int g = lane / 6, j = lane - 6 * g;
  const bool lane_on = g < kGroups;
  const int gc = lane_on ? g : 0;
  const int jj = lane_on ? j : 0;
  const int c = jj % 3, h = jj / 3;
  const int site_in_unit = (warp & 3) * kGroups + gc;
  constexpr int NQ = (MODE == MV_T) ? 3 : ((MODE == MV_RES || MODE == MV_V || MODE == MV_RESC) ? 2 : 0);
  double qs[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k) qs[k][0] = qs[k][1] = qs[k][2] = 0.0;
  const cplx ak = C.kin[sp], am = C.mag[sp], ad = C.dar[sp];
  const cplx dg = C.dkin * ak + cplx{1.0, 0.0};
  bool dead = false;
  int ld = 0;  // index of the next load this CTA consumes
  // plane of the thread's entry (row 2c + s, column 3h + k) in the species
  auto plane = [&](int s, int k) { return (3 * h + k) * 6 + 2 * c + s; };

  for (int u = 0; u < my_units; ++u) {
    const int x0 = ((int)blockIdx.x + u * (int)gridDim.x) * kUnit;
    const int x = x0 + site_in_unit;
    const bool act = lane_on && x < V;
    const int xs = x < V ? x : V - 1;  // a valid site for the idle lanes' addresses
    int nb[6];
    neighbours5(L, xs, nb);
    double acc[2][3][2];
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[s][k][0] = acc[s][k][1] = 0.0;
    // the epilogue's operand at the own site (b for the residuals, rh for V,
    // the input itself for RHS and T), requested now so that its latency
    // hides behind the unit's products
    constexpr bool kEpiIn = MODE != MV_PLAIN;
    double2 epi[2][3];
    if (kEpiIn) {
      const double2 *src = (MODE == MV_V) ? A.in2 : (MODE == MV_RES || MODE == MV_RESC) ? A.bvec : A.in;
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int k = 0; k < 3; ++k)
          epi[s][k] = act ? __ldg(src + (int64_t)(sp * 36 + plane(s, k)) * V + x) : make_double2(0.0, 0.0);
    }

#pragma unroll
    for (int stg = 0; stg < kStages; ++stg, ++ld) {
      const int b = ld % kBufs;
      const bool expired = !dead && !wait(&full_bar[b], (uint32_t)((ld / kBufs) & 1));
      // warp-uniform: the products below use warp votes
      if (__any_sync(0xffffffffu, expired) && !dead) {
        dead = true;
        if (lane == 0) atomicExch(err, NRQ_ERR_TIMEOUT);
      }
      const unsigned char *bb = smem + b * kBufBytes;
      const uint32_t s_tile = smem_u32(bb) + (uint32_t)(sp * 36 * kTileS * 16);  // the species' planes
      const uint32_t s_w = smem_u32(bb) + kOffW + (uint32_t)sp * kWSpecies;
      if (!dead) {
        const int ss = spin_start5(L, x0, stg);
        const int ws = blk_start5(x0, ss, stg);
        const int wn = blk_count5(V, ws, stg);
        if (stg == 0) {
          // diagonal (colour only): row (c, s) takes input rows (j, s);
          // x - ss = site_in_unit + 1 lies inside the tile for every lane
          const uint32_t s_d = smem_u32(bb) + kOffD + (uint32_t)(site_in_unit * 16);
          const uint32_t s_b = smem_u32(bb) + kOffB + (uint32_t)(site_in_unit * 8);
          const uint32_t s_own = s_tile + (uint32_t)((site_in_unit + 1) * 16 + 18 * h * kTileS * 16);
#pragma unroll
          for (int jc = 0; jc < 3; ++jc) {
            const int e = jc * 3 + c;
            const double2 dv = lds_d2(s_d + (uint32_t)(e * kUnit * 16));
            const double bv = lds_d1(s_b + (uint32_t)(e * kUnit * 8));
            cplx cd = ad * cplx{dv.x, dv.y} + bv * am;
            if (jc == c) cd = cd + dg;
#pragma unroll
            for (int s = 0; s < 2; ++s)
#pragma unroll
              for (int k = 0; k < 3; ++k) {
                const double2 p = lds_d2(s_own + (uint32_t)((k * 6 + 2 * jc + s) * kTileS * 16));
                acc[s][k][0] = fma(cd.re, p.x, fma(-cd.im, p.y, acc[s][k][0]));
                acc[s][k][1] = fma(cd.re, p.y, fma(cd.im, p.x, acc[s][k][1]));
              }
          }
        }
        // neighbours of this load: stage 0 = +x (forward) and -x (backward)
#pragma unroll
        for (int hh = 0; hh < (stg == 0 ? 2 : 1); ++hh) {
          const bool bwd = stg == 0 ? (hh == 1) : (stg % 2 == 0);
          const int d = stg == 0 ? hh : stg + 1;  // neighbour index in nb[]
          const int I = d >> 1;
          const int y = nb[d];                   // neighbour site
          const int m = bwd ? y : xs;            // site of the forward block
          const int woff = bwd ? 2 * c : 12 * c; // the thread's rows (or columns) in the block
          const bool ps = (unsigned)(y - ss) < (unsigned)kTileS;  // spinor in the tile
          const bool ws_ = (unsigned)(m - ws) < (unsigned)wn;     // block in the tile
          if (__all_sync(0xffffffffu, (ps && ws_) || !act)) {
            // every operand of the warp in shared memory: compile-time offsets
            const uint32_t wrow = s_w + (uint32_t)(((m - ws) * kBlk + woff) * 16);
            const uint32_t psi = s_tile + (uint32_t)((y - ss) * 16 + 18 * h * kTileS * 16);
            if (bwd)
              nb_products_smem<true>(acc, wrow, psi, nb_sign);
            else
              nb_products_smem<false>(acc, wrow, psi, nb_sign);
          } else if (act) {
            // some lanes' operands outside the tiles (periodic wraps, tile
            // edges): those lanes read global memory, the others the tiles
            const double2 *wt = (const double2 *)(bb + kOffW + sp * kWSpecies);
            const double2 *tsp = (const double2 *)bb + sp * 36 * kTileS;
            const double2 *wrow =
                (ws_ ? wt + (m - ws) * kBlk : W + ((int64_t)(I * 2 + sp) * V + m) * kBlk) + woff;
            const double2 *psi = (ps ? tsp + (y - ss) + 18 * h * kTileS
                                     : A.in + (int64_t)(sp * 36 + 18 * h) * V + y);
            const int pstride = ps ? kTileS : V;
            if (bwd)
              nb_products<true>(acc, wrow, psi, pstride, nb_sign);
            else
              nb_products<false>(acc, wrow, psi, pstride, nb_sign);
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty_bar[b]);
    }

    // ---------------------------------------------------------- epilogue
    if (!dead && act) {
#pragma unroll
      for (int s = 0; s < 2; ++s)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int64_t off = (int64_t)(sp * 36 + plane(s, k)) * V + x;
          const cplx y_ = {acc[s][k][0], acc[s][k][1]};
          const cplx ev = {epi[s][k].x, epi[s][k].y};
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

  // one partial row per CTA: column 3h + k of each lane, summed over the
  // warp's lanes of that half, then over the 4 warps of each species in a
  // fixed order
  if constexpr (NQ > 0) {
#pragma unroll
    for (int n = 0; n < 6; ++n)
#pragma unroll
      for (int kk = 0; kk < NQ; ++kk) {
        double v = (lane_on && h == n / 3) ? qs[n % 3][kk] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][n][kk] = v;
      }
    named_bar_sync(1, kWarps * 32);
    if (threadIdx.x < CN_COLS * NQ) {
      const int col12 = threadIdx.x / NQ, kk = threadIdx.x % NQ;
      const int spc = col12 / 6, n = col12 % 6;
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < 4; ++w) v += red[spc * 4 + w][n][kk];
      A.partials[((int64_t)blockIdx.x * CN_COLS + col12) * NQ + kk] = v;
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
int64_t cn_mv5_block_entries(int64_t V) { return 6 * V * mv5::kBlk; }

int launch_cn_mv5(int mode, Lat L, const CnCoef &C, double nb_sign, const double2 *W, const double2 *Dsum,
                  const double *Bsum, const MvArgs &a, int *err, int sm_count, cudaStream_t st,
                  long long wait_cycles, int stall_load) {
  using namespace mv5;
  const uint64_t V = (uint64_t)L.V;
  // B tiles start at x0 = 20 u: 16-byte aligned rows need an even V as well
  if (L.V < kTileS || L.V > 0x7fffffffLL || (L.V & 1)) return -1;
  Mv5Maps maps;
  memset(&maps, 0, sizeof(maps));
  if (!stage::encode(&maps.spin, a.in, 2 * V, 72, 2 * kTileS, 72) ||
      !stage::encode(&maps.D, Dsum, 2 * V, 9, 2 * kUnit, 9) || !stage::encode(&maps.B, Bsum, V, 9, kUnit, 9))
    return -1;
  const int nunits = (int)cn_mv5_units(L.V);
  const unsigned grid = (unsigned)cn_mv5_rows(L.V, sm_count);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    kern<<<grid, kThreads, kSmemBytes, st>>>(L, C, nb_sign, maps, W, Dsum, Bsum, a, nunits, err, wait_cycles,
                                             stall_load);
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
