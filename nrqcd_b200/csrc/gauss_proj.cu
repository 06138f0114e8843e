// Gauss-law projection of the thermal initial condition (EquilibriumInit,
// src/gaugeconfiguration_su3.f90:455-500, abbreviated "gauge"): Jacobi
// sweeps
//   E_k(x) <- coords( kdt (U_k(x) G(x) U_k(x)^+ G(x+k) - G(x)) + E_k(x) ),
//   kdt = 0.01 a0,
// with G(x) = sum_i (E_i(x) - U_i(x-i)^+ E_i(x-i) U_i(x-i)) / a_i / a0
// (GetG, gauge:786-812) taken from the field before the sweep, until the
// max-norm deviation max_{x,a} 2|Tr(T^a G(x))| (GetGdeviation,
// gauge:724-768) is at most the tolerance.
//
// One sweep is two launches (V < 2^31 sites): k_gauss_g writes G of every site (9 complex
// planes) and the deviation (the last block to finish reduces the per-block
// maxima and decides convergence), then k_gauss_sweep updates E in place
// (each thread reads and writes only its own site's E).  Convergence is
// decided on the device: once the deviation is at most the tolerance both
// kernels return at entry, so the host can queue many sweeps between reads
// and the sweep count is the reference's exactly.
#include "nrq_kernels.cuh"

namespace nrq {

namespace {
// site coordinates with 32-bit arithmetic (V < 2^31, checked by the host),
// computed once per thread; neighbours by periodic offsets
struct Pos32 {
  uint32_t s, x, y, z, nx, nxy;
};
__device__ __forceinline__ Pos32 pos32(const Lat &L, uint32_t s) {
  Pos32 p;
  p.s = s;
  p.nx = (uint32_t)L.nx;
  p.nxy = p.nx * (uint32_t)L.ny;
  const uint32_t t = s / p.nx;
  p.x = s - t * p.nx;
  p.z = t / (uint32_t)L.ny;
  p.y = t - p.z * (uint32_t)L.ny;
  return p;
}
__device__ __forceinline__ uint32_t fwd32(const Lat &L, const Pos32 &p, int d) {
  if (d == 0) return p.x + 1 == p.nx ? p.s + 1 - p.nx : p.s + 1;
  if (d == 1) return p.y + 1 == (uint32_t)L.ny ? p.s + p.nx - p.nxy : p.s + p.nx;
  return p.z + 1 == (uint32_t)L.nz ? p.s + p.nxy - (uint32_t)L.V : p.s + p.nxy;
}
__device__ __forceinline__ uint32_t bwd32(const Lat &L, const Pos32 &p, int d) {
  if (d == 0) return p.x == 0 ? p.s + p.nx - 1 : p.s - 1;
  if (d == 1) return p.y == 0 ? p.s + p.nxy - p.nx : p.s - p.nx;
  return p.z == 0 ? p.s + (uint32_t)L.V - p.nxy : p.s - p.nxy;
}
}  // namespace

__global__ void __launch_bounds__(128, 3) k_gauss_g(Lat L, const double2 *__restrict__ U,
                                                 const double *__restrict__ E, double2 *__restrict__ G,
                                                 double *__restrict__ partials, GaussProjState *st, double tol,
                                                 int count) {
  if (*(volatile int *)&st->done) return;
  const int64_t V = L.V;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double mx = 0.0;
  if (s < V) {
    const Pos32 p = pos32(L, (uint32_t)s);
    m3 g = m3_zero();
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int64_t xm = bwd32(L, p, i);
      double al[8], aln[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        al[a] = E[(int64_t)(i * 8 + a) * V + s];
        aln[a] = E[(int64_t)(i * 8 + a) * V + xm];
      }
      const m3 un = load_link(U, V, xm, i);
      const m3 t = mul(mul_dn(un, algebra_matrix(aln)), un);
      const m3 d = sub(algebra_matrix(al), t);
      const double c = 1.0 / (L.a[i] * L.a0);  // one division per direction, not per entry
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        g.e[k].re = fma(d.e[k].re, c, g.e[k].re);
        g.e[k].im = fma(d.e[k].im, c, g.e[k].im);
      }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) G[(int64_t)k * V + s] = make_double2(g.e[k].re, g.e[k].im);
    cplx tr[8];
    traces_with_generators(g, tr);
    // max |Tr(T^a G)|^2 here; the deviation 2|Tr| is taken once, by the last block
#pragma unroll
    for (int a = 0; a < 8; ++a) mx = fmax(mx, tr[a].re * tr[a].re + tr[a].im * tr[a].im);
  }
  // block maximum
  __shared__ double sh[4];  // one per warp of the 128-thread block
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if (lane == 0) sh[warp] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
    partials[blockIdx.x] = m;
    __threadfence();
    last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  // last block: maximum over all blocks (order-independent, exact)
  __threadfence();
  double m = 0.0;
  for (int64_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) m = fmax(m, ((volatile double *)partials)[b]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if (lane == 0) sh[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m2 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m2 = fmax(m2, sh[w]);
    const double dev = 2.0 * sqrt(m2);
    st->dev = dev;
    if (count) st->sweeps += 1;
    if (!(dev > tol)) st->done = 1;
    st->ticket = 0u;
    __threadfence();
  }
}

__global__ void __launch_bounds__(128) k_gauss_sweep(Lat L, const double2 *__restrict__ U,
                                                     const double2 *__restrict__ G, double *__restrict__ E,
                                                     const GaussProjState *st, double kdt) {
  if (*(const volatile int *)&st->done) return;
  const int64_t V = L.V;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  const Pos32 p = pos32(L, (uint32_t)s);
  m3 g;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 v = G[(int64_t)k * V + s];
    g.e[k] = {v.x, v.y};
  }
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const int64_t xp = fwd32(L, p, k);
    m3 gn;
#pragma unroll
    for (int m = 0; m < 9; ++m) {
      const double2 v = G[(int64_t)m * V + xp];
      gn.e[m] = {v.x, v.y};
    }
    double al[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) al[a] = E[(int64_t)(k * 8 + a) * V + s];
    const m3 u = load_link(U, V, s, k);
    const m3 t = mul(mul_nd(mul(u, g), u), gn);  // U G U^+ G(x+k)
    const m3 e = algebra_matrix(al);
    m3 term;
#pragma unroll
    for (int m = 0; m < 9; ++m) {
      term.e[m].re = kdt * (t.e[m].re - g.e[m].re) + e.e[m].re;
      term.e[m].im = kdt * (t.e[m].im - g.e[m].im) + e.e[m].im;
    }
    cplx tr[8];
    traces_with_generators(term, tr);
#pragma unroll
    for (int a = 0; a < 8; ++a) E[(int64_t)(k * 8 + a) * V + s] = 2.0 * tr[a].re;
  }
}

}  // namespace nrq
