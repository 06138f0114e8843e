// Gluon-distribution observables on the device (src/gaugeconfiguration_su3.f90,
// abbreviated "gauge"; src/lattice.f90 "lattice"):
//   - Coulomb gauge fixing of the links, CoulombGaugefixing_Links
//     (gauge:2297-2456): the divergence D(x) = sum_i AH(U_i(x-i) - U_i(x))
//     (gauge:2460-2478), Fourier acceleration by (pmax/|p|)^2, the gauge
//     transformation G = ExpAH(alpha D) and U_i(x) <- G(x) U_i(x) G(x+i)^+;
//     the electric field is not transformed, as in the reference
//   - the transverse AA and EE correlators (gauge:1825-1972): algebra
//     coordinates of ArgLogU(U_i)/a_i and of E/(a_i a0), their x2p transforms
//     and f_i P_ij conj(f_j) / Volume with the real part of the transverse
//     projector (lattice:1184-1198) at the backward-derivative momentum
//     (lattice:963-979), averaged over the eight generators.
// The FFTs are cuFFT Z2Z transforms over all components at once; the x2p
// (a1 a2 a3) and p2x (1/Volume) scales of the reference are applied in the
// kernels around them.
#include "nrq_eigen.cuh"
#include "nrq_kernels.cuh"

namespace nrq {

namespace {
// backward-derivative lattice momentum (lattice:963-979) of site s; returns |p|
__device__ __forceinline__ double lattice_momentum(const Lat &L, int64_t s, cplx p[3]) {
  const int64_t x = s % L.nx, t = s / L.nx;
  const int64_t y = t % L.ny, z = t / L.ny;
  const int64_t pos[3] = {x, y, z};
  const int64_t ext[3] = {L.nx, L.ny, L.nz};
  double n2 = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double sn, cs;
    sincospi((double)pos[i] / (double)ext[i], &sn, &cs);
    const double m = 2.0 * sn / L.a[i];
    p[i] = {m * cs, -m * sn};
    n2 += m * m;
  }
  return sqrt(n2);
}
}  // namespace

// D(x) = sum_i AH(U_i(x-i) - U_i(x)), AH(M) = (M - M^+)/2, as 9 complex
// planes (r*3 + c); partials[block] = max over the block of |D(x)|_F / 9
__global__ void __launch_bounds__(128) k_cg_divergence(Lat L, const double2 *__restrict__ U,
                                                       double2 *__restrict__ D, double *__restrict__ partials) {
  const int64_t V = L.V;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double f = 0.0;
  if (s < V) {
    m3 d = m3_zero();
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const m3 u = load_link(U, V, s, i), um = load_link(U, V, nb(L, s, i, -1), i);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const cplx a = um.e[r * 3 + c] - u.e[r * 3 + c];
          const cplx b = um.e[c * 3 + r] - u.e[c * 3 + r];
          d.e[r * 3 + c].re += 0.5 * (a.re - b.re);
          d.e[r * 3 + c].im += 0.5 * (a.im + b.im);
        }
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      D[(int64_t)k * V + s] = make_double2(d.e[k].re, d.e[k].im);
      f += norm2(d.e[k]);
    }
    f = sqrt(f) / 9.0;
  }
  __shared__ double sh[4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) f = fmax(f, __shfl_down_sync(0xffffffffu, f, o));
  if (lane == 0) sh[warp] = f;
  __syncthreads();
  if (threadIdx.x == 0) partials[blockIdx.x] = fmax(fmax(sh[0], sh[1]), fmax(sh[2], sh[3]));
}

// p-space step of the Fourier acceleration: D(p) *= scale (pmax/|p|)^2 for
// |p| above the reference's zero tolerance, D(p) *= scale otherwise (scale
// carries alpha and the x2p/p2x normalisation)
__global__ void k_cg_accelerate(Lat L, double2 *__restrict__ D, double pmax, double scale) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= L.V) return;
  cplx p[3];
  const double pn = lattice_momentum(L, s, p);
  const double f = pn > 1e-12 ? scale * (pmax / pn) * (pmax / pn) : scale;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double2 v = D[(int64_t)k * L.V + s];
    v.x *= f;
    v.y *= f;
    D[(int64_t)k * L.V + s] = v;
  }
}

// G = ExpAH(A) = exp(i H), H = -i A (hermitian; A anti-hermitian, not
// traceless), in place: exp(i H) = exp(i tr(H)/3) exp(i (H - tr(H)/3))
__global__ void __launch_bounds__(128) k_cg_expah(int64_t V, double2 *__restrict__ D) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  m3 a;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 v = D[(int64_t)k * V + s];
    a.e[k] = {v.x, v.y};
  }
  // H = -i A, made exactly hermitian
  m3 h;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      // (H + H^+)/2 with H = -i A: -i x = (x.im, -x.re), conj(-i y) = (y.im, y.re)
      const cplx x = a.e[r * 3 + c], y = a.e[c * 3 + r];
      h.e[r * 3 + c] = {0.5 * (x.im + y.im), 0.5 * (y.re - x.re)};
    }
  const double tr = (h.e[0].re + h.e[4].re + h.e[8].re) / 3.0;
  h.e[0].re -= tr;
  h.e[4].re -= tr;
  h.e[8].re -= tr;
  const m3 g0 = expi_herm(h);
  double sn, cs;
  sincos(tr, &sn, &cs);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const cplx v = g0.e[k];
    D[(int64_t)k * V + s] = make_double2(cs * v.re - sn * v.im, cs * v.im + sn * v.re);
  }
}

// U_i(x) <- G(x) U_i(x) G(x+i)^+ (in place: a thread reads and writes only
// its own site's links)
__global__ void __launch_bounds__(128) k_cg_transform(Lat L, double2 *__restrict__ U, const double2 *__restrict__ G) {
  const int64_t V = L.V;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  m3 g;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double2 v = G[(int64_t)k * V + s];
    g.e[k] = {v.x, v.y};
  }
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
    const int64_t xp = nb(L, s, i, +1);
    m3 gp;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const double2 v = G[(int64_t)k * V + xp];
      gp.e[k] = {v.x, v.y};
    }
    store_link(U, V, s, i, mul_nd(mul(g, load_link(U, V, s, i)), gp));
  }
}

// F plane (field*24 + i*8 + a): field 0 the gauge field 2 Re Tr(T^a ArgLogU(U_i))/a_i
// (gauge:1992-2000, su3:318-334), field 1 the electric field E^a_i/(a_i a0)
// (gauge:2032-2049); complex with zero imaginary part, for the FFT
__global__ void __launch_bounds__(128) k_gluon_fields(Lat L, const double2 *__restrict__ U,
                                                      const double *__restrict__ E, double2 *__restrict__ F) {
  const int64_t V = L.V;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
    cplx ev[3];
    m3 S;
    eigenc3(load_link(U, V, s, i), ev, S);
    double th[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) th[k] = atan2(ev[k].im, ev[k].re);
    // ArgLogU = S^+ diag(theta) S
    m3 h;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cplx acc = {0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const cplx a = conj(S.e[k * 3 + r]), b = S.e[k * 3 + c];
          acc = acc + th[k] * (a * b);
        }
        h.e[r * 3 + c] = acc;
      }
    cplx tr[8];
    traces_with_generators(h, tr);
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      F[(int64_t)(i * 8 + a) * V + s] = make_double2(2.0 * tr[a].re / L.a[i], 0.0);
      F[(int64_t)(24 + i * 8 + a) * V + s] = make_double2(E[(int64_t)(i * 8 + a) * V + s] / L.a[i] / L.a0, 0.0);
    }
  }
}

// per momentum site: out[0][s] = AA, out[1][s] = EE, out[2][s] = |p|
// (F holds the unscaled forward transforms; fwd = a1 a2 a3)
__global__ void __launch_bounds__(128) k_transverse_corr(Lat L, const double2 *__restrict__ F, double fwd,
                                                         double volume, double *__restrict__ out) {
  const int64_t V = L.V;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= V) return;
  cplx p[3];
  const double pn = lattice_momentum(L, s, p);
  // the reference's projector is real: Re[(delta_ij - conj(p_i) p_j / |p|^2) / 2]
  double P[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double re = p[i].re * p[j].re + p[i].im * p[j].im;  // Re(conj(p_i) p_j)
      P[i][j] = pn < 1e-12 ? 0.0 : ((i == j ? 1.0 : 0.0) - re / (pn * pn)) / 2.0;
    }
#pragma unroll 1
  for (int field = 0; field < 2; ++field) {
    double acc = 0.0;
#pragma unroll 1
    for (int a = 0; a < 8; ++a) {
      cplx f[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double2 v = F[(int64_t)(field * 24 + i * 8 + a) * V + s];
        f[i] = {v.x * fwd, v.y * fwd};
      }
      double res = 0.0;  // Re sum_ij f_i P_ij conj(f_j)
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) res += P[i][j] * (f[i].re * f[j].re + f[i].im * f[j].im);
      acc += (res / volume) / 8.0;
    }
    out[(int64_t)field * V + s] = acc;
  }
  out[2 * V + s] = pn;
}

}  // namespace nrq
