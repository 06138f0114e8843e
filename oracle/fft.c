/*
 * Oracle (test infrastructure only): 3-D complex DFT with the conventions the
 * reference configures on its MKL cluster DFT (src/xpfft.f90:129-139):
 *   forward  (x2p, :607-621): X(k) = scale * sum_n x(n) exp(-2 pi i k.n/N)
 *   backward (p2x, :628-645): x(n) = scale * sum_k X(k) exp(+2 pi i k.n/N)
 * with forward scale = prod a_i and backward scale = 1/Volume, Volume =
 * prod N_i a_i (src/lattice.f90:149).  The data layout is the reference's
 * lattice order, x fastest.
 *
 * Mixed-radix recursive Cooley-Tukey (any extent; small prime factors are
 * handled by a direct DFT of that radix).
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

typedef double complex cplx;

static int smallest_factor(int n) {
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

/* out[k] = sum_j in[j*stride] w^(j*k*tws), n = length, tw = table of size N */
static void fft_rec(const cplx *in, int stride, cplx *out, int n, const cplx *tw,
                    int N, int tws, cplx *scratch) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = smallest_factor(n);
  int m = n / p;
  for (int r = 0; r < p; ++r)
    fft_rec(in + r * stride, stride * p, out + r * m, m, tw, N, tws * p, scratch + n);
  /* combine: X[k + q m] = sum_r W_n^{r(k+qm)} Y_r[k] */
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) {
      int kk = k + q * m;
      cplx acc = 0;
      for (int r = 0; r < p; ++r) {
        long e = ((long)r * kk) % n;
        acc += tw[(e * tws) % N] * out[r * m + k];
      }
      scratch[kk] = acc;
    }
  }
  memcpy(out, scratch, sizeof(cplx) * (size_t)n);
}

static void fft_line(cplx *line, int N, const cplx *tw, cplx *work) {
  /* work: 3N entries (copy of input, scratch recursion) */
  cplx *in = work;
  memcpy(in, line, sizeof(cplx) * (size_t)N);
  cplx *scratch = work + N;
  fft_rec(in, 1, line, N, tw, N, 1, scratch);
}

void oc_fft3d(double *data_, const int64_t n[3], int sign, double scale) {
  cplx *data = (cplx *)data_;
  const int64_t nx = n[0], ny = n[1], nz = n[2];
  const double twopi = 2.0 * acos(-1.0);
  for (int axis = 0; axis < 3; ++axis) {
    int N = (int)n[axis];
    cplx *tw = (cplx *)malloc(sizeof(cplx) * (size_t)N);
    for (int k = 0; k < N; ++k) {
      double ang = sign * twopi * (double)k / (double)N;
      tw[k] = cos(ang) + I * sin(ang);
    }
    int64_t stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
    int64_t nlines = (nx * ny * nz) / N;
#pragma omp parallel
    {
      cplx *line = (cplx *)malloc(sizeof(cplx) * (size_t)N);
      /* recursion depth <= log2 N; each level uses n <= N scratch */
      cplx *work = (cplx *)malloc(sizeof(cplx) * (size_t)N * 40);
#pragma omp for schedule(static)
      for (int64_t l = 0; l < nlines; ++l) {
        int64_t base;
        if (axis == 0) base = l * nx;
        else if (axis == 1) base = (l % nx) + (l / nx) * nx * ny;
        else base = l;
        for (int k = 0; k < N; ++k) line[k] = data[base + k * stride];
        fft_line(line, N, tw, work);
        for (int k = 0; k < N; ++k) data[base + k * stride] = line[k];
      }
      free(line);
      free(work);
    }
    free(tw);
  }
  if (scale != 1.0) {
    int64_t V = nx * ny * nz;
    for (int64_t s = 0; s < V; ++s) data[s] *= scale;
  }
}
