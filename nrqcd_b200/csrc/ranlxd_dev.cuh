// Device draw of the ranlxd stream (level 1 or 2) for the initial
// conditions: the generator of src/ranlxd_generator.f90:72-350 (the
// subtract-with-borrow recurrence with lags (12, 5) in base 2^48 and pr
// steps per 12 delivered numbers), carried in 48-bit integers as in
// ranlxd_host.h, so that every number equals the host stream's bit for bit.
// The host computes each thread's starting state with one modular
// multiplication (block_states in ranlxd_host.h); the recurrence, the
// Box-Muller transform of random.f90:238-255 and the writes of the field
// run on the device.
//
// Stream layout: pair e of a draw is numbers (first + 2e, first + 2e + 1).
// Thread t draws the pairs [t ppt, (t+1) ppt); ppt is a multiple of 6, so
// every thread starts first % 12 numbers into a block, and first is even,
// so no pair straddles two blocks.
#pragma once
#include <cstdint>
#include <vector>

#include "nrq_common.cuh"
#include "nrq_internal.h"
#include "ranlxd_host.h"

namespace nrq {

// one recurrence step on ring slot i (the oldest word) with lag slot j
__device__ __forceinline__ void swb_step(int64_t &xi, int64_t xj, int64_t &c) {
  const int64_t y = xj - xi - c;
  c = (int64_t)((uint64_t)y >> 63);
  xi = y + (c << 48);
}

// PR steps over the ring held oldest first, then the ring rotated back to
// oldest first: x then holds the block's 12 numbers (times 2^48) in the
// order ranlxd delivers them
template <int PR>
__device__ __forceinline__ void swb_refill(int64_t (&x)[12], int64_t &c) {
#pragma unroll 1
  for (int rep = 0; rep < PR / 12; ++rep) {
#pragma unroll
    for (int i = 0; i < 12; ++i) swb_step(x[i], x[i < 5 ? i + 7 : i - 5], c);
  }
  constexpr int kRest = PR % 12;
#pragma unroll
  for (int i = 0; i < kRest; ++i) swb_step(x[i], x[i < 5 ? i + 7 : i - 5], c);
  int64_t r[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) r[k] = x[(kRest + k) % 12];
#pragma unroll
  for (int k = 0; k < 12; ++k) x[k] = r[k];
}

// op(e, u1, u2) for the pairs e in [t ppt, min(npairs, (t+1) ppt)) of thread t
template <int PR, class OP>
__global__ void __launch_bounds__(128) k_ranlxd_pairs(const int64_t *__restrict__ words, int skip, int64_t npairs,
                                                      int64_t ppt, OP op) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t e = t * ppt;
  if (e >= npairs) return;
  const int64_t hi = min(npairs, e + ppt);
  int64_t x[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) x[k] = words[12 * t + k];
  int64_t c = 0;
  constexpr double kUnit = 3.552713678800501e-15;  // 2^-48
  int from = skip;
  while (e < hi) {
    swb_refill<PR>(x, c);
#pragma unroll
    for (int j = 0; j < 6; ++j)
      if (2 * j >= from && e < hi) {
        op(e, kUnit * (double)x[2 * j], kUnit * (double)x[2 * j + 1]);
        ++e;
      }
    from = 0;
  }
}

// the real part of the complex Box-Muller normal of a pair, in the host's
// expression (random.f90:238-255, gauge:1334-1340)
__device__ __forceinline__ double box_muller_re(double u1, double u2) {
  constexpr double kTwoPi = 6.283185307179586;  // 2 acos(-1) in FP64
  return sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
}

// the transverse box initial condition: pair e = 16 s + 8 pol + a goes to
// plane (e % 16) of the normals at site e / 16 (real part, imaginary zero)
struct BoxPairs {
  double2 *R;
  int64_t V;
  __device__ void operator()(int64_t e, double u1, double u2) const {
    R[(e % 16) * V + e / 16] = make_double2(box_muller_re(u1, u2), 0.0);
  }
};
// the thermal field of EquilibriumInit: pair i is entry i of the
// reference's efield(8, 3, V) (i = (site*3 + dir)*8 + a), times sigma a0,
// written straight into the device plane (dir*8 + a)
struct ThermalPairs {
  double *E;
  int64_t V;
  double sigma, a0;
  __device__ void operator()(int64_t i, double u1, double u2) const {
    E[(i % 24) * V + i / 24] = (sigma * box_muller_re(u1, u2)) * a0;
  }
};
// the stream itself, or its Box-Muller normals (the generator's test)
struct UniformPairs {
  double *out;
  __device__ void operator()(int64_t e, double u1, double u2) const {
    out[2 * e] = u1;
    out[2 * e + 1] = u2;
  }
};
struct NormalPairs {
  double *out;
  __device__ void operator()(int64_t e, double u1, double u2) const { out[e] = box_muller_re(u1, u2); }
};

// Draw npairs pairs from number `first` (even) of the stream of (level,
// seed) on ctx's stream and apply op to each on the device.  Returns an NRQ
// status; the call waits for the draw before it frees the starting states.
template <class OP>
int device_draw_pairs(nrq_ctx *ctx, int level, int64_t seed, uint64_t first, int64_t npairs, const OP &op) {
  if ((first & 1) || npairs < 0 || (level != 1 && level != 2)) return NRQ_ERR_BAD_ARG;
  if (npairs == 0) return NRQ_OK;
  const int64_t target = (int64_t)ctx->sm_count * 128;  // threads
  const int64_t ppt = 6 * std::max<int64_t>(1, (npairs + 6 * target - 1) / (6 * target));
  const int64_t nthreads = (npairs + ppt - 1) / ppt;
  std::vector<int64_t> words((size_t)nthreads * 12);
  if (!nrqh::block_states(level, seed, first / 12, (uint64_t)(2 * ppt / 12), (size_t)nthreads, words.data())) {
    ctx->last_error = "ranlxd: the random stream could not be positioned";
    return NRQ_ERR_BAD_ARG;
  }
  int64_t *dw = nullptr;
  NRQ_CUDA_TRY(ctx, cudaMalloc(&dw, sizeof(int64_t) * words.size()));
  cudaError_t e = cudaMemcpyAsync(dw, words.data(), sizeof(int64_t) * words.size(), cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess) {
    const unsigned grid = (unsigned)((nthreads + 127) / 128);
    const int skip = (int)(first % 12);
    if (level == 2)
      k_ranlxd_pairs<397><<<grid, 128, 0, ctx->stream>>>(dw, skip, npairs, ppt, op);
    else
      k_ranlxd_pairs<202><<<grid, 128, 0, ctx->stream>>>(dw, skip, npairs, ppt, op);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(dw);
  if (e != cudaSuccess) {
    ctx->last_error = std::string("ranlxd draw: ") + cudaGetErrorString(e);
    return NRQ_ERR_CUDA;
  }
  return NRQ_OK;
}

}  // namespace nrq
