// Shared-memory staging helpers of the persistent stencil kernels
// (cn_mv3.cu, cn_mv4.cu): mbarriers with bounded waits, 2D tensor-map copies
// (cp.async.bulk.tensor) and 1D bulk copies (cp.async.bulk) into shared
// memory that complete on an mbarrier, 2D tensor-map stores from shared
// memory (bulk async-groups), explicit shared-memory loads and stores, and
// the host-side encoder of 2D FP64 tensor maps.
//
// Single-GPU code: every copy reads this GPU's own memory and no copy uses
// cluster multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include "nrq_common.cuh"
#include "../../include/nrqcd_b200.h"

namespace nrq {

// ~2 s at 2 GHz: bound of every mbarrier wait of the staged kernels
constexpr long long kStageWaitCycles = 4000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
// 16-byte complex load from a shared-memory address (ld.shared, never generic)
__device__ __forceinline__ cplx lds2(uint32_t a) {
  double re, im;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(re), "=d"(im) : "r"(a));
  return {re, im};
}
__device__ __forceinline__ double lds1(uint32_t a) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; returns false on expiry
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > kStageWaitCycles) return false;
  }
  return true;
}
// Record an expired pipeline wait: err[0] = NRQ_ERR_TIMEOUT; the first
// expiry of a launch also records where (err[1] = stencil * 16 + role,
// err[2] = the load's index in its CTA, err[3] = the CTA).  Roles: 0 a
// consumer's wait for a load, 1 for the diagonal matrices, 2 the loader's
// wait for a released buffer, 3 for a landed load, 4 its final drain.
__device__ __forceinline__ void record_timeout(int *err, int stencil, int role, int load) {
  atomicExch(err, NRQ_ERR_TIMEOUT);
  if (atomicCAS(err + 1, 0, stencil * 16 + role) == 0) {
    atomicExch(err + 2, load);
    atomicExch(err + 3, (int)blockIdx.x);
  }
}

// 2D tile of a tensor map at (c0, c1) into shared memory
__device__ __forceinline__ void tma_2d(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}
// 2D tile from shared memory to a tensor map at (c0, c1) (bulk async-group
// of the issuing thread; c0, c1 >= 0; elements outside the tensor are not
// written)
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, int c0, int c1, const void *src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"((uint64_t)map),
               "r"(c0), "r"(c1), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the issuing thread's committed bulk stores have read their shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// this thread's shared-memory writes become visible to later bulk copies
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void sts2(uint32_t a, double re, double im) {
  asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(re), "d"(im) : "memory");
}
__device__ __forceinline__ void sts2f(uint32_t a, float re, float im) {
  asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(re), "f"(im) : "memory");
}
// barrier `id` (1-15) among the first `nthreads` threads of the CTA (whole warps)
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// contiguous copy of `bytes` (multiple of 16; both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_1d(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

namespace stage {
inline PFN_cuTensorMapEncodeTiled_v12000 get_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 2D map over `planes` planes of `elems_per_plane` elements (FP64 unless
// dt says FP32; plane stride = elems)
inline bool encode(CUtensorMap *m, const void *base, uint64_t elems_per_plane, uint64_t planes, uint32_t box0,
                   uint32_t box1, CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_NONE,
                   CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64) {
  auto fn = get_encoder();
  if (!fn) return false;
  const uint64_t esize = dt == CU_TENSOR_MAP_DATA_TYPE_FLOAT32 ? 4 : 8;
  cuuint64_t dims[2] = {elems_per_plane, planes};
  cuuint64_t strides[1] = {elems_per_plane * esize};
  cuuint32_t box[2] = {box0, box1};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(m, dt, 2, const_cast<void *>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}
}  // namespace stage

}  // namespace nrq
