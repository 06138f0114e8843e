// Gauge energy for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc.  A port of the driver that keeps the
// gauge fields in device memory owned by another runtime falls in this group:
// OpenACC or CUDA Fortran data regions, or a framework's caching allocator.
// Such callers must not grow the device footprint or allocate inside their
// time loop.  They still want the energy observable of fields already in
// their own buffers.  nrq_gauge_energy needs a context and a gauge handle,
// and both allocate device memory.  This entry point allocates nothing: the
// caller passes the inputs and the output, and the per-block partial sums
// go into a fixed-size array in the library's own device memory.
//
// The scratch array is a file-scope __device__ array, so every GPU that loads
// this library holds it (128 KiB) until the process exits.  Host code cannot
// use the array's name as a device address.  The first call in each CUDA
// context (one per device unless the caller manages contexts itself) looks
// the address up with cudaGetSymbolAddress, with that device current, and
// caches it under the context's unique id.  After cudaDeviceReset, or under a
// different driver-API context, the module is loaded anew and its address can
// move: the id changes with it, so the next call looks the address up again.
// Make the first call in a context before any stream capture.
//
// Every call shares the one array and leaves its partial sums there.  The
// block-sum kernel writes every slot that the final reduction then reads, so
// nothing has to start at zero.  Calls that overlap on the GPU, from two
// streams or two host threads, race on the array and return wrong sums.
// Serialise them.
#include <mutex>

#include "../../include/nrqcd_b200.h"
#include "nrq_kernels.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = NRQ_NOALLOC_MAX_SITES / kThreads;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_energy_partials[kMaxBlocks];

std::mutex g_mutex;
struct Cached {
  unsigned long long ctx_id;
  double *ptr;
};
Cached g_scratch[kMaxDevices] = {};

// unique id of the current CUDA context (cuCtxGetId, CUDA 12.0+), through
// the runtime's driver entry point so the library needs no -lcuda
using CtxGetCurrentFn = int (*)(void **);
using CtxGetIdFn = int (*)(void *, unsigned long long *);
bool current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void *p = nullptr, *q = nullptr;
    cudaDriverEntryPointQueryResult r1, r2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1) == cudaSuccess &&
        r1 == cudaDriverEntryPointSuccess && cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2) ==
                                                 cudaSuccess && r2 == cudaDriverEntryPointSuccess) {
      get_current = (CtxGetCurrentFn)p;
      get_id = (CtxGetIdFn)q;
    }
    looked_up = true;
  }
  if (!get_current || !get_id) return false;
  void *ctx = nullptr;
  return get_current(&ctx) == 0 && ctx != nullptr && get_id(ctx, id) == 0;
}

// Device address of the scratch array in the current context (set up once
// per context).
int scratch_on_current_device(double **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return NRQ_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_mutex);
  unsigned long long id = 0;
  double *p = nullptr;
  if (!current_context_id(&id)) {
    // no context is current yet: the symbol lookup makes the device's
    // primary context current, then the id is read
    if (cudaGetSymbolAddress((void **)&p, g_energy_partials) != cudaSuccess || p == nullptr ||
        !current_context_id(&id)) {
      cudaGetLastError();  // this call's own error (none was pending before it)
      return NRQ_ERR_CUDA;
    }
    g_scratch[dev].ptr = p;
    g_scratch[dev].ctx_id = id;
  } else if (g_scratch[dev].ptr == nullptr || g_scratch[dev].ctx_id != id) {
    if (cudaGetSymbolAddress((void **)&p, g_energy_partials) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return NRQ_ERR_CUDA;
    }
    g_scratch[dev].ptr = p;
    g_scratch[dev].ctx_id = id;
  }
  *out = g_scratch[dev].ptr;
  return NRQ_OK;
}

}  // namespace

extern "C" int nrq_gauge_energy_noalloc(const int64_t extents[3], const double spacings[4],
                                        const double *links_soa, const double *efield_soa,
                                        double *energy_out, void *stream) {
  if (!extents || !spacings || !links_soa || !efield_soa || !energy_out) return NRQ_ERR_BAD_ARG;
  // every factor and partial product is checked against the cap before the
  // next multiplication, so the site count cannot overflow
  const int64_t cap = (int64_t)NRQ_NOALLOC_MAX_SITES;
  for (int k = 0; k < 3; ++k) {
    if (extents[k] < 1) return NRQ_ERR_BAD_ARG;
    if (extents[k] > cap) return NRQ_ERR_CAPACITY;
  }
  for (int k = 0; k < 4; ++k)
    if (!(spacings[k] > 0.0)) return NRQ_ERR_BAD_ARG;
  const int64_t Vxy = extents[0] * extents[1];
  if (Vxy > cap) return NRQ_ERR_CAPACITY;
  const int64_t V = Vxy * extents[2];
  if (V > cap) return NRQ_ERR_CAPACITY;
  // an error left pending by the caller's earlier work stays the caller's:
  // report it without clearing it
  if (cudaPeekAtLastError() != cudaSuccess) return NRQ_ERR_CUDA;
  double *scratch = nullptr;
  int rc = scratch_on_current_device(&scratch);
  if (rc != NRQ_OK) return rc;
  nrq::Lat L;
  L.nx = extents[0];
  L.ny = extents[1];
  L.nz = extents[2];
  L.V = V;
  L.a0 = spacings[0];
  for (int k = 0; k < 3; ++k) L.a[k] = spacings[k + 1];
  const int64_t nblk = (V + kThreads - 1) / kThreads;
  cudaStream_t st = (cudaStream_t)stream;
  nrq::k_energy<<<(unsigned)nblk, kThreads, 0, st>>>(L, (const double2 *)links_soa, efield_soa, scratch);
  if (cudaGetLastError() != cudaSuccess) return NRQ_ERR_CUDA;
  nrq::k_reduce_final<<<1, 256, 0, st>>>(scratch, nblk, 1, 0u, energy_out);
  if (cudaGetLastError() != cudaSuccess) return NRQ_ERR_CUDA;
  return NRQ_OK;
}
