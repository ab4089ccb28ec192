// sa_noalloc.cu -- energy measurement that allocates nothing.
//
// sa_measure_noalloc() computes the same exact per-replica E and M as
// sa_sys_measure(), but its scratch (one 128-counter partial per block) lives
// in a file-scope __device__ array instead of memory obtained from cudaMalloc.
// It exists for callers that cannot allocate device memory at the point they
// need an energy: a process that reserved its whole HBM budget up front and
// treats any further driver allocation as a failure, or a hot loop that must
// not pay cudaMalloc/cudaFree's latency and implicit device synchronisation.
// The caller owns every input and output buffer.
//
// The array is reached from host code only through its device address,
// obtained once per device with cudaGetSymbolAddress (the host-side symbol is
// a stand-in, not a device pointer).
#include <cuda_runtime.h>

#include <mutex>

#include "sa_b200.h"
#include "sa_device.cuh"
#include "sa_host.hpp"
#include "sa_measure.cuh"

namespace sa {

// Maximum number of measurement blocks, i.e. of 128-counter partials.
constexpr int kNoAllocMaxBlocks = 512;

// 512 blocks x 128 counters x 4 bytes = 256 KB on every device that loads the
// library, kept until the process exits.
static __device__ __align__(256) unsigned int g_noalloc_partials[kNoAllocMaxBlocks * 128];

constexpr int kNoAllocMaxDevices = 64;
static unsigned int* g_scratch_ptr[kNoAllocMaxDevices];
static std::once_flag g_scratch_once[kNoAllocMaxDevices];
static cudaError_t g_scratch_err[kNoAllocMaxDevices];

// Each block writes its own 128 partial counts (every entry, so nothing in the
// shared array needs clearing between calls).
__global__ void __launch_bounds__(kMeasureThreads) k_measure_partials(const word_t* __restrict__ s,
                                                                      const word_t* __restrict__ J, int L,
                                                                      int lattice, unsigned int* partials) {
  __shared__ unsigned int sm[128];
  measure_block_counts(s, J, L, lattice, sm);
  for (int i = threadIdx.x; i < 128; i += blockDim.x) partials[blockIdx.x * 128 + i] = sm[i];
}

__global__ void k_measure_sum(const unsigned int* partials, int nblocks, long nbonds, long N, int64_t* E,
                              int64_t* M) {
  const int i = threadIdx.x;
  if (i >= 128) return;
  unsigned long long v = 0;
  for (int b = 0; b < nblocks; ++b) v += partials[b * 128 + i];
  if (i < 64) E[i] = 2 * (int64_t)v - nbonds;
  else M[i - 64] = 2 * (int64_t)v - N;
}

}  // namespace sa

using namespace sa;

extern "C" int sa_measure_noalloc(int lattice, int L, const uint64_t* d_spins, const uint64_t* d_J,
                                  int64_t* d_E, int64_t* d_M, void* stream) {
  if (lattice < 0 || lattice > 2) return fail(SA_ERR_INVALID, "unknown lattice kind");
  if (L < 2 || (L & 1)) return fail(L & 1 ? SA_ERR_ODD_L : SA_ERR_INVALID, "L must be even and >= 2");
  if (!d_spins || !d_J || !d_E || !d_M) return fail(SA_ERR_INVALID, "null buffer");
  const int dim = lattice_dim(lattice);
  const long N = (dim == 3) ? (long)L * L * L : (long)L * L;
  const long per_block = (long)kMeasureThreads * kMeasureMaxSitesPerThread;
  const long min_nb = (N + per_block - 1) / per_block;
  if (min_nb > kNoAllocMaxBlocks)
    return fail(SA_ERR_BUDGET, "lattice too large for sa_measure_noalloc: at most " +
                                   std::to_string((long)kNoAllocMaxBlocks * per_block) + " sites");
  int dev = 0;
  SA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(SA_ERR_UNSUPPORTED, "device index out of range");
  // First call on this device: resolve the array's device address (the device
  // is current here); later calls reuse it.
  std::call_once(g_scratch_once[dev], [dev]() {
    g_scratch_err[dev] = cudaGetSymbolAddress((void**)&g_scratch_ptr[dev], g_noalloc_partials);
  });
  if (g_scratch_err[dev] != cudaSuccess) return cuda_fail(g_scratch_err[dev], "cudaGetSymbolAddress");
  long nb = (N + kMeasureThreads * 8 - 1) / (kMeasureThreads * 8);
  if (nb > kNoAllocMaxBlocks) nb = kNoAllocMaxBlocks;
  if (nb < min_nb) nb = min_nb;
  if (nb < 1) nb = 1;
  cudaStream_t st = (cudaStream_t)stream;
  const long nbonds = (long)dim * N - (lattice == SA_LATTICE_2D_OPEN_X ? L : 0);
  k_measure_partials<<<(unsigned)nb, kMeasureThreads, 0, st>>>((const word_t*)d_spins, (const word_t*)d_J, L,
                                                                lattice, g_scratch_ptr[dev]);
  SA_CUDA_TRY(cudaGetLastError());
  k_measure_sum<<<1, 128, 0, st>>>(g_scratch_ptr[dev], (int)nb, nbonds, N, d_E, d_M);
  SA_CUDA_TRY(cudaGetLastError());
  return SA_OK;
}
