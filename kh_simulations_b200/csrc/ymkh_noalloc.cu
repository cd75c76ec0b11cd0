// ymkh_noalloc.cu — total energy of a caller-bound state with no device
// allocation by the library.
//
// Who needs it.  ymkh_energy / ymkh_energy_async need a context, and
// ymkh_create cudaMalloc's the per-CTA partial sums of the reduction (plus
// the step's own buffers).  Some callers cannot let the library allocate:
//  * a host whose device memory is carved out by its own arena up front
//    (a serving process that admits runs against a fixed byte budget counts
//    every byte it hands out; a hidden cudaMalloc breaks that accounting and
//    can fail once the arena holds the rest of the GPU);
//  * a latency-critical loop on several streams, where cudaMalloc/cudaFree
//    can synchronise the device and stall the other streams;
//  * code that only holds the 24 state arrays (bound by another framework)
//    and has no context to create.
// For them this entry point keeps the partial sums in a file-scope
// __device__ array of fixed size, and allocates nothing.
//
// The reduction is the one ymkh_energy_async runs (same kernels, same
// partition into CTA blocks, same Neumaier order: ymgpu2d/YM_Energy.cu:3-21
// per cell), so the two return bit-identical totals for the same state.
//
// Limit: nx * nz <= YMKH_NOALLOC_MAX_CELLS (134,217,728 cells; the scratch
// holds 32,768 (sum, compensation) pairs, 512 KiB).  Larger grids are
// rejected with YMKH_EINVAL before anything is launched.
//
// Nothing in the scratch needs to start at zero: the partial kernel writes
// every (sum, compensation) pair the final kernel reads, in stream order,
// so the array is never cleared.
//
// Set-up: the first call on each device (with that device current) looks up
// the scratch's device address with cudaGetSymbolAddress, checks the result
// and caches it for that device; later calls reuse it.  The lookup can make
// the runtime load this module onto the device, so make the first call on a
// device before any stream capture begins.  The cached address belongs to
// the device's primary context, the one the CUDA runtime uses: a caller that
// makes its own driver-API context current, or that calls cudaDeviceReset
// after the first call, must not use this entry point afterwards (the cache
// would hand out an address of another or a destroyed context).
//
// Concurrency: all calls on one device share the one scratch array.  Two
// calls whose kernels may overlap (different streams, or different host
// threads without ordering) race on it and can return wrong totals; issue
// them on one stream, or one after another.

#include "ymkh_common.cuh"

#include <atomic>
#include <cstdio>

namespace {

constexpr int kNoallocMaxParts = 32768;
constexpr size_t kNoallocMaxCells = (size_t)YMKH_NOALLOC_MAX_CELLS;
constexpr int kMaxDevices = 64;

// (sum, compensation) per CTA of the energy reduction.
static __device__ __align__(256) double g_energy_scratch[2 * kNoallocMaxParts];

std::atomic<double*> g_scratch_addr[kMaxDevices];

}  // namespace

extern "C" int ymkh_energy_noalloc(double* const* state, int nx, int nz, double* dev_out, void* stream) {
  using namespace ymkh;
  if (!state || !dev_out) return capi_error(YMKH_EINVAL, "ymkh_energy_noalloc: null argument");
  if (nx <= 0 || nz <= 0) return capi_error(YMKH_EINVAL, "ymkh_energy_noalloc: nx and nz must be > 0");
  const size_t N = (size_t)nx * (size_t)nz;
  if (N > kNoallocMaxCells || energy_nparts(N) > kNoallocMaxParts) {
    char msg[200];
    snprintf(msg, sizeof msg,
             "ymkh_energy_noalloc: nx*nz = %zu cells exceeds the static scratch limit of %zu cells", N,
             kNoallocMaxCells);
    return capi_error(YMKH_EINVAL, msg);
  }
  for (int i = 0; i < YMKH_NSTATE; ++i)
    if (!state[i]) return capi_error(YMKH_EINVAL, "ymkh_energy_noalloc: null state array");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return capi_error(YMKH_ECUDA, "ymkh_energy_noalloc: cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return capi_error(YMKH_EINVAL, "ymkh_energy_noalloc: device index out of range");
  double* part = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!part) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_energy_scratch);
    if (e != cudaSuccess || !p) {
      char msg[200];
      snprintf(msg, sizeof msg, "ymkh_energy_noalloc: cudaGetSymbolAddress of the scratch failed: %s",
               cudaGetErrorString(e));
      return capi_error(YMKH_ECUDA, msg);
    }
    part = static_cast<double*>(p);
    g_scratch_addr[dev].store(part, std::memory_order_release);
  }

  State st;
  for (int i = 0; i < 12; ++i) st.f[i] = state[i];
  for (int i = 0; i < 6; ++i) {
    st.a[i] = state[12 + i];
    st.b[i] = state[18 + i];
  }
  e = launch_energy(st, N, part, dev_out, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof msg, "ymkh_energy_noalloc: energy kernels: %s", cudaGetErrorString(e));
    return capi_error(YMKH_ECUDA, msg);
  }
  capi_count_launches(2);
  return 0;
}
