// Test kernel: the library's div_rn (ymkh_common.cuh) against the IEEE
// division a / b, bit for bit, for one divisor and many numerators.
// Built by tests/test_gpu_division.py with nvcc; not part of the library.
#include "ymkh_common.cuh"

namespace {

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// kind 0: random sign, mantissa and exponent (|a| in [2^-700, 2^700));
// kind 1: a = RN(q * b) for random q, so a / b lies next to a double;
// kind 2: kind 1 moved by one ulp either way (quotients near a rounding tie);
// kind 3: special values (zeros, tiny, huge, infinities, NaN).
__global__ void check(double b, double y, unsigned long long seed, long long n, int kind,
                      unsigned long long* bad, double* first_a) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long h = mix64(seed ^ mix64((unsigned long long)i));
    double a;
    if (kind == 0 || kind == 1 || kind == 2) {
      const unsigned long long mant = h & 0x000FFFFFFFFFFFFFull;
      const unsigned long long e = 1023 - 700 + (mix64(h) % 1400);
      const double x = __longlong_as_double((long long)(((h >> 63) << 63) | (e << 52) | mant));
      if (kind == 0) {
        a = x;
      } else {
        a = x * b;
        if (kind == 2) {
          const long long bits = __double_as_longlong(a);
          a = __longlong_as_double(bits + ((h >> 1) & 1 ? 1 : -1));
        }
      }
    } else {
      // (quotients below 2^-900, where div_rn may differ in the last bit,
      // are left out: denormal numerators do not occur here)
      const double sp[12] = {0.0, -0.0, 0x1p-880, -0x1p-880, 0x1p-700, 0x1p-100, 0x1p900, -0x1p950,
                             __longlong_as_double(0x7FF0000000000000ll), __longlong_as_double(0xFFF0000000000000ll),
                             __longlong_as_double(0x7FF8000000000000ll), 1.0};
      a = sp[i % 12];
    }
    const double got = ymkh::div_rn(a, b, y), want = a / b;
    const bool same = __double_as_longlong(got) == __double_as_longlong(want) || (got != got && want != want);
    if (!same) {
      if (atomicAdd(bad, 1ull) == 0ull) *first_a = a;
    }
  }
}

}  // namespace

extern "C" int div_rn_check(double b, double y, unsigned long long seed, long long n, int kind,
                            unsigned long long* host_bad, double* host_first_a) {
  unsigned long long* d_bad = nullptr;
  double* d_first = nullptr;
  if (cudaMalloc(&d_bad, sizeof(unsigned long long)) != cudaSuccess) return 1;
  if (cudaMalloc(&d_first, sizeof(double)) != cudaSuccess) return 1;
  cudaMemset(d_bad, 0, sizeof(unsigned long long));
  cudaMemset(d_first, 0, sizeof(double));
  check<<<148 * 8, 256>>>(b, y, seed, n, kind, d_bad, d_first);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(host_bad, d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaMemcpy(host_first_a, d_first, sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_bad);
  cudaFree(d_first);
  return e == cudaSuccess ? 0 : 2;
}
