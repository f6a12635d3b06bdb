// libpqi: exhaustive search for n < 24 (replaces exact_maxcut / exact_spin_glass,
// pyqrackising/maxcut_tfim.py:288-339, which the reference runs below its
// heuristic threshold). One thread per mask; each value is summed in float64 in
// the reference's order (i ascending, j > i ascending), so values are
// bit-identical to the reference's. The reference keeps the first mask whose
// value beats the running best, starting from (-1.0, mask 0); that is the
// smallest mask attaining the maximum if the maximum exceeds -1.0, else mask 0.
#include <algorithm>

#include "pqi_common.cuh"

namespace pqi {

__device__ __forceinline__ unsigned long long ord_f64(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double exact_value(const float* Ws, int n, unsigned mask, int spin) {
  double cut = 0.0;
  for (int i = 0; i < n; ++i) {
    const unsigned bi = (mask >> i) & 1u;
    for (int j = i + 1; j < n; ++j) {
      const double v = (double)Ws[i * n + j];
      const unsigned bj = (mask >> j) & 1u;
      if (spin) {
        cut += (bi == bj) ? v : -v;  // exact_spin_glass: +val for equal bits (maxcut_tfim.py:329)
      } else if (bi != bj) {
        cut += v;
      }
    }
  }
  return cut;
}

__global__ void exact_max_kernel(const float* __restrict__ W, int n, int spin,
                                 unsigned long long* best_ord) {
  __shared__ float Ws[32 * 32];
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) Ws[e] = W[e];
  __syncthreads();
  const unsigned total = 1u << n;
  unsigned long long best = 0;
  for (unsigned m = blockIdx.x * blockDim.x + threadIdx.x; m < total; m += gridDim.x * blockDim.x) {
    const unsigned long long o = ord_f64(exact_value(Ws, n, m, spin));
    best = o > best ? o : best;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long x = __shfl_xor_sync(0xFFFFFFFFu, best, o);
    best = x > best ? x : best;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(best_ord, best);
}

__global__ void exact_argmin_kernel(const float* __restrict__ W, int n, int spin,
                                    const unsigned long long* best_ord, unsigned* best_mask) {
  __shared__ float Ws[32 * 32];
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) Ws[e] = W[e];
  __syncthreads();
  const unsigned total = 1u << n;
  const unsigned long long target = *best_ord;
  unsigned found = 0xFFFFFFFFu;
  for (unsigned m = blockIdx.x * blockDim.x + threadIdx.x; m < total; m += gridDim.x * blockDim.x) {
    if (ord_f64(exact_value(Ws, n, m, spin)) == target) {
      found = m;
      break;  // masks of one thread ascend
    }
  }
  for (int o = 16; o > 0; o >>= 1) found = min(found, __shfl_xor_sync(0xFFFFFFFFu, found, o));
  if ((threadIdx.x & 31) == 0 && found != 0xFFFFFFFFu) atomicMin(best_mask, found);
}

__global__ void exact_finish_kernel(const unsigned long long* best_ord, const unsigned* best_mask,
                                    double* best_value, int* mask_out) {
  const unsigned long long o = *best_ord;
  const unsigned long long b = (o & 0x8000000000000000ull) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
  const double v = __longlong_as_double((long long)b);
  if (v > -1.0) {
    *best_value = v;
    *mask_out = (int)*best_mask;
  } else {
    *best_value = -1.0;
    *mask_out = 0;
  }
}

}  // namespace pqi

using namespace pqi;

extern "C" pqi_status pqi_exact_search(const float* W, int n, int is_spin_glass,
                                       double* best_value, int* best_mask, void* workspace,
                                       size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(W && best_value && best_mask && n >= 1 && n <= 30);
  Workspace ws(workspace, workspace_bytes);
  unsigned long long* ord = ws.take<unsigned long long>(1);
  unsigned* mask = ws.take<unsigned>(1);
  PQI_CHECK_ARG(ord && mask);
  cudaStream_t s = as_stream(stream);
  PQI_TRY(cudaMemsetAsync(ord, 0, sizeof(*ord), s));
  PQI_TRY(cudaMemsetAsync(mask, 0xFF, sizeof(*mask), s));
  const long long total = 1ll << n;
  const int grid = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 16));
  exact_max_kernel<<<grid, 256, 0, s>>>(W, n, is_spin_glass, ord);
  PQI_LAUNCHED("exact_max_kernel");
  exact_argmin_kernel<<<grid, 256, 0, s>>>(W, n, is_spin_glass, ord, mask);
  PQI_LAUNCHED("exact_argmin_kernel");
  exact_finish_kernel<<<1, 1, 0, s>>>(ord, mask, best_value, best_mask);
  PQI_LAUNCHED("exact_finish_kernel");
  return PQI_OK;
}
