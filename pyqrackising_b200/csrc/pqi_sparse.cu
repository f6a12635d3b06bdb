// libpqi: device-side expansion of the sparse entry points' coordinate lists to
// the dense matrices the rest of the path runs on. The reference's sparse path
// keeps a CSR of the stored entries (maxcut_tfim_util.py:533-542) and its
// kernels add every stored entry (u, v) once to the cut (kernels.cl:233-251),
// which is the dense form W = S + S^T of the stored entries S; S alone gives the
// sampler's J / degrees (maxcut_tfim_sparse.py:204-224).
#include <algorithm>

#include "pqi_common.cuh"

namespace pqi {

// One thread per stored entry (grid-stride). Diagonal entries are dropped (the
// dense path keeps a zero diagonal). W_rc collects at most the two entries
// (r, c) and (c, r) (coordinates are unique), so the float32 sum is the same in
// either order: the result equals the host's np.add.at over a zero matrix
// followed by S + S^T, signed zeros included.
__global__ void coo_expand_kernel(const int* __restrict__ rows, const int* __restrict__ cols,
                                  const float* __restrict__ vals, long long nnz, int n,
                                  float* __restrict__ S, float* __restrict__ W,
                                  int* __restrict__ bad) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = rows[e], c = cols[e];
    if (r < 0 || r >= n || c < 0 || c >= n) {
      atomicExch(bad, 1);
      continue;
    }
    if (r == c) continue;
    const float v = vals[e];
    if (S) atomicAdd(S + (size_t)r * n + c, v);
    atomicAdd(W + (size_t)r * n + c, v);
    atomicAdd(W + (size_t)c * n + r, v);
  }
}

}  // namespace pqi

using namespace pqi;

extern "C" {

pqi_status pqi_coo_to_dense(const int* rows, const int* cols, const float* vals, long long nnz,
                            int n, float* S, float* W, int* bad, void* stream) {
  PQI_CHECK_ARG(n > 0 && nnz >= 0 && W && bad && (nnz == 0 || (rows && cols && vals)));
  cudaStream_t s = as_stream(stream);
  const size_t bytes = (size_t)n * (size_t)n * sizeof(float);
  PQI_TRY(cudaMemsetAsync(W, 0, bytes, s));
  if (S) PQI_TRY(cudaMemsetAsync(S, 0, bytes, s));
  PQI_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
  if (nnz == 0) return PQI_OK;
  const long long blocks = std::min<long long>((nnz + 255) / 256, 148LL * 32);
  coo_expand_kernel<<<(int)blocks, 256, 0, s>>>(rows, cols, vals, nnz, n, S, W, bad);
  PQI_LAUNCHED("coo_expand_kernel");
  return PQI_OK;
}

}  // extern "C"
