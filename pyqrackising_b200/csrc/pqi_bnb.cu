// libpqi: one batch of branch-and-bound frontier nodes for the exact solver
// (the parallel kernels of solve_maxcut_bnb.py:47-121, used by the B&B loop of
// solve_maxcut_bnb.py:128-199).
//
// One thread per frontier node. A node is n int8 entries (-1 free, 0 / 1
// fixed), stored node-minor ([n][count]) so a warp's reads of entry i are one
// coalesced load; every thread of a warp reads the same W element at the same
// step (a broadcast). Each sum runs in the reference's order (i ascending, then
// j ascending) in float64 with float32 weights, so bounds, leaf values and
// scores are the reference's values bit for bit:
//   bound  = sum over i < j, W_ij != 0 of: W_ij if both fixed and different,
//            0 if both fixed and equal, max(W_ij, 0) otherwise (:47-71);
//   then, unless bound <= best_value + 1e-9 (pruned, :156-158):
//   leaf   (no free entry): cut = sum of W_ij != 0 over differing pairs
//            (:74-84), or energy = sum of (equal ? -W_ij : W_ij) (:87-97);
//   interior: the branch variable = first free i with the largest
//            sum over free j != i of |W_ij| (:100-121, np.argmax).
#include "pqi_common.cuh"

namespace pqi {

__global__ void bnb_eval_kernel(const float* __restrict__ W, int n, const int8_t* __restrict__ fv,
                                int count, double best_value, int spin, double* __restrict__ ub,
                                double* __restrict__ leaf_value, int* __restrict__ branch_var,
                                int8_t* __restrict__ state) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= count) return;
  const size_t B = (size_t)count;
  double total = 0.0;
  bool leaf = true;
  for (int i = 0; i < n; ++i) {
    const int fi = fv[(size_t)i * B + b];
    if (fi < 0) leaf = false;
    const float* __restrict__ row = W + (size_t)i * n;
    for (int j = i + 1; j < n; ++j) {
      const float w = __ldg(row + j);
      if (w == 0.0f) continue;
      const int fj = fv[(size_t)j * B + b];
      if (fi >= 0 && fj >= 0) {
        if (fi != fj) total += (double)w;
      } else if (w > 0.0f) {
        total += (double)w;
      }
    }
  }
  ub[b] = total;
  if (total <= best_value + 1e-9) {
    state[b] = 0;  // pruned
    return;
  }
  if (leaf) {
    double v = 0.0;
    for (int i = 0; i < n; ++i) {
      const int fi = fv[(size_t)i * B + b];
      const float* __restrict__ row = W + (size_t)i * n;
      for (int j = i + 1; j < n; ++j) {
        const float w = __ldg(row + j);
        const int fj = fv[(size_t)j * B + b];
        if (spin) {
          v += (fi == fj) ? -(double)w : (double)w;
        } else if (w != 0.0f && fi != fj) {
          v += (double)w;
        }
      }
    }
    leaf_value[b] = v;
    state[b] = 1;
    return;
  }
  double best_s = -2.0;  // fixed entries score -1.0, free ones >= 0
  int best_i = 0;
  for (int i = 0; i < n; ++i) {
    double s = -1.0;
    if (fv[(size_t)i * B + b] < 0) {
      s = 0.0;
      for (int j = 0; j < n; ++j) {
        if (j == i || fv[(size_t)j * B + b] >= 0) continue;
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        s += (double)fabsf(__ldg(W + (size_t)lo * n + hi));
      }
    }
    if (s > best_s) {  // first maximum, as np.argmax
      best_s = s;
      best_i = i;
    }
  }
  branch_var[b] = best_i;
  state[b] = 2;
}

}  // namespace pqi

using namespace pqi;

extern "C" {

pqi_status pqi_bnb_eval(const float* W, int n, const int8_t* fixed_t, int count, double best_value,
                        int is_spin_glass, double* ub, double* leaf_value, int* branch_var,
                        int8_t* state, void* stream) {
  PQI_CHECK_ARG(W && fixed_t && ub && leaf_value && branch_var && state && n > 0 && count > 0);
  const int threads = 128;
  bnb_eval_kernel<<<(count + threads - 1) / threads, threads, 0, as_stream(stream)>>>(
      W, n, fixed_t, count, best_value, is_spin_glass ? 1 : 0, ub, leaf_value, branch_var, state);
  PQI_LAUNCHED("bnb_eval_kernel");
  return PQI_OK;
}

}  // extern "C"
