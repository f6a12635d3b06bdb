// libpqi: batched cut scoring (replaces calculate_cut, kernels.cl:64-94, and the
// host argmax of run_cut_opencl, maxcut_tfim.py:212-285).
//
// With x = 2s - 1 and W symmetric with a zero diagonal, every candidate's
// value follows from q = x^T W x:
//   cut  (sum_{u<v} W_uv [s_u != s_v])           = (2 S - q) / 4
//   spin (sum_{u<v} W_uv (s_u != s_v ? 1 : -1))  = -q / 2
// where S = sum_{u<v} W_uv. q is the row-dot of X with Y = X W, so the batch is
// one GEMM plus an epilogue. This file holds the CUDA-core tiled path; the
// tensor-core (tcgen05) path lives in pqi_score_tc.cu and shares the finish
// kernel below. A failed tensor-core launch (a bounded wait that expired)
// surfaces as NaN values and best_index -1.
#include <algorithm>

#include "pqi_common.cuh"

namespace pqi {

constexpr int kBM = 64, kBN = 64, kBK = 32;

// grid (ceil(n/64) column tiles, ceil(shots/64) row tiles), 256 threads.
// qpart[tile_n * shots + b] = sum over the tile's 64 columns j of x_bj * Y_bj.
template <typename WT, typename AT>
__global__ void __launch_bounds__(256) xw_rowdot_kernel(const WT* __restrict__ Wp, int ld, int n,
                                                        const uint32_t* __restrict__ theta,
                                                        int n32, int shots,
                                                        double* __restrict__ qpart) {
  __shared__ AT xs[kBK][kBM];
  __shared__ AT wsm[kBK][kBN];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int b0 = blockIdx.y * kBM, j0 = blockIdx.x * kBN;
  AT acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = (AT)0;

  for (int v0 = 0; v0 < n; v0 += kBK) {
    // X tile: word (v0 >> 5) of each of the 64 candidates -> 32 values of +-1
    if (threadIdx.x < kBM) {
      const int b = b0 + threadIdx.x;
      const uint32_t wd = b < shots ? theta[(size_t)b * n32 + (v0 >> 5)] : 0u;
#pragma unroll 8
      for (int kk = 0; kk < kBK; ++kk) xs[kk][threadIdx.x] = ((wd >> kk) & 1u) ? (AT)1 : (AT)-1;
    }
    // W tile: rows v0..v0+31, columns j0..j0+63 (rows >= n read as 0)
    for (int e = threadIdx.x; e < kBK * kBN; e += 256) {
      const int kk = e >> 6, jj = e & 63;
      const int v = v0 + kk;
      wsm[kk][jj] = v < n ? (AT)Wp[(size_t)v * ld + j0 + jj] : (AT)0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kBK; ++kk) {
      AT xa[4], wb[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) xa[a] = xs[kk][ty * 4 + a];
#pragma unroll
      for (int c = 0; c < 4; ++c) wb[c] = wsm[kk][tx * 4 + c];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] += xa[a] * wb[c];
    }
    __syncthreads();
  }
  // epilogue: row-dot with x over this tile's columns
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int b = b0 + ty * 4 + a;
    double part = 0.0;
    if (b < shots) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int j = j0 + tx * 4 + c;
        if (j < n) {
          const int xj = (theta[(size_t)b * n32 + (j >> 5)] >> (j & 31)) & 1u;
          part += xj ? (double)acc[a][c] : -(double)acc[a][c];
        }
      }
    }
    // reduce over the 16 threads (tx) sharing this row: a half-warp
    for (int o = 8; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
    if (tx == 0 && b < shots) qpart[(size_t)blockIdx.x * shots + b] = part;
  }
}

// Sum the column-tile partials in a fixed order, convert to the reference's
// value, store it and fold it into the selection key.
__global__ void score_finish_kernel(const double* __restrict__ qpart, int tiles, int shots,
                                    double upper_sum, int spin, SelGeom geo,
                                    float* __restrict__ energies, unsigned long long* key,
                                    const int* __restrict__ err) {
  __shared__ uint64_t scratch[32];
  uint64_t best = 0;
  const bool failed = err && *err;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < shots; b += gridDim.x * blockDim.x) {
    double q = 0.0;
    for (int t = 0; t < tiles; ++t) q += qpart[(size_t)t * shots + b];
    const double val = spin ? -q / 2.0 : (2.0 * upper_sum - q) / 4.0;
    const float v = failed ? __int_as_float(0x7FC00000) : (float)val;  // NaN marks a failed GEMM
    if (energies) energies[b] = v;
    const uint64_t k = sel_key(v, (uint64_t)b, geo);
    best = k > best ? k : best;
  }
  best = block_max_u64(best, scratch);
  if (threadIdx.x == 0 && best) atomicMax(key, (unsigned long long)best);
}

__global__ void score_select_finish_kernel(const unsigned long long* key, SelGeom geo,
                                           float* best_val, int* best_idx,
                                           const int* __restrict__ err) {
  float v;
  int64_t i;
  sel_decode(*key, geo, &v, &i);
  if (err && *err) {
    v = __int_as_float(0x7FC00000);
    i = -1;
  }
  if (best_val) *best_val = v;
  if (best_idx) *best_idx = (int)i;
}

pqi_status score_finish(const double* qpart, int tiles, int shots, double upper_sum, int spin,
                        const SelGeom& geo, float* energies, unsigned long long* key,
                        float* best_energy, int* best_index, const int* err, cudaStream_t s) {
  PQI_TRY(cudaMemsetAsync(key, 0, sizeof(unsigned long long), s));
  const int grid = std::max(1, std::min((shots + 255) / 256, 148 * 4));
  score_finish_kernel<<<grid, 256, 0, s>>>(qpart, tiles, shots, upper_sum, spin, geo, energies,
                                           key, err);
  PQI_LAUNCHED("score_finish_kernel");
  score_select_finish_kernel<<<1, 1, 0, s>>>(key, geo, best_energy, best_index, err);
  PQI_LAUNCHED("score_select_finish_kernel");
  return PQI_OK;
}

pqi_status score_simt(const pqi_weights* w, const uint32_t* theta, int shots, double* qpart,
                      cudaStream_t s) {
  const int n = w->n, n32 = (n + 31) >> 5;
  dim3 grid((n + kBN - 1) / kBN, (shots + kBM - 1) / kBM);
  if (w->kind == PQI_W_I8) {
    xw_rowdot_kernel<int8_t, int><<<grid, 256, 0, s>>>(w->W_i8, w->ld, n, theta, n32, shots, qpart);
  } else {
    xw_rowdot_kernel<float, float><<<grid, 256, 0, s>>>(w->W_f32z, w->ld, n, theta, n32, shots,
                                                         qpart);
  }
  PQI_LAUNCHED("xw_rowdot_kernel");
  return PQI_OK;
}

// Set by pqi_score_set_path: 0 = automatic (tensor cores when available, CTA
// pairs fed by a separate expansion pass), 1 = CUDA cores only, 2 = single
// CTAs, 3 = CTA pairs (as 0), 4 = as 0 with float weights as split bf16,
// 5 = single CTAs that expand the candidates themselves. Used by tests to
// compare the paths.
int g_score_path = 0;

pqi_status score_tc(const pqi_weights* w, const uint32_t* theta, int shots, int spin,
                    const SelGeom& geo, float* energies, float* best_energy, int* best_index,
                    Workspace& ws, cudaStream_t s);

// Optional events recorded around the scoring GEMM launch (bench timing).
cudaEvent_t g_score_ev_before = nullptr, g_score_ev_after = nullptr;

// Set by pqi_score_set_grid: CTAs of the persistent tensor-core scoring kernel
// (0 = one per SM).
int g_score_grid = 0;

}  // namespace pqi

using namespace pqi;

extern "C" {

pqi_status pqi_score_set_path(int path) {
  if (path < 0 || path > 5) return PQI_EINVAL;
  g_score_path = path;
  return PQI_OK;
}

pqi_status pqi_score_set_events(void* before, void* after) {
  g_score_ev_before = reinterpret_cast<cudaEvent_t>(before);
  g_score_ev_after = reinterpret_cast<cudaEvent_t>(after);
  return PQI_OK;
}

pqi_status pqi_score_set_grid(int ctas) {
  if (ctas < 0) return PQI_EINVAL;
  g_score_grid = ctas;
  return PQI_OK;
}

pqi_status pqi_calculate_cut(const pqi_weights* w, const uint32_t* theta, int shots,
                             int is_spin_glass, int global_size, int local_size,
                             float* energies, float* best_energy, int* best_index,
                             void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(w && theta && shots > 0 && w->n > 0);
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(shots, global_size, local_size, &geo));
  cudaStream_t s = as_stream(stream);
  Workspace ws(workspace, workspace_bytes);
  unsigned long long* key = ws.take<unsigned long long>(1);
  PQI_CHECK_ARG(key);
  if (g_score_path != 1) {
    pqi_status rc = score_tc(w, theta, shots, is_spin_glass, geo, energies, best_energy,
                             best_index, ws, s);
    if (rc != PQI_ENOTSUP) return rc;
  }
  const int tiles = (w->n + kBN - 1) / kBN;
  double* qpart = ws.take<double>((size_t)tiles * shots);
  PQI_CHECK_ARG(qpart);
  if (g_score_ev_before) PQI_TRY(cudaEventRecord(g_score_ev_before, s));
  pqi_status rc = score_simt(w, theta, shots, qpart, s);
  if (g_score_ev_after) PQI_TRY(cudaEventRecord(g_score_ev_after, s));
  if (rc != PQI_OK) return rc;
  const int* err = nullptr;
  return score_finish(qpart, tiles, shots, w->upper_sum, is_spin_glass, geo, energies, key,
                      best_energy, best_index, err, s);
}

}  // extern "C"
