// libpqi: kernels of the learned flip-proposal network (a small message-passing
// net; no reference counterpart). Weights and activations are stored in bf16,
// every product accumulates in float32.
//
//   A_hat = D^-1/2 W D^-1/2 (bf16), D = diag(sum_u |W_vu|)
//   h0 = relu(F A0 + b0);  h_l = relu([h_{l-1}, A_hat h_{l-1}] [A_l; B_l] + b_l)
//   logit = h_3 c + c0;  proposal = softmax(logit)
//
// Kernels: a tiled bf16 GEMM with optional transposes and a fused
// (alpha, beta, bias, ReLU) epilogue that writes float32 and/or bf16; the
// normalised adjacency; node features of a state; softmax cross-entropy with
// its gradient; ReLU backward; column sums (bias gradients); Adam.
#include <cuda_bf16.h>

#include <algorithm>

#include "pqi_common.cuh"

namespace pqi {

namespace mp {

constexpr int TM = 64, TN = 64, TK = 32;

__device__ __forceinline__ float bf(const __nv_bfloat16* p, size_t i) { return __bfloat162float(p[i]); }

// C[M x N] = alpha * op(A)[M x K] * op(B)[K x N] + beta * C32 + bias, then ReLU.
// op(A)[m][k] = transA ? A[k*lda + m] : A[m*lda + k]; likewise B.
__global__ void __launch_bounds__(256) gemm_bf16_kernel(int transA, int transB, int M, int N,
                                                        int K, float alpha,
                                                        const __nv_bfloat16* __restrict__ A,
                                                        int lda,
                                                        const __nv_bfloat16* __restrict__ B,
                                                        int ldb, float beta, float* C32,
                                                        __nv_bfloat16* C16, int ldc,
                                                        const float* __restrict__ bias, int relu) {
  __shared__ float As[TK][TM + 1];
  __shared__ float Bs[TK][TN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int e = threadIdx.x; e < TK * TM; e += 256) {
      const int kk = transA ? e / TM : e % TK, mm = transA ? e % TM : e / TK;
      const int m = m0 + mm, k = k0 + kk;
      float v = 0.0f;
      if (m < M && k < K) v = transA ? bf(A, (size_t)k * lda + m) : bf(A, (size_t)m * lda + k);
      As[kk][mm] = v;
    }
    for (int e = threadIdx.x; e < TK * TN; e += 256) {
      const int kk = transB ? e % TK : e / TN, nn = transB ? e / TK : e % TN;
      const int n = n0 + nn, k = k0 + kk;
      float v = 0.0f;
      if (n < N && k < K) v = transB ? bf(B, (size_t)n * ldb + k) : bf(B, (size_t)k * ldb + n);
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < TK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = alpha * acc[i][j];
      if (beta != 0.0f) v += beta * C32[(size_t)m * ldc + n];
      if (bias) v += bias[n];
      if (relu) v = fmaxf(v, 0.0f);
      if (C32) C32[(size_t)m * ldc + n] = v;
      if (C16) C16[(size_t)m * ldc + n] = __float2bfloat16_rn(v);
    }
  }
}

// row sums of |W| (caller's matrix, pitch n, diagonal ignored)
__global__ void abs_rowsum_kernel(const float* __restrict__ W, int n, float* __restrict__ s) {
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int r = blockIdx.x * warps + (threadIdx.x >> 5); r < n; r += gridDim.x * warps) {
    float acc = 0.0f;
    for (int c = lane; c < n; c += 32)
      if (c != r) acc += fabsf(W[(size_t)r * n + c]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) s[r] = acc;
  }
}

__global__ void norm_adj_kernel(const float* __restrict__ W, int n, const float* __restrict__ s,
                                __nv_bfloat16* __restrict__ Ah, int ld) {
  const size_t total = (size_t)n * ld;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / ld), c = (int)(e - (size_t)r * ld);
    float v = 0.0f;
    if (c < n && c != r) {
      const float d = sqrtf(fmaxf(s[r], 1e-30f) * fmaxf(s[c], 1e-30f));
      v = W[(size_t)r * n + c] / d;
    }
    Ah[e] = __float2bfloat16_rn(v);
  }
}

// features of a state: [x_v, g_v / s_v, s_v / mean(s), 1] (F = 4), bf16
__global__ void features_kernel(const uint32_t* __restrict__ theta, const double* __restrict__ g64,
                                const float* __restrict__ s, float mean_s, int n,
                                __nv_bfloat16* __restrict__ F) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const float x = ((theta[v >> 5] >> (v & 31)) & 1u) ? 1.0f : -1.0f;
    const float sv = fmaxf(s[v], 1e-30f);
    F[(size_t)v * 4 + 0] = __float2bfloat16_rn(x);
    F[(size_t)v * 4 + 1] = __float2bfloat16_rn((float)(g64[v] / sv));
    F[(size_t)v * 4 + 2] = __float2bfloat16_rn(sv / fmaxf(mean_s, 1e-30f));
    F[(size_t)v * 4 + 3] = __float2bfloat16_rn(1.0f);
  }
}

// loss = -sum_v t_v log softmax(z)_v, dz = softmax(z) - t (t sums to 1); one block
__global__ void softmax_xent_kernel(const float* __restrict__ z, const float* __restrict__ t,
                                    int n, float* __restrict__ loss, float* __restrict__ dz,
                                    float* __restrict__ prob) {
  __shared__ float red[32];
  __shared__ float bc;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float mx = -INFINITY;
  for (int v = threadIdx.x; v < n; v += blockDim.x) mx = fmaxf(mx, z[v]);
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
  if (lane == 0) red[w] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = -INFINITY;
    for (int i = 0; i < nw; ++i) m = fmaxf(m, red[i]);
    bc = m;
  }
  __syncthreads();
  mx = bc;
  float se = 0.0f;
  for (int v = threadIdx.x; v < n; v += blockDim.x) se += expf(z[v] - mx);
  for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xFFFFFFFFu, se, o);
  __syncthreads();
  if (lane == 0) red[w] = se;
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.0f;
    for (int i = 0; i < nw; ++i) a += red[i];
    bc = a;
  }
  __syncthreads();
  const float lse = mx + logf(bc);
  float l = 0.0f;
  for (int v = threadIdx.x; v < n; v += blockDim.x) {
    const float p = expf(z[v] - lse);
    if (prob) prob[v] = p;
    const float tv = t ? t[v] : 0.0f;
    if (dz) dz[v] = p - tv;
    l += -tv * (z[v] - lse);
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xFFFFFFFFu, l, o);
  __syncthreads();
  if (lane == 0) red[w] = l;
  __syncthreads();
  if (threadIdx.x == 0 && loss) {
    float a = 0.0f;
    for (int i = 0; i < nw; ++i) a += red[i];
    *loss = a;
  }
}

// dZ = dY * (Z > 0), written as float32 and bf16
__global__ void relu_bwd_kernel(const float* __restrict__ dY, const float* __restrict__ Y,
                                size_t count, float* __restrict__ dZ,
                                __nv_bfloat16* __restrict__ dZ16) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count;
       e += (size_t)gridDim.x * blockDim.x) {
    const float v = Y[e] > 0.0f ? dY[e] : 0.0f;
    dZ[e] = v;
    if (dZ16) dZ16[e] = __float2bfloat16_rn(v);
  }
}

// out[c] (+)= sum_r X[r*ld + c], one warp per column, fixed order
__global__ void colsum_kernel(const float* __restrict__ X, int rows, int cols, int ld,
                              float* __restrict__ out, int accumulate) {
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  for (int c = blockIdx.x * warps + (threadIdx.x >> 5); c < cols; c += gridDim.x * warps) {
    float acc = 0.0f;
    for (int r = lane; r < rows; r += 32) acc += X[(size_t)r * ld + c];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) out[c] = accumulate ? out[c] + acc : acc;
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ x, size_t count,
                               __nv_bfloat16* __restrict__ y) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count;
       e += (size_t)gridDim.x * blockDim.x)
    y[e] = __float2bfloat16_rn(x[e]);
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v,
                            __nv_bfloat16* __restrict__ w16, size_t count, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count;
       e += (size_t)gridDim.x * blockDim.x) {
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.0f - b1) * gg;
    const float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    const float upd = lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    const float nw = w[e] - upd;
    w[e] = nw;
    if (w16) w16[e] = __float2bfloat16_rn(nw);
  }
}

static int grid1(size_t work, int block = 256) {
  return (int)std::max<size_t>(1, std::min<size_t>((work + block - 1) / block, 148 * 16));
}

}  // namespace mp
}  // namespace pqi

using namespace pqi;

// Kick distribution of each task from its logits (one CTA per task): p =
// softmax(logit / T) in float64, mixed with the uniform distribution
// ((1 - mix) p + mix / n), as a normalised cumulative array; any non-finite
// logit makes the task's distribution uniform (the search must not depend on
// the network being right).
__global__ void __launch_bounds__(1024) kick_cdf_kernel(const float* __restrict__ logits, int n,
                                                        double temp, float mix,
                                                        double* __restrict__ cdf) {
  __shared__ double sred[32];
  __shared__ double s_bcast;
  __shared__ int s_bad;
  const float* z = logits + (size_t)blockIdx.x * n;
  double* out = cdf + (size_t)blockIdx.x * n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  // 1. max of z / T (and a non-finite check)
  double m = -INFINITY;
  for (int v = threadIdx.x; v < n; v += blockDim.x) {
    const float x = z[v];
    if (!isfinite(x)) s_bad = 1;
    m = fmax(m, (double)x / temp);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if (lane == 0) sred[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = -INFINITY;
    for (int i = 0; i < nw; ++i) t = fmax(t, sred[i]);
    s_bcast = t;
  }
  __syncthreads();
  const bool uniform = s_bad != 0;
  const double zmax = s_bcast;
  __syncthreads();
  // 2. sum of the unnormalised weights
  double sum = 0.0;
  for (int v = threadIdx.x; v < n; v += blockDim.x)
    sum += uniform ? 1.0 : exp((double)z[v] / temp - zmax);
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
  if (lane == 0) sred[warp] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < nw; ++i) t += sred[i];
    s_bcast = t;
  }
  __syncthreads();
  const double total = s_bcast;
  __syncthreads();
  // 3. running sum in chunks of blockDim, warp scans then the warp totals
  double carry = 0.0;
  for (int base = 0; base < n; base += blockDim.x) {
    const int v = base + threadIdx.x;
    double p = 0.0;
    if (v < n) {
      const double w = uniform ? 1.0 : exp((double)z[v] / temp - zmax);
      p = (1.0 - (double)mix) * (w / total) + (double)mix / (double)n;
    }
    double x = p;
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sred[warp] = x;
    __syncthreads();
    if (warp == 0) {
      double t = lane < nw ? sred[lane] : 0.0;
      for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xFFFFFFFFu, t, o);
        if (lane >= o) t += y;
      }
      if (lane < nw) sred[lane] = t;  // inclusive prefix of the warp totals
    }
    __syncthreads();
    const double before = carry + (warp > 0 ? sred[warp - 1] : 0.0);
    if (v < n) out[v] = before + x;
    carry += sred[nw - 1];
    __syncthreads();
  }
  // 4. normalise by the last entry
  const double last = out[n - 1];
  __syncthreads();
  for (int v = threadIdx.x; v < n; v += blockDim.x) out[v] = out[v] / last;
}

// One block: sum of squares (float64) of count floats, then, when its root
// exceeds max_norm > 0, every element scaled by max_norm / norm.
__global__ void __launch_bounds__(1024) grad_clip_kernel(float* __restrict__ g, size_t count,
                                                         float max_norm, float* __restrict__ norm_out) {
  __shared__ double red[32];
  __shared__ double s_norm;
  double acc = 0.0;
  for (size_t i = threadIdx.x; i < count; i += blockDim.x) acc += (double)g[i] * (double)g[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    s_norm = sqrt(t);
    if (norm_out) *norm_out = (float)s_norm;
  }
  __syncthreads();
  const double norm = s_norm;
  if (max_norm > 0.0f && norm > (double)max_norm) {
    const float scale = (float)((double)max_norm / norm);
    for (size_t i = threadIdx.x; i < count; i += blockDim.x) g[i] *= scale;
  }
}

// Sum of count floats in float64 (one block, fixed order).
__global__ void __launch_bounds__(1024) sum_kernel(const float* __restrict__ x, size_t count,
                                                   double* __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (size_t i = threadIdx.x; i < count; i += blockDim.x) acc += (double)x[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    *out = t;
  }
}

extern "C" {

pqi_status pqi_mpnn_grad_clip(float* g, size_t count, float max_norm, float* norm_out, void* stream) {
  PQI_CHECK_ARG(g && count > 0 && max_norm >= 0.0f);
  grad_clip_kernel<<<1, 1024, 0, as_stream(stream)>>>(g, count, max_norm, norm_out);
  PQI_LAUNCHED("grad_clip_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_sum(const float* x, size_t count, double* out, void* stream) {
  PQI_CHECK_ARG(x && out && count > 0);
  sum_kernel<<<1, 1024, 0, as_stream(stream)>>>(x, count, out);
  PQI_LAUNCHED("sum_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_kick_cdf(const float* logits, int n, int tasks, float temperature, float mix,
                             double* cdf, void* stream) {
  PQI_CHECK_ARG(logits && cdf && n > 0 && tasks > 0 && temperature > 0.0f && mix >= 0.0f && mix <= 1.0f);
  kick_cdf_kernel<<<tasks, 1024, 0, as_stream(stream)>>>(logits, n, (double)temperature, mix, cdf);
  PQI_LAUNCHED("kick_cdf_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_gemm(int transA, int transB, int M, int N, int K, float alpha, const void* A,
                         int lda, const void* B, int ldb, float beta, float* C32, void* C16,
                         int ldc, const float* bias, int relu, void* stream) {
  PQI_CHECK_ARG(A && B && (C32 || C16) && M > 0 && N > 0 && K > 0);
  PQI_CHECK_ARG(beta == 0.0f || C32);
  dim3 grid((N + mp::TN - 1) / mp::TN, (M + mp::TM - 1) / mp::TM);
  mp::gemm_bf16_kernel<<<grid, 256, 0, as_stream(stream)>>>(
      transA, transB, M, N, K, alpha, static_cast<const __nv_bfloat16*>(A), lda,
      static_cast<const __nv_bfloat16*>(B), ldb, beta, C32, static_cast<__nv_bfloat16*>(C16), ldc,
      bias, relu);
  PQI_LAUNCHED("gemm_bf16_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_norm_adj(const float* W, int n, void* Ahat, int ld, float* s, void* stream) {
  PQI_CHECK_ARG(W && Ahat && s && n > 0 && ld >= n);
  cudaStream_t st = as_stream(stream);
  mp::abs_rowsum_kernel<<<std::max(1, std::min((n + 7) / 8, 148 * 8)), 256, 0, st>>>(W, n, s);
  PQI_LAUNCHED("abs_rowsum_kernel");
  mp::norm_adj_kernel<<<mp::grid1((size_t)n * ld), 256, 0, st>>>(
      W, n, s, static_cast<__nv_bfloat16*>(Ahat), ld);
  PQI_LAUNCHED("norm_adj_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_features(const uint32_t* theta, const double* gains64, const float* s,
                             float mean_s, int n, void* F, void* stream) {
  PQI_CHECK_ARG(theta && gains64 && s && F && n > 0);
  mp::features_kernel<<<mp::grid1(n), 256, 0, as_stream(stream)>>>(
      theta, gains64, s, mean_s, n, static_cast<__nv_bfloat16*>(F));
  PQI_LAUNCHED("features_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_softmax_xent(const float* logits, const float* target, int n, float* loss,
                                 float* dlogits, float* prob, void* stream) {
  PQI_CHECK_ARG(logits && n > 0);
  mp::softmax_xent_kernel<<<1, 1024, 0, as_stream(stream)>>>(logits, target, n, loss, dlogits,
                                                             prob);
  PQI_LAUNCHED("softmax_xent_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_relu_bwd(const float* dY, const float* Y, size_t count, float* dZ, void* dZ16,
                             void* stream) {
  PQI_CHECK_ARG(dY && Y && dZ && count > 0);
  mp::relu_bwd_kernel<<<mp::grid1(count), 256, 0, as_stream(stream)>>>(
      dY, Y, count, dZ, static_cast<__nv_bfloat16*>(dZ16));
  PQI_LAUNCHED("relu_bwd_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_colsum(const float* X, int rows, int cols, int ld, float* out,
                           int accumulate, void* stream) {
  PQI_CHECK_ARG(X && out && rows > 0 && cols > 0);
  mp::colsum_kernel<<<std::max(1, std::min((cols + 7) / 8, 148)), 256, 0, as_stream(stream)>>>(
      X, rows, cols, ld, out, accumulate);
  PQI_LAUNCHED("colsum_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_to_bf16(const float* x, size_t count, void* y, void* stream) {
  PQI_CHECK_ARG(x && y && count > 0);
  mp::to_bf16_kernel<<<mp::grid1(count), 256, 0, as_stream(stream)>>>(
      x, count, static_cast<__nv_bfloat16*>(y));
  PQI_LAUNCHED("to_bf16_kernel");
  return PQI_OK;
}

pqi_status pqi_mpnn_adam(float* w, const float* g, float* m, float* v, void* w16, size_t count,
                         float lr, float b1, float b2, float eps, int step, void* stream) {
  PQI_CHECK_ARG(w && g && m && v && count > 0 && step >= 1);
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  mp::adam_kernel<<<mp::grid1(count), 256, 0, as_stream(stream)>>>(
      w, g, m, v, static_cast<__nv_bfloat16*>(w16), count, lr, b1, b2, eps, c1, c2);
  PQI_LAUNCHED("adam_kernel");
  return PQI_OK;
}

}  // extern "C"
