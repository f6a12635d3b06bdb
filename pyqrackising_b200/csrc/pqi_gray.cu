// libpqi: parallel Gray-code search (replaces the reference's `gray` kernel,
// pyqrackising/kernels.cl:894-978) and the device-resident single-flip
// descent (the repeated single-flip passes of spin_glass_solver.py:605-627).
//
// Both keep each state's gain vector on chip and update it in O(n) per
// accepted flip (g_v -= 2 x_v x_k W_kv, g_k = -g_k) instead of recomputing an
// O(n) row sum for every candidate flip as the reference does.
#include <algorithm>

#include "pqi_common.cuh"

namespace pqi {

// Gain storage: exact int32 for int8 weights, float64 otherwise.
template <typename WT>
struct GainOf {
  typedef double type;
};
template <>
struct GainOf<int8_t> {
  typedef int type;
};

template <typename W64>
__device__ __forceinline__ int bit_of(const W64* bits, int v);

template <>
__device__ __forceinline__ int bit_of<uint64_t>(const uint64_t* bits, int v) {
  return (int)((bits[v >> 6] >> (v & 63)) & 1ull);
}
template <>
__device__ __forceinline__ int bit_of<uint32_t>(const uint32_t* bits, int v) {
  return (int)((bits[v >> 5] >> (v & 31)) & 1u);
}

// Flip node k of the block's state: every thread updates its slice of the
// gains, then one thread toggles the bit. Must be reached by all threads of
// the block with the same k. Caller guarantees a barrier after its own reads
// of g[k] / bits.
template <typename GT, typename WT, typename W64, int CH = 16>
__device__ __forceinline__ void block_flip(GT* g, W64* bits, const WT* __restrict__ Wp, int ld,
                                           int n, int k) {
  const int xk = bit_of<W64>(bits, k);
  const WT* __restrict__ row = Wp + (size_t)k * ld;
  __syncthreads();
  // row read in chunks of CH per thread, loads issued before the gains change
  for (int base = threadIdx.x; base < n; base += CH * blockDim.x) {
    WT w[CH];
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int v = base + i * blockDim.x;
      w[i] = v < n ? __ldg(row + v) : (WT)0;
    }
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int v = base + i * blockDim.x;
      if (v < n) {
        if (v == k) {
          g[v] = -g[v];
        } else {
          const GT w2 = (GT)2 * (GT)w[i];
          g[v] += (bit_of<W64>(bits, v) == xk) ? -w2 : w2;
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    constexpr int kShift = sizeof(W64) == 8 ? 6 : 5;
    constexpr int kMask = sizeof(W64) == 8 ? 63 : 31;
    bits[k >> kShift] ^= (W64)1 << (k & kMask);
  }
  __syncthreads();
}

template <typename GT>
__device__ __forceinline__ GT from_f64(double v);
template <>
__device__ __forceinline__ double from_f64<double>(double v) {
  return v;
}
template <>
__device__ __forceinline__ int from_f64<int>(double v) {
  return (int)llrint(v);
}

// One CTA per seed (grid-stride). Dynamic smem: 64-bit state words, then the
// gains (unless g_global is given: then CTA b uses g_global + b*n).
template <typename WT>
__global__ void __launch_bounds__(256) gray_kernel(
    const WT* __restrict__ Wp, int ld, int n, const uint64_t* __restrict__ theta64,
    const double* __restrict__ base_g, int spin, long long iters_bound, int S,
    uint64_t* __restrict__ theta_out, float* __restrict__ energy_out,
    typename GainOf<WT>::type* g_global) {
  typedef typename GainOf<WT>::type GT;
  extern __shared__ __align__(16) unsigned char smem[];
  const int blocks = (n + 63) >> 6;
  uint64_t* bits = reinterpret_cast<uint64_t*>(smem);
  GT* g = g_global ? g_global + (size_t)blockIdx.x * n
                   : reinterpret_cast<GT*>(smem + (((size_t)blocks * 8 + 15) & ~size_t(15)));
  const int lane = threadIdx.x & 31;

  for (int s = blockIdx.x; s < S; s += gridDim.x) {
    for (int q = threadIdx.x; q < blocks; q += blockDim.x) bits[q] = theta64[q];
    for (int v = threadIdx.x; v < n; v += blockDim.x) g[v] = from_f64<GT>(base_g[v]);
    __syncthreads();

    // Seed mask of work-item s (kernels.cl:915-926): seed bit 63-b flips node
    // n-1-b through a 32-bit int shift, so the mask is 1 << (offset & 31),
    // sign-extended to 64 bits when the count is 31. Every thread computes it.
    const uint64_t seed = (uint64_t)s ^ ((uint64_t)s >> 1);
    const int w0 = (n > 64 ? n - 64 : 0) >> 6;
    uint64_t m[2] = {0ull, 0ull};
    const int max_lcv = n < 64 ? n : 64;
    for (int b = 0; b < max_lcv; ++b) {
      if (!((seed >> (63 - b)) & 1ull)) continue;
      const int off = n - (b + 1);
      const int32_t m32 = (int32_t)(1u << ((unsigned)off & 31u));
      m[(off >> 6) - w0] ^= (uint64_t)(int64_t)m32;
    }
    // Apply the mask one node at a time; the sum of the successive gains is
    // the prologue's cut change (kernels.cl:928-941).
    double E = 0.0;
    for (int q = 0; q < 2; ++q) {
      uint64_t mq = m[q];
      while (mq) {
        const int p = __ffsll((long long)mq) - 1;
        mq &= mq - 1;
        const int node = ((w0 + q) << 6) + p;
        if (node < n) {
          E += (double)g[node];
          block_flip<GT, WT, uint64_t>(g, bits, Wp, ld, n, node);
        } else if (node < (blocks << 6)) {
          // padding bit of the last word: no energy, kept for the output words
          __syncthreads();
          if (threadIdx.x == 0) bits[node >> 6] ^= 1ull << (node & 63);
          __syncthreads();
        }
      }
    }

    // Gray walk: positions p = m*blocks + b for i = s + m*S < iters_bound; the
    // candidate node is ctz(i+1) + 64b; a flip is kept iff its gain is > 0. All
    // warps scan the same 32 positions (identical ballots, no barrier) and the
    // block applies the first accepted flip together.
    const long long Pm = iters_bound > s ? (iters_bound - 1 - s) / S + 1 : 0;
    const long long P = Pm * blocks;
    long long p0 = 0;
    while (p0 < P) {
      const long long p = p0 + lane;
      int k = -1;
      bool pos = false;
      if (p < P) {
        const long long mm = p / blocks;
        const int b = (int)(p - mm * blocks);
        const long long i = (long long)s + mm * S;
        k = (__ffsll(i + 1) - 1) + (b << 6);
        if (k < n) pos = g[k] > (GT)0;
      }
      const unsigned bal = __ballot_sync(0xFFFFFFFFu, pos);
      if (!bal) {
        p0 += 32;
        continue;
      }
      const int f = __ffs(bal) - 1;
      const int kk = __shfl_sync(0xFFFFFFFFu, k, f);
      E += (double)g[kk];
      block_flip<GT, WT, uint64_t>(g, bits, Wp, ld, n, kk);
      p0 += f + 1;
    }

    for (int q = threadIdx.x; q < blocks; q += blockDim.x)
      theta_out[(size_t)s * blocks + q] = bits[q];
    if (threadIdx.x == 0) energy_out[s] = (float)(spin ? E : E / 2.0);
    __syncthreads();
  }
}

// Single CTA: repeat (select best single flip under the reference geometry,
// flip it if its value is > 0) until none improves or max_flips is reached.
template <typename WT>
__global__ void __launch_bounds__(1024) descent_kernel(
    const WT* __restrict__ Wp, int ld, int n, uint32_t* __restrict__ theta,
    double* __restrict__ g64, int spin, SelGeom geo, int max_flips, int gains_in_smem,
    double* __restrict__ energy_sum, int* __restrict__ flips, int* __restrict__ trace,
    int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint64_t scratch[32];
  const int n32 = (n + 31) >> 5;
  uint32_t* bits = reinterpret_cast<uint32_t*>(smem);
  double* g = gains_in_smem
                  ? reinterpret_cast<double*>(smem + (((size_t)n32 * 4 + 15) & ~size_t(15)))
                  : g64;
  for (int q = threadIdx.x; q < n32; q += blockDim.x) bits[q] = theta[q];
  if (gains_in_smem)
    for (int v = threadIdx.x; v < n; v += blockDim.x) g[v] = g64[v];
  __syncthreads();
  double esum = 0.0;
  int cnt = 0, st = PQI_OK;
  while (true) {
    // a value below the thread's best so far cannot give a larger key: the
    // key (and its divisions) only for candidates that reach it
    uint64_t best = 0;
    float bv = -INFINITY;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      float v = (float)g[k];
      if (spin) v *= 2.0f;
      if (v >= bv) {
        const uint64_t kk = sel_key(v, (uint64_t)k, geo);
        if (kk > best) {
          best = kk;
          bv = v;
        }
      }
    }
    best = block_max_u64(best, scratch);
    float val;
    int64_t idx;
    sel_decode(best, geo, &val, &idx);
    if (!(val > 0.0f)) break;
    if (cnt >= max_flips) {
      st = PQI_ETIMEOUT;
      break;
    }
    esum += (double)val;
    if (threadIdx.x == 0 && trace) trace[cnt] = (int)idx;
    ++cnt;
    block_flip<double, WT, uint32_t, 8>(g, bits, Wp, ld, n, (int)idx);
  }
  for (int q = threadIdx.x; q < n32; q += blockDim.x) theta[q] = bits[q];
  if (gains_in_smem)
    for (int v = threadIdx.x; v < n; v += blockDim.x) g64[v] = g[v];
  if (threadIdx.x == 0) {
    *energy_sum = esum;
    *flips = cnt;
    if (status) *status = st;
  }
}

static size_t gray_smem_bytes(int n, size_t gain_bytes) {
  const int blocks = (n + 63) >> 6;
  return (((size_t)blocks * 8 + 15) & ~size_t(15)) + (size_t)n * gain_bytes;
}

static constexpr size_t kMaxDynSmem = 200 * 1024;

}  // namespace pqi

using namespace pqi;

extern "C" {

pqi_status pqi_gray(const pqi_weights* w, const uint64_t* theta64, const double* gains64,
                    int is_spin_glass, int iters_bound, int seeds, uint64_t* theta_out,
                    float* energy_out, void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(w && theta64 && theta_out && energy_out && seeds > 0 && iters_bound >= 0);
  const int n = w->n;
  cudaStream_t s = as_stream(stream);
  Workspace ws(workspace, workspace_bytes);
  if (!gains64) {
    // gains of theta: unpack the 64-bit words as 32-bit words (same bit order)
    double* g = ws.take<double>(n);
    PQI_CHECK_ARG(g);
    pqi_status rc = launch_gains(w, reinterpret_cast<const uint32_t*>(theta64), 1, nullptr, g, s);
    if (rc) return rc;
    gains64 = g;
  }
  const bool i8 = w->kind == PQI_W_I8;
  const size_t gbytes = i8 ? sizeof(int) : sizeof(double);
  size_t smem = gray_smem_bytes(n, gbytes);
  int grid = seeds;
  void* gglob = nullptr;
  if (smem > kMaxDynSmem) {
    // gains in global memory, one n-vector per CTA
    const int blocks = (n + 63) >> 6;
    smem = (size_t)blocks * 8;
    PQI_CHECK_ARG(smem <= kMaxDynSmem);
    const size_t avail = (ws.size > ws.used + 256) ? (ws.size - ws.used - 256) : 0;
    const long long ctas = (long long)(avail / ((size_t)n * gbytes));
    PQI_CHECK_ARG(ctas >= 1);
    grid = (int)std::min<long long>(std::min<long long>(ctas, seeds), 148 * 4);
    gglob = ws.take<char>((size_t)grid * n * gbytes);
    PQI_CHECK_ARG(gglob);
  }
  if (i8) {
    PQI_TRY(cudaFuncSetAttribute(gray_kernel<int8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    gray_kernel<int8_t><<<grid, 256, smem, s>>>(w->W_i8, w->ld, n, theta64, gains64,
                                                is_spin_glass, iters_bound, seeds, theta_out,
                                                energy_out, static_cast<int*>(gglob));
  } else {
    PQI_TRY(cudaFuncSetAttribute(gray_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    gray_kernel<float><<<grid, 256, smem, s>>>(w->W_f32z, w->ld, n, theta64, gains64,
                                               is_spin_glass, iters_bound, seeds, theta_out,
                                               energy_out, static_cast<double*>(gglob));
  }
  PQI_LAUNCHED("gray_kernel");
  return PQI_OK;
}

pqi_status pqi_single_descent(const pqi_weights* w, uint32_t* theta, double* gains64,
                              int is_spin_glass, int global_size, int local_size, int max_flips,
                              double* energy_sum, int* flips, int* trace, void* workspace,
                              size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(w && theta && gains64 && energy_sum && flips && max_flips >= 0);
  const int n = w->n;
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(n, global_size, local_size, &geo));
  Workspace ws(workspace, workspace_bytes);
  int* status = ws.take<int>(1);
  PQI_CHECK_ARG(status);
  cudaStream_t s = as_stream(stream);
  const size_t bits_bytes = (((size_t)((n + 31) >> 5) * 4 + 15) & ~size_t(15));
  size_t smem = bits_bytes + (size_t)n * 8;
  int in_smem = 1;
  if (smem > kMaxDynSmem) {
    smem = bits_bytes;
    in_smem = 0;
  }
  PQI_CHECK_ARG(smem <= kMaxDynSmem);
  if (w->kind == PQI_W_I8) {
    PQI_TRY(cudaFuncSetAttribute(descent_kernel<int8_t>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    descent_kernel<int8_t><<<1, 1024, smem, s>>>(w->W_i8, w->ld, n, theta, gains64,
                                                 is_spin_glass, geo, max_flips, in_smem,
                                                 energy_sum, flips, trace, status);
  } else {
    PQI_TRY(cudaFuncSetAttribute(descent_kernel<float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    descent_kernel<float><<<1, 1024, smem, s>>>(w->W_f32z, w->ld, n, theta, gains64,
                                                is_spin_glass, geo, max_flips, in_smem, energy_sum,
                                                flips, trace, status);
  }
  PQI_LAUNCHED("descent_kernel");
  int hst = 0;
  PQI_TRY(cudaMemcpyAsync(&hst, status, sizeof(int), cudaMemcpyDeviceToHost, s));
  PQI_TRY(cudaStreamSynchronize(s));
  return (pqi_status)hst;
}

}  // extern "C"
