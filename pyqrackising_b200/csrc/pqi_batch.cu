// libpqi: batched local search over many graphs and many seeds per graph in one
// persistent launch (the batched form of the search; no reference
// counterpart beyond the single-graph loop of spin_glass_solver.py:603-717).
//
// One CTA runs one task (graph g, starting state s) at a time, grid-stride over
// tasks, with the task's state and gain vector in shared memory:
//   1. gains of the starting state, O(n^2) over the graph's rows (W rows of
//      small graphs stay in L2 across the graph's tasks);
//   2. `rounds` times: steepest single-flip ascent to a local optimum (largest
//      gain, lowest node on ties, accept while > 0), record the best state,
//      then a kick: `kick` forced flips, each node drawn uniformly at random
//      or, when a per-graph proposal distribution is given (the learned
//      proposal network's softmax, as a normalised cumulative array), drawn
//      from it by bisection (with replacement);
//   3. a last ascent; the best value and state of the task are written out.
// Values are tracked incrementally: flipping node k changes the cut by its gain
// g_k and the spin energy by 2 g_k. Local fields (and so gains) are exact int32
// for int8 weights and float64 otherwise. Every loop is bounded (flip budget
// per ascent).
#include <algorithm>
#include <type_traits>

#include "pqi_common.cuh"

namespace pqi {

struct BatchGraph {
  const void* W;  // prepared copy: int8 (kind PQI_W_I8) or float32 zero-diagonal (PQI_W_F32)
  int n;
  int ld;
  int kind;
  int pad;
  double upper_sum;
};

__device__ __forceinline__ uint64_t bmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;  // SplitMix64 finaliser
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double bunif(uint64_t seed, uint64_t a, uint64_t b) {
  const uint64_t h = bmix64(seed ^ bmix64(a * 0x632BE59BD9B4E019ull + b));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

template <typename WT, typename GT>
struct TaskCtx {
  const WT* W;
  int n, ld;
  GT* g;  // local fields y = W x
  uint32_t* bits;
};

// The task keeps the local field y = W x (x = 2s - 1) instead of the gains:
// the gain of node v is g_v = x_v y_v, and flipping node k changes every
// field by y_v -= 2 x_k W_kv (W's prepared copy has a zero diagonal, so y_k is
// unchanged). One fused pass per flip: each thread loads its whole slice of
// row k first (all loads in flight at once), applies the update, and folds
// the new gains into a (float gain, lowest node) block argmax. Thread 0
// toggles bit k between the reduction's two barriers, when every thread has
// finished reading the bits and before anyone reads them again. Two barriers
// per flip. k < 0: no flip, only the argmax.
template <typename WT, typename GT, int CH>
__device__ __forceinline__ void flip_and_select(const TaskCtx<WT, GT>& c, int k, float* red_v,
                                                int* red_i, float* out_v, int* out_i) {
  float bv = -INFINITY;
  int bi = 0x7FFFFFFF;
  const int n = c.n;
  const GT coef = (k >= 0) ? (((c.bits[k >> 5] >> (k & 31)) & 1) ? (GT)-2 : (GT)2) : (GT)0;
  const WT* __restrict__ row = c.W + (size_t)(k >= 0 ? k : 0) * c.ld;
  for (int base = threadIdx.x; base < n; base += CH * blockDim.x) {
    WT w[CH];
    if (k >= 0) {
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        const int v = base + i * blockDim.x;
        w[i] = v < n ? __ldg(row + v) : (WT)0;
      }
    }
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int v = base + i * blockDim.x;
      if (v < n) {
        GT y = c.g[v];
        if (k >= 0) {
          y += coef * (GT)w[i];
          c.g[v] = y;
        }
        // node k's bit is toggled only after this pass: use its new value here
        const bool xv = (((c.bits[v >> 5] >> (v & 31)) & 1) != 0) != (v == k);
        const float gv = (float)(xv ? y : -y);
        if (gv > bv) {  // v ascends within a thread: strict '>' keeps the lowest node
          bv = gv;
          bi = v;
        }
      }
    }
  }
  // warp then block argmax: larger gain, then lower node
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
    const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  if (lane == 0) {
    red_v[warp] = bv;
    red_i[warp] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0 && k >= 0) c.bits[k >> 5] ^= 1u << (k & 31);
  bv = lane < nwarps ? red_v[lane] : -INFINITY;
  bi = lane < nwarps ? red_i[lane] : 0x7FFFFFFF;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
    const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
    }
  }
  __syncthreads();
  *out_v = bv;
  *out_i = bi;
}

template <typename WT, int CH>
__global__ void __launch_bounds__(256, 3) batch_search_kernel(
    const BatchGraph* __restrict__ graphs, const int* __restrict__ task_graph,
    const uint32_t* __restrict__ init_states, int words_pitch, int tasks, int spin, int rounds,
    int kick, int flip_budget, uint64_t seed, const double* __restrict__ kick_cdf,
    const long long* __restrict__ cdf_offset, uint32_t* __restrict__ best_states,
    double* __restrict__ best_values, unsigned long long* __restrict__ flips_total,
    int* __restrict__ status) {
  typedef typename std::conditional<sizeof(WT) == 1, int, double>::type GT;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[32];
  __shared__ float red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_pick;
  for (int task = blockIdx.x; task < tasks; task += gridDim.x) {
    const BatchGraph G = graphs[task_graph[task]];
    const int n = G.n, n32 = (n + 31) >> 5;
    TaskCtx<WT, GT> c;
    c.W = static_cast<const WT*>(G.W);
    c.n = n;
    c.ld = G.ld;
    c.bits = reinterpret_cast<uint32_t*>(smem);
    c.g = reinterpret_cast<GT*>(smem + (((size_t)n32 * 4 + 15) & ~size_t(15)));
    uint32_t* best_bits = best_states + (size_t)task * words_pitch;
    for (int w = threadIdx.x; w < n32; w += blockDim.x) c.bits[w] = init_states[(size_t)task * words_pitch + w];
    __syncthreads();
    // 1. gains of the starting state, one warp per row
    {
      const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
      for (int k = threadIdx.x >> 5; k < n; k += warps) {
        const WT* row = c.W + (size_t)k * c.ld;
        GT acc = 0;
        for (int v = lane; v < n; v += 32) {
          const GT w = (GT)row[v];
          acc += ((c.bits[v >> 5] >> (v & 31)) & 1) ? w : -w;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
        if (lane == 0) c.g[k] = acc;  // local field y_k
      }
    }
    __syncthreads();
    // q = x^T W x = sum_k x_k y_k; value from q
    double part = 0.0;
    for (int v = threadIdx.x; v < n; v += blockDim.x)
      part += ((c.bits[v >> 5] >> (v & 31)) & 1) ? (double)c.g[v] : -(double)c.g[v];
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    double q = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) q += red[i];
    __syncthreads();
    const double scale = spin ? 2.0 : 1.0;
    double val = spin ? -q / 2.0 : (2.0 * G.upper_sum - q) / 4.0;
    double best = -INFINITY;
    unsigned long long nflips = 0;
    int timeout = 0;
    float gv;
    int k;
    flip_and_select<WT, GT, CH>(c, -1, red_v, red_i, &gv, &k);
    for (int r = 0; r <= rounds; ++r) {
      // steepest ascent: flip the best node while its gain is positive
      for (int f = 0;; ++f) {
        if (!(gv > 0.0f)) break;
        if (f >= flip_budget) {
          timeout = 1;
          break;
        }
        // exact gain before the flip: x_k y_k (bits and fields are stable here)
        const double gk = ((c.bits[k >> 5] >> (k & 31)) & 1) ? (double)c.g[k] : -(double)c.g[k];
        __syncthreads();
        val += scale * gk;
        flip_and_select<WT, GT, CH>(c, k, red_v, red_i, &gv, &k);
        ++nflips;
      }
      if (val > best) {
        best = val;
        for (int w = threadIdx.x; w < n32; w += blockDim.x) best_bits[w] = c.bits[w];
      }
      if (r == rounds) break;
      // kick: forced flips
      for (int j = 0; j < kick; ++j) {
        if (threadIdx.x == 0) {
          int pick;
          const double u = bunif(seed, (uint64_t)task * 1315423911ull + r, (uint64_t)j);
          if (kick_cdf) {
            // first node whose cumulative proposal mass exceeds u
            const double* cdf = kick_cdf + cdf_offset[task_graph[task]];
            int lo = 0, hi = n - 1;
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (cdf[mid] > u) {
                hi = mid;
              } else {
                lo = mid + 1;
              }
            }
            pick = lo;
          } else {
            pick = (int)(u * n);
            if (pick >= n) pick = n - 1;
          }
          s_pick = pick;
        }
        __syncthreads();
        const int kk = s_pick;
        const double gk = ((c.bits[kk >> 5] >> (kk & 31)) & 1) ? (double)c.g[kk] : -(double)c.g[kk];
        __syncthreads();
        val += scale * gk;
        flip_and_select<WT, GT, CH>(c, kk, red_v, red_i, &gv, &k);
        ++nflips;
      }
    }
    if (threadIdx.x == 0) {
      best_values[task] = best;
      atomicAdd(flips_total, nflips);
      if (timeout) atomicExch(status, PQI_ETIMEOUT);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Warp-per-task form for small graphs (n <= 128 * NG): the same search, the
// same selection rule and the same kick stream as batch_search_kernel, with
// one warp per task and no shared memory. Lane l owns the nodes
// v = 128 i + 4 l + j (i < NG, j < 4), keeps their local fields and bits in
// registers, and reads its four weights of row k with one vector load per i
// (a warp reads 512 B of a float row, 128 B of an int8 row, per i). A flip is
// NG loads, 4 NG updates and a two-step 32-bit redux argmax: no barrier.

__device__ __forceinline__ unsigned long long wkey(float gv, int v, int xv) {
  return ((unsigned long long)ord_f32(gv) << 32) |
         (unsigned long long)(((0x3FFFFFFFu - (uint32_t)v) << 1) | (uint32_t)xv);
}

__device__ __forceinline__ unsigned long long wmax_key(unsigned long long key) {
  const uint32_t hi = __reduce_max_sync(0xFFFFFFFFu, (uint32_t)(key >> 32));
  const uint32_t lo =
      __reduce_max_sync(0xFFFFFFFFu, ((uint32_t)(key >> 32) == hi) ? (uint32_t)key : 0u);
  return ((unsigned long long)hi << 32) | lo;
}

// One pass of the warp form: apply flip k (coef = -2 x_k; k < 0: none) to the
// lane's fields and bits, then the warp's best key (float gain, lowest node)
// and the exact gain of that node.
template <typename WT, typename GT, int NG>
__device__ __forceinline__ void warp_pass(const WT* __restrict__ W, int ld, int n, int lane, int k,
                                          GT coef, GT (&y)[4 * NG], uint32_t& xm,
                                          unsigned long long* gkey, double* gk) {
  if (k >= 0) {
    const WT* __restrict__ row = W + (size_t)k * ld;
    WT w[4 * NG];
#pragma unroll
    for (int i = 0; i < NG; ++i) {
      const int u0 = 128 * i + 4 * lane;
      if (u0 < n) {
        if constexpr (sizeof(WT) == 4) {
          const float4 t = __ldg(reinterpret_cast<const float4*>(row + u0));
          w[4 * i] = t.x; w[4 * i + 1] = t.y; w[4 * i + 2] = t.z; w[4 * i + 3] = t.w;
        } else {
          const char4 t = __ldg(reinterpret_cast<const char4*>(row + u0));
          w[4 * i] = t.x; w[4 * i + 1] = t.y; w[4 * i + 2] = t.z; w[4 * i + 3] = t.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) w[4 * i + j] = (WT)0;
      }
    }
#pragma unroll
    for (int e = 0; e < 4 * NG; ++e) y[e] += coef * (GT)w[e];
    if (lane == ((k & 127) >> 2)) xm ^= 1u << (4 * (k >> 7) + (k & 3));
  }
  // nodes ascend with the slot within a lane: strict '>' keeps the lowest
  float bv = -INFINITY;
  int bs = -1;
#pragma unroll
  for (int e = 0; e < 4 * NG; ++e) {
    const int v = 128 * (e >> 2) + 4 * lane + (e & 3);
    const float gv = (float)(((xm >> e) & 1u) ? y[e] : -y[e]);
    if (v < n && gv > bv) {
      bv = gv;
      bs = e;
    }
  }
  double bg = 0.0;
  int bx = 0;
#pragma unroll
  for (int e = 0; e < 4 * NG; ++e)
    if (e == bs) {
      bx = (xm >> e) & 1;
      bg = bx ? (double)y[e] : -(double)y[e];
    }
  const unsigned long long key =
      bs >= 0 ? wkey(bv, 128 * (bs >> 2) + 4 * lane + (bs & 3), bx) : 0ull;
  const unsigned long long wk = wmax_key(key);
  const uint32_t src = __ballot_sync(0xFFFFFFFFu, key == wk && wk != 0ull);
  *gk = __shfl_sync(0xFFFFFFFFu, bg, src ? __ffs(src) - 1 : 0);
  *gkey = wk;
}

template <typename WT, int NG>
__global__ void __launch_bounds__(128) warp_search_kernel(
    const BatchGraph* __restrict__ graphs, const int* __restrict__ task_graph,
    const uint32_t* __restrict__ init_states, int words_pitch, int tasks, int spin, int rounds,
    int kick, int flip_budget, uint64_t seed, const double* __restrict__ kick_cdf,
    const long long* __restrict__ cdf_offset, uint32_t* __restrict__ best_states,
    double* __restrict__ best_values, unsigned long long* __restrict__ flips_total,
    int* __restrict__ status) {
  typedef typename std::conditional<sizeof(WT) == 1, int, double>::type GT;
  const int lane = threadIdx.x & 31;
  const int warps_total = (gridDim.x * blockDim.x) >> 5;
  unsigned long long nflips_all = 0;
  for (int task = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; task < tasks; task += warps_total) {
    const BatchGraph G = graphs[task_graph[task]];
    const int n = G.n;
    const WT* __restrict__ W = static_cast<const WT*>(G.W);
    const uint32_t* __restrict__ init = init_states + (size_t)task * words_pitch;
    uint32_t* __restrict__ best_bits = best_states + (size_t)task * words_pitch;
    // my bits: nibble i holds nodes 128 i + 4 lane + (0..3)
    uint32_t xm = 0;
#pragma unroll
    for (int i = 0; i < NG; ++i) {
      const int v0 = 128 * i + 4 * lane;
      if (v0 < n) {
        const uint32_t word = __ldg(init + (v0 >> 5));
        uint32_t nib = (word >> (v0 & 31)) & 15u;
        if (v0 + 4 > n) nib &= (1u << (n - v0)) - 1u;
        xm |= nib << (4 * i);
      }
    }
    // starting local fields y_v = sum_u x_u W_uv (W symmetric): every row u
    // adds +-W_u to the lane's own columns, x_u read from the state word held
    // by lane u / 32. Rows are independent: loads stream, nothing is reduced.
    const uint32_t word_l = (32 * lane < n) ? __ldg(init + lane) : 0u;
    GT y[4 * NG];
#pragma unroll
    for (int e = 0; e < 4 * NG; ++e) y[e] = 0;
#pragma unroll 2
    for (int u = 0; u < n; ++u) {
      const WT* __restrict__ row = W + (size_t)u * G.ld;
      const bool xu = (__shfl_sync(0xFFFFFFFFu, word_l, u >> 5) >> (u & 31)) & 1u;
#pragma unroll
      for (int i = 0; i < NG; ++i) {
        const int u0 = 128 * i + 4 * lane;
        if (u0 < n) {
          WT w4[4];
          if constexpr (sizeof(WT) == 4) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(row + u0));
            w4[0] = t.x; w4[1] = t.y; w4[2] = t.z; w4[3] = t.w;
          } else {
            const char4 t = __ldg(reinterpret_cast<const char4*>(row + u0));
            w4[0] = t.x; w4[1] = t.y; w4[2] = t.z; w4[3] = t.w;
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) y[4 * i + j] += xu ? (GT)w4[j] : -(GT)w4[j];
        }
      }
    }
    // value of the starting state from q = sum_v x_v y_v
    double qp = 0.0;
#pragma unroll
    for (int e = 0; e < 4 * NG; ++e) qp += ((xm >> e) & 1u) ? (double)y[e] : -(double)y[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qp += __shfl_xor_sync(0xFFFFFFFFu, qp, o);
    const double scale = spin ? 2.0 : 1.0;
    double val = spin ? -qp / 2.0 : (2.0 * G.upper_sum - qp) / 4.0;
    double best = -INFINITY;
    unsigned long long nflips = 0;
    int timeout = 0;
    unsigned long long gkey;
    double gk;
    warp_pass<WT, GT, NG>(W, G.ld, n, lane, -1, (GT)0, y, xm, &gkey, &gk);
    for (int r = 0; r <= rounds; ++r) {
      for (int f = 0;; ++f) {
        if (gkey == 0ull || !(unord_f32((uint32_t)(gkey >> 32)) > 0.0f)) break;
        if (f >= flip_budget) {
          timeout = 1;
          break;
        }
        const int k = (int)(0x3FFFFFFFu - (((uint32_t)gkey) >> 1));
        const GT coef = (gkey & 1ull) ? (GT)-2 : (GT)2;
        val += scale * gk;
        warp_pass<WT, GT, NG>(W, G.ld, n, lane, k, coef, y, xm, &gkey, &gk);
        ++nflips;
      }
      if (val > best) {
        best = val;
#pragma unroll
        for (int i = 0; i < NG; ++i) {
          const int v0 = 128 * i + 4 * lane;
          uint32_t wd = ((xm >> (4 * i)) & 15u) << (4 * (lane & 7));
          wd |= __shfl_xor_sync(0xFFFFFFFFu, wd, 1);
          wd |= __shfl_xor_sync(0xFFFFFFFFu, wd, 2);
          wd |= __shfl_xor_sync(0xFFFFFFFFu, wd, 4);
          if ((lane & 7) == 0 && v0 < n) best_bits[v0 >> 5] = wd;
        }
      }
      if (r == rounds) break;
      for (int j = 0; j < kick; ++j) {
        // every lane draws the same node (same hash, same cumulative array)
        int pick;
        const double u = bunif(seed, (uint64_t)task * 1315423911ull + r, (uint64_t)j);
        if (kick_cdf) {
          const double* cdf = kick_cdf + cdf_offset[task_graph[task]];
          int lo = 0, hi = n - 1;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cdf[mid] > u) {
              hi = mid;
            } else {
              lo = mid + 1;
            }
          }
          pick = lo;
        } else {
          pick = (int)(u * n);
          if (pick >= n) pick = n - 1;
        }
        // the owner reads the node's bit and exact gain
        const int owner = (pick & 127) >> 2, slot = 4 * (pick >> 7) + (pick & 3);
        double g = 0.0;
        int xv = 0;
#pragma unroll
        for (int e = 0; e < 4 * NG; ++e)
          if (e == slot) {
            xv = (xm >> e) & 1;
            g = xv ? (double)y[e] : -(double)y[e];
          }
        g = __shfl_sync(0xFFFFFFFFu, g, owner);
        xv = __shfl_sync(0xFFFFFFFFu, xv, owner);
        val += scale * g;
        warp_pass<WT, GT, NG>(W, G.ld, n, lane, pick, xv ? (GT)-2 : (GT)2, y, xm, &gkey, &gk);
        ++nflips;
      }
    }
    if (lane == 0) {
      best_values[task] = best;
      nflips_all += nflips;
      if (timeout) atomicExch(status, PQI_ETIMEOUT);
    }
  }
  if (lane == 0 && nflips_all) atomicAdd(flips_total, nflips_all);
}

}  // namespace pqi

using namespace pqi;

extern "C" {

size_t pqi_batch_graph_desc_bytes(void) { return sizeof(BatchGraph); }

pqi_status pqi_batch_search(const void* graphs, int num_graphs, const int* task_graph,
                            const uint32_t* init_states, int words_pitch, int tasks, int max_n,
                            int kind, int is_spin_glass, int rounds, int kick, int flip_budget,
                            uint64_t seed, const double* kick_cdf, const long long* cdf_offset,
                            uint32_t* best_states, double* best_values,
                            unsigned long long* flips_total, int* status, void* stream) {
  PQI_CHECK_ARG(graphs && num_graphs > 0 && task_graph && init_states && tasks > 0 && max_n > 0);
  PQI_CHECK_ARG(best_states && best_values && flips_total && status && rounds >= 0 && kick >= 0);
  PQI_CHECK_ARG(words_pitch >= (max_n + 31) / 32 && flip_budget > 0);
  PQI_CHECK_ARG(!kick_cdf || cdf_offset);
  cudaStream_t s = as_stream(stream);
  const bool i8 = kind == PQI_W_I8;
  const size_t smem = (((size_t)((max_n + 31) >> 5) * 4 + 15) & ~size_t(15)) +
                      (size_t)max_n * (i8 ? sizeof(int) : sizeof(double));
  PQI_CHECK_ARG(smem <= 200 * 1024);
  static int num_sms = 0;
  if (!num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int per_sm = std::max(1, std::min(8, (int)((220 * 1024) / (smem + 2048))));
  const int grid = std::max(1, std::min(tasks, num_sms * per_sm));
  const BatchGraph* gd = static_cast<const BatchGraph*>(graphs);
  // row loads per thread in chunks of CH (8 for n <= 2048, else 16; three CTAs
  // per SM cap the registers)
#define PQI_BATCH_LAUNCH(WT_, CH_)                                                              \
  do {                                                                                         \
    PQI_TRY(cudaFuncSetAttribute(batch_search_kernel<WT_, CH_>,                               \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));     \
    PQI_TRY(cudaFuncSetAttribute(batch_search_kernel<WT_, CH_>,                               \
                                 cudaFuncAttributePreferredSharedMemoryCarveout, 100));        \
    batch_search_kernel<WT_, CH_><<<grid, 256, smem, s>>>(                                     \
        gd, task_graph, init_states, words_pitch, tasks, is_spin_glass, rounds, kick,          \
        flip_budget, seed, kick_cdf, cdf_offset, best_states, best_values, flips_total,        \
        status);                                                                               \
  } while (0)
  const int per_thread = (max_n + 255) / 256;
  if (i8) {
    if (per_thread <= 8) {
      PQI_BATCH_LAUNCH(int8_t, 8);
    } else {
      PQI_BATCH_LAUNCH(int8_t, 16);
    }
  } else {
    if (per_thread <= 8) {
      PQI_BATCH_LAUNCH(float, 8);
    } else {
      PQI_BATCH_LAUNCH(float, 16);
    }
  }
#undef PQI_BATCH_LAUNCH
  PQI_LAUNCHED("batch_search_kernel");
  return PQI_OK;
}

pqi_status pqi_batch_search_warp(const void* graphs, int num_graphs, const int* task_graph,
                                 const uint32_t* init_states, int words_pitch, int tasks,
                                 int max_n, int kind, int is_spin_glass, int rounds, int kick,
                                 int flip_budget, uint64_t seed, const double* kick_cdf,
                                 const long long* cdf_offset, uint32_t* best_states,
                                 double* best_values, unsigned long long* flips_total,
                                 int* status, int warps_per_sm, void* stream) {
  PQI_CHECK_ARG(graphs && num_graphs > 0 && task_graph && init_states && tasks > 0 && max_n > 0);
  PQI_CHECK_ARG(best_states && best_values && flips_total && status && rounds >= 0 && kick >= 0);
  PQI_CHECK_ARG(words_pitch >= (max_n + 31) / 32 && flip_budget > 0);
  PQI_CHECK_ARG(!kick_cdf || cdf_offset);
  PQI_CHECK_ARG(max_n <= 1024 && warps_per_sm >= 0 && warps_per_sm <= 64);
  cudaStream_t s = as_stream(stream);
  const bool i8 = kind == PQI_W_I8;
  static int num_sms = 0;
  if (!num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int NG = max_n <= 128 ? 1 : max_n <= 256 ? 2 : max_n <= 512 ? 4 : 8;
  auto launch = [&](auto kern) -> pqi_status {
    int per_sm = 0;  // resident 128-thread blocks per SM
    PQI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0));
    if (warps_per_sm > 0) per_sm = std::min(per_sm, std::max(1, warps_per_sm / 4));
    per_sm = std::max(1, per_sm);
    const long long want = ((long long)tasks + 3) / 4;
    const int grid = (int)std::max(1ll, std::min(want, (long long)num_sms * per_sm));
    kern<<<grid, 128, 0, s>>>(static_cast<const BatchGraph*>(graphs), task_graph, init_states,
                              words_pitch, tasks, is_spin_glass, rounds, kick, flip_budget, seed,
                              kick_cdf, cdf_offset, best_states, best_values, flips_total, status);
    return PQI_OK;
  };
  pqi_status st;
  if (i8) {
    st = NG == 1   ? launch(warp_search_kernel<int8_t, 1>)
         : NG == 2 ? launch(warp_search_kernel<int8_t, 2>)
         : NG == 4 ? launch(warp_search_kernel<int8_t, 4>)
                   : launch(warp_search_kernel<int8_t, 8>);
  } else {
    st = NG == 1   ? launch(warp_search_kernel<float, 1>)
         : NG == 2 ? launch(warp_search_kernel<float, 2>)
         : NG == 4 ? launch(warp_search_kernel<float, 4>)
                   : launch(warp_search_kernel<float, 8>);
  }
  if (st != PQI_OK) return st;
  PQI_LAUNCHED("warp_search_kernel");
  return PQI_OK;
}

}  // extern "C"
