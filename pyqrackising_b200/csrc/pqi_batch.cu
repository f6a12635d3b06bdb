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
#include <climits>
#include <type_traits>

#include "pqi_common.cuh"
#include "pqi_tc.cuh"

namespace pqi {

struct BatchGraph {
  const void* W;  // prepared copy: int8 (kind PQI_W_I8) or float32 zero-diagonal (PQI_W_F32)
  int n;
  int ld;
  int kind;
  int pad;
  double upper_sum;
  // optional row lists of the graph's nonzero weights (row r: columns
  // adj_col[adj_ptr[r] .. adj_ptr[r+1]) ascending, values adj_val; the
  // diagonal may be listed and is skipped): the starting fields then cost
  // O(nonzeros) instead of O(n^2)
  const long long* adj_ptr;
  const int* adj_col;
  const float* adj_val;
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

// Shared-memory position of node v's field in a CTA of BT threads (BT a power
// of two): node v = 4 t + 4 BT j + i (thread t's group j, lane i of the group)
// sits at (4 j + i) * BT + t, so a warp's accesses in the flip pass are
// contiguous. Holds ceil(n / (4 BT)) * 4 BT entries.
template <int BT>
__device__ __forceinline__ int fpos(int v) {
  return (((v / (4 * BT)) << 2) + (v & 3)) * BT + ((v >> 2) & (BT - 1));
}

template <typename WT, typename GT>
struct TaskCtx {
  const WT* W;
  int n, ld;
  GT* g;  // local fields y = W x
  uint32_t* bits;
  WT* stage;  // staged row groups (kStageGroups x threads x 4 weights), or null
};

// Row groups per thread that the staged form copies with cp.async (no
// registers held while in flight) on top of the CH groups loaded to registers.
constexpr int kStageGroups = 4;

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}

// Node for a uniform draw u in [0, 1): from the normalised cumulative array
// `cdf` (first entry above u) or uniformly.
__device__ __forceinline__ int draw_node(double u, int n, const double* __restrict__ cdf) {
  if (cdf) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (cdf[mid] > u) {
        hi = mid;
      } else {
        lo = mid + 1;
      }
    }
    return lo;
  }
  const int pick = (int)(u * n);
  return pick >= n ? n - 1 : pick;
}

__device__ __forceinline__ unsigned long long bkey(float gv, int v, int xv) {
  return ((unsigned long long)ord_f32(gv) << 32) |
         (unsigned long long)(((0x3FFFFFFFu - (uint32_t)v) << 1) | (uint32_t)xv);
}

__device__ __forceinline__ unsigned long long bmax_key(unsigned long long key) {
  const uint32_t hi = __reduce_max_sync(0xFFFFFFFFu, (uint32_t)(key >> 32));
  const uint32_t lo =
      __reduce_max_sync(0xFFFFFFFFu, ((uint32_t)(key >> 32) == hi) ? (uint32_t)key : 0u);
  return ((unsigned long long)hi << 32) | lo;
}

// The task keeps the local field y = W x (x = 2s - 1) instead of the gains:
// the gain of node v is g_v = x_v y_v, and flipping node k changes every
// field by y_v -= 2 x_k W_kv (W's prepared copy has a zero diagonal, so y_k is
// unchanged). One fused pass per flip, one CTA barrier: each thread owns
// groups of four consecutive nodes v = 4 t + 4 BT j + i, loads CH groups of
// row k at once (float4 / char4), updates their fields, toggles bit k if it
// owns k (the only writer of that bit; the other nodes of the word are read
// by their own threads only), and folds the new gains into a key (float gain,
// then the lowest node, then the node's bit). Warp maxima go to a slot array
// chosen by the pass parity; after the barrier every warp reduces the slots
// itself, so the next pass starts without a second barrier (a warp can be at
// most one pass ahead of another, which writes the other slot array).
// k < 0: no flip, only the selection. Returns the key and the exact gain of
// the selected node. With float32 fields the pass also sums x_v W_kv over row
// k as it streams by (per thread a compensated float pair, across threads in
// float64): *out_gx = x_k sum_v x_v W_kv is then the gain of the flipped node
// k to float64 accuracy (its acceptance test and the running value use it; the
// float32 fields only rank the candidates). The partial sums ride on the same
// barrier as the selection.
template <typename WT, typename GT, int CH, bool STG, int BT>
__device__ __forceinline__ void flip_and_select(const TaskCtx<WT, GT>& c, int k, int xk,
                                                unsigned long long (*red_key)[8],
                                                double (*red_x)[8], int par,
                                                unsigned long long* out_key, double* out_g,
                                                double* out_gx) {
  constexpr bool GX = std::is_same<GT, float>::value;
  // this thread's share of sum_v x_v W_kv (GX) as an unevaluated float pair
  // px_hi + px_lo: each term is added with an error-free two-sum, so the pair
  // holds the sum to about 2^-47 of its magnitude without a float64
  // conversion per term (those run on the slow conversion pipe)
  float px_hi = 0.0f, px_lo = 0.0f;
  const int n = c.n;
  const GT coef = (k >= 0) ? (xk ? (GT)-2 : (GT)2) : (GT)0;
  const WT* __restrict__ row = c.W + (size_t)(k >= 0 ? k : 0) * c.ld;
  float bv = -INFINITY;
  int bi = -1;
  // The selection compares gains as float32, lowest node on ties. Per field
  // type the comparison uses as few conversions as give the same result:
  // float fields compare in float (no conversion); int fields compare as int
  // (exact in float below 2^24, more than 127 x the largest n); double fields
  // round each field to float once (rounding is symmetric, so the gain's
  // float is +-the field's). Only the best node is kept per thread; its bit
  // and the winner's exact gain are read back after the selection.
  int bint = INT_MIN;
  constexpr int stride = 4 * BT;  // 4 nodes x BT threads
  // one group of four nodes v0 .. v0 + 3 with their weights of row k
  // (v0 is a multiple of four: node v0 + i sits at fpos(v0) + BT i)
  auto group = [&](int v0, const WT* w4) {
    if ((unsigned)(k - v0) < 4u) c.bits[k >> 5] ^= 1u << (k & 31);
    const uint32_t nib = c.bits[v0 >> 5] >> (v0 & 31);  // bits of v0 .. v0 + 3
    GT* const g0 = c.g + fpos<BT>(v0);
    const bool full = v0 + 3 < n;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (full || v0 + i < n) {
        GT y = g0[BT * i];
        if (k >= 0) {
          y += coef * (GT)w4[i];
          g0[BT * i] = y;
        }
        const uint32_t xv = (nib >> i) & 1u;
        if constexpr (GX) {
          // bit k may already be toggled here; W_kk = 0 in the prepared copy
          if (k >= 0) {
            const float t0 = xv ? (float)w4[i] : -(float)w4[i];
            const float t = px_hi + t0;
            const float bb = t - px_hi;
            px_lo += (px_hi - (t - bb)) + (t0 - bb);
            px_hi = t;
          }
        }
        // v ascends within a thread: strict '>' keeps the lowest node
        if constexpr (std::is_same<GT, int>::value) {
          const int gi = xv ? y : -y;
          if (gi > bint) {
            bint = gi;
            bi = v0 + i;
          }
        } else {
          const float yf = (float)y;
          const float gv = xv ? yf : -yf;
          if (gv > bv) {
            bv = gv;
            bi = v0 + i;
          }
        }
      }
    }
  };
  constexpr int PER = STG ? CH + kStageGroups : CH;  // groups per pass
  for (int base = 4 * threadIdx.x; base < n; base += PER * stride) {
    if constexpr (STG) {
      // the pass's last kStageGroups groups go to shared memory first, so the
      // whole pass is in flight while the register groups are waited on; each
      // thread reads back only the slots it copied itself
      if (k >= 0) {
#pragma unroll
        for (int j = 0; j < kStageGroups; ++j) {
          const int v = base + (CH + j) * stride;
          if (v < n)
            cp_async16(c.stage + (size_t)(j * BT + threadIdx.x) * 4, row + v,
                       (n - v) >= 4 ? 16 : (n - v) * (int)sizeof(WT));
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
      }
    }
    WT w[4 * CH];
    if (k >= 0) {
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int v = base + j * stride;
        if (v + 3 < n) {
          if constexpr (sizeof(WT) == 4) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(row + v));
            w[4 * j] = t.x; w[4 * j + 1] = t.y; w[4 * j + 2] = t.z; w[4 * j + 3] = t.w;
          } else {
            const char4 t = __ldg(reinterpret_cast<const char4*>(row + v));
            w[4 * j] = t.x; w[4 * j + 1] = t.y; w[4 * j + 2] = t.z; w[4 * j + 3] = t.w;
          }
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i) w[4 * j + i] = (v + i < n) ? __ldg(row + v + i) : (WT)0;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < CH; ++j) {
      const int v0 = base + j * stride;
      if (v0 < n) group(v0, w + 4 * j);
    }
    if constexpr (STG) {
      if (k >= 0) asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
      for (int j = 0; j < kStageGroups; ++j) {
        const int v0 = base + (CH + j) * stride;
        if (v0 < n) {
          WT w4[4] = {(WT)0, (WT)0, (WT)0, (WT)0};
          if (k >= 0) {
            const float4 t =
                *reinterpret_cast<const float4*>(c.stage + (size_t)(j * BT + threadIdx.x) * 4);
            w4[0] = t.x; w4[1] = t.y; w4[2] = t.z; w4[3] = t.w;
          }
          group(v0, w4);
        }
      }
    }
  }
  if constexpr (std::is_same<GT, int>::value) bv = (float)bint;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // (bit bi is written only by this thread, the owner of node bi)
  const int bx = bi >= 0 ? (int)((c.bits[bi >> 5] >> (bi & 31)) & 1u) : 0;
  const unsigned long long key = bi >= 0 ? bkey(bv, bi, bx) : 0ull;
  const unsigned long long wk = bmax_key(key);
  if (lane == 0) red_key[par][warp] = wk;
  if constexpr (GX) {
    double px = (double)px_hi + (double)px_lo;
    for (int o = 16; o > 0; o >>= 1) px += __shfl_xor_sync(0xFFFFFFFFu, px, o);
    if (lane == 0) red_x[par][warp] = px;
  }
  __syncthreads();
  const int nwarps = blockDim.x >> 5;
  const unsigned long long sk = lane < nwarps ? red_key[par][lane] : 0ull;
  const unsigned long long gk = bmax_key(sk);
  // the winner's gain from its field: written before the barrier, and a
  // warp already in the next pass (which flips the winner) leaves it as it
  // is (W_kk = 0)
  double g_win = 0.0;
  if (gk != 0ull) {
    const int kw = (int)(0x3FFFFFFFu - ((uint32_t)gk >> 1));
    const double y = (double)c.g[fpos<BT>(kw)];
    g_win = (gk & 1ull) ? y : -y;
  }
  *out_g = g_win;
  *out_key = gk;
  if constexpr (GX) {
    // every warp sums the slots in the same order: one value CTA-wide
    double sx = 0.0;
    for (int i = 0; i < nwarps; ++i) sx += red_x[par][i];
    *out_gx = xk ? sx : -sx;
  } else {
    *out_gx = 0.0;
  }
}

// Starting local fields of many tasks at once, for graphs without row lists:
// Y[t][v] = sum_u x_tu W[u][v] (x = +-1), u ascending from 0 - the order and
// the accumulation type (float64 for float weights, int32 for int8) of the
// search kernel's own column-order sum, so the fields are the same numbers.
// A CTA takes SF_T tasks x SF_V nodes: each row chunk of W (SF_U rows) is
// read once into shared memory (converted once) and used by all SF_T tasks,
// instead of every task streaming all of W. The tasks of a tile may belong to
// different graphs: the tile runs once per distinct graph among its tasks
// (one pass for tasks grouped by graph). Row-list graphs are skipped (the
// search kernel sums their nonzeros itself).
constexpr int SF_T = 64;
constexpr int SF_V = 64;
constexpr int SF_U = 32;

template <typename WT>
__global__ void __launch_bounds__(256) start_fields_kernel(
    const BatchGraph* __restrict__ graphs, const int* __restrict__ task_graph,
    const uint32_t* __restrict__ init_states, int words_pitch, int tasks,
    double* __restrict__ Y, int ypitch) {
  typedef typename std::conditional<sizeof(WT) == 1, int, double>::type AT;
  __shared__ __align__(16) AT Ws[SF_U][SF_V];
  __shared__ uint32_t Xs[SF_T];
  __shared__ int gid[SF_T];
  const int t0 = blockIdx.x * SF_T, v0 = blockIdx.y * SF_V;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // nodes v0+4tx+i, tasks t0+4ty+j
  if (threadIdx.x < SF_T) gid[threadIdx.x] = t0 + (int)threadIdx.x < tasks ? task_graph[t0 + threadIdx.x] : -1;
  __syncthreads();
  uint64_t done = 0;  // tile tasks handled (the same in every thread)
  for (int i = 0; i < SF_T; ++i)
    if (gid[i] < 0) done |= 1ull << i;
  while (done != ~0ull) {
    const int g = gid[__ffsll((long long)~done) - 1];
    uint64_t mine = 0;
    for (int i = 0; i < SF_T; ++i)
      if (gid[i] == g) mine |= 1ull << i;
    done |= mine;
    const BatchGraph G = graphs[g];
    if (G.adj_ptr || v0 >= G.n) continue;
    const WT* __restrict__ W = static_cast<const WT*>(G.W);
    const int n = G.n;
    AT acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0;
    for (int u0 = 0; u0 < n; u0 += SF_U) {
      __syncthreads();  // the previous chunk's reads are done
      for (int idx = threadIdx.x; idx < SF_U * SF_V; idx += blockDim.x) {
        const int r = idx / SF_V, c = idx - r * SF_V;
        const int u = u0 + r, v = v0 + c;
        Ws[r][c] = (u < n && v < n) ? (AT)__ldg(W + (size_t)u * G.ld + v) : (AT)0;
      }
      if (threadIdx.x < SF_T)
        Xs[threadIdx.x] = ((mine >> threadIdx.x) & 1ull)
                              ? __ldg(init_states + (size_t)(t0 + threadIdx.x) * words_pitch + (u0 >> 5))
                              : 0u;
      __syncthreads();
      uint32_t xw[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) xw[j] = Xs[4 * ty + j];
      // acc += (+-1) w as one fused multiply-add with an exact product: the
      // same rounding as the add of +-w, and the sign is chosen once per task
      // and row instead of once per element
      auto row = [&](int r) {
        AT w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = Ws[r][4 * tx + i];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const AT sj = ((xw[j] >> r) & 1u) ? (AT)1 : (AT)-1;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            if constexpr (std::is_same<AT, double>::value) {
              acc[i][j] = fma(sj, w[i], acc[i][j]);
            } else {
              acc[i][j] += sj * w[i];
            }
          }
        }
      };
      if (n - u0 >= SF_U) {
#pragma unroll 8
        for (int r = 0; r < SF_U; ++r) row(r);
      } else {
        for (int r = 0; r < n - u0; ++r) row(r);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (!((mine >> (4 * ty + j)) & 1ull)) continue;
      const int t = t0 + 4 * ty + j;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int v = v0 + 4 * tx + i;
        if (v < n) Y[(size_t)t * ypitch + v] = (double)acc[i][j];
      }
    }
  }
}

// F32: float graphs keep float32 local fields (half the shared memory and
// fewer registers, so more resident tasks per SM); gains, the selection rule
// and the float64 running value are unchanged in form.
// STG (float32 fields only): each flip pass also stages kStageGroups row
// groups per thread through cp.async, so a pass of SK n = 8192 has its whole
// 32 KB row in flight at once instead of in two register chunks.
// BT: threads per CTA (256; 128 or 64 for small graphs: two or four times the
// resident tasks per SM, at the same registers per thread).
template <typename WT, int CH, bool F32, bool STG, int BT>
__global__ void __launch_bounds__(BT, (F32 ? 4 : 3) * 256 / BT) batch_search_kernel(
    const BatchGraph* __restrict__ graphs, const int* __restrict__ task_graph,
    const uint32_t* __restrict__ init_states, int words_pitch, int tasks, int spin, int rounds,
    int kick, int flip_budget, uint64_t seed, const double* __restrict__ kick_cdf,
    const long long* __restrict__ cdf_offset, uint32_t* __restrict__ best_states,
    double* __restrict__ best_values, unsigned long long* __restrict__ flips_total,
    int* __restrict__ status, const double* __restrict__ start_fields, int fields_pitch) {
  typedef typename std::conditional<
      sizeof(WT) == 1, int, typename std::conditional<F32, float, double>::type>::type GT;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[32];
  __shared__ unsigned long long red_key[2][8];
  __shared__ double red_x[2][8];
  for (int task = blockIdx.x; task < tasks; task += gridDim.x) {
    const BatchGraph G = graphs[task_graph[task]];
    const int n = G.n, n32 = (n + 31) >> 5;
    TaskCtx<WT, GT> c;
    c.W = static_cast<const WT*>(G.W);
    c.n = n;
    c.ld = G.ld;
    c.bits = reinterpret_cast<uint32_t*>(smem);
    c.g = reinterpret_cast<GT*>(smem + (((size_t)n32 * 4 + 15) & ~size_t(15)));
    uint32_t* kicked = reinterpret_cast<uint32_t*>(
        smem + (((size_t)n32 * 4 + 15) & ~size_t(15)) +
        (size_t)((n + 4 * BT - 1) / (4 * BT) * (4 * BT)) * sizeof(GT));
    static_assert(!STG || (F32 && sizeof(WT) == 4), "staged groups: float rows, float32 fields");
    c.stage = STG ? reinterpret_cast<WT*>(reinterpret_cast<unsigned char*>(kicked) +
                                          (((size_t)n32 * 4 + 15) & ~size_t(15)))
                  : nullptr;
    uint32_t* best_bits = best_states + (size_t)task * words_pitch;
    for (int w = threadIdx.x; w < n32; w += blockDim.x) c.bits[w] = init_states[(size_t)task * words_pitch + w];
    __syncthreads();
    // 1. local fields of the starting state, y_v = sum_u x_u W_uv (W is
    // symmetric). With row lists, each field sums its own row's nonzero
    // entries in column order (the dense column-order sum without its zero
    // terms). Else, below 2048 nodes a warp per row (row dot product, shuffle
    // reduction): more rows in flight per CTA; from 2048 nodes every row u adds
    // +-W_u to each thread's own nodes (rows ascending, CH groups of four per
    // pass in registers): a memory stream with few instructions, which leaves
    // the SM to the flips of the other resident tasks.
    // Float32 fields are summed in float64 and rounded once when stored; the
    // thread that stores field v also adds x_v y_v (float64) to its share of
    // q = x^T W x, so the starting value is the float64 one for every field type.
    typedef typename std::conditional<F32, double, GT>::type AT;
    double qpart = 0.0;
    auto store_field = [&](int v, AT acc) {
      c.g[fpos<BT>(v)] = (GT)acc;
      qpart += ((c.bits[v >> 5] >> (v & 31)) & 1) ? (double)acc : -(double)acc;
    };
    if (start_fields && !G.adj_ptr) {
      // computed for all tasks beforehand (start_fields_kernel)
      const double* __restrict__ yrow = start_fields + (size_t)task * fields_pitch;
      for (int v = threadIdx.x; v < n; v += blockDim.x) store_field(v, (AT)yrow[v]);
    } else if (G.adj_ptr) {
      for (int v = threadIdx.x; v < n; v += blockDim.x) {
        AT acc = 0;
        const long long e1 = G.adj_ptr[v + 1];
        for (long long e = G.adj_ptr[v]; e < e1; ++e) {
          const int u = G.adj_col[e];
          if (u == v) continue;
          const AT w = (AT)G.adj_val[e];
          acc += ((c.bits[u >> 5] >> (u & 31)) & 1) ? w : -w;
        }
        store_field(v, acc);
      }
    } else if (n < 2048) {
      const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
      for (int k = threadIdx.x >> 5; k < n; k += warps) {
        const WT* row = c.W + (size_t)k * c.ld;
        AT acc = 0;
        for (int v = lane; v < n; v += 32) {
          const AT w = (AT)row[v];
          acc += ((c.bits[v >> 5] >> (v & 31)) & 1) ? w : -w;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
        if (lane == 0) store_field(k, acc);
      }
    } else {
      // at most two groups per pass: eight accumulators keep the register
      // budget of three resident CTAs per SM. Float32 fields sum each field
      // as an unevaluated float pair (error-free two-sum per term: float32
      // adds only, no float64 conversion per term), so the field and the
      // starting value are float64-accurate.
      constexpr int CI = F32 ? 1 : (CH > 2 ? 2 : CH);  // (float pairs: one group)
      for (int base = 4 * threadIdx.x; base < n; base += CI * 4 * BT) {
        GT acc[4 * CI];
        float alo[F32 ? 4 * CI : 1];
#pragma unroll
        for (int e = 0; e < 4 * CI; ++e) acc[e] = 0;
#pragma unroll
        for (int e = 0; e < (F32 ? 4 * CI : 1); ++e) alo[e] = 0.0f;
#pragma unroll 2
        for (int u = 0; u < n; ++u) {
          const WT* __restrict__ row = c.W + (size_t)u * c.ld;
          const bool xu = (c.bits[u >> 5] >> (u & 31)) & 1u;
#pragma unroll
          for (int j = 0; j < CI; ++j) {
            const int v = base + j * 4 * BT;
            if (v < n) {
              WT w4[4];
              if (v + 3 < n) {
                if constexpr (sizeof(WT) == 4) {
                  const float4 t = __ldg(reinterpret_cast<const float4*>(row + v));
                  w4[0] = t.x; w4[1] = t.y; w4[2] = t.z; w4[3] = t.w;
                } else {
                  const char4 t = __ldg(reinterpret_cast<const char4*>(row + v));
                  w4[0] = t.x; w4[1] = t.y; w4[2] = t.z; w4[3] = t.w;
                }
              } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) w4[i] = (v + i < n) ? __ldg(row + v + i) : (WT)0;
              }
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                if constexpr (F32) {
                  const float y = xu ? (float)w4[i] : -(float)w4[i];
                  const float t = acc[4 * j + i] + y;
                  const float bb = t - acc[4 * j + i];
                  alo[4 * j + i] += (acc[4 * j + i] - (t - bb)) + (y - bb);
                  acc[4 * j + i] = t;
                } else {
                  acc[4 * j + i] += xu ? (GT)w4[i] : -(GT)w4[i];
                }
              }
            }
          }
        }
#pragma unroll
        for (int j = 0; j < CI; ++j)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int v = base + j * 4 * BT + i;
            if constexpr (F32) {
              if (v < n) store_field(v, (double)acc[4 * j + i] + (double)alo[4 * j + i]);
            } else {
              if (v < n) store_field(v, acc[4 * j + i]);
            }
          }
      }
    }
    __syncthreads();
    // q = x^T W x = sum_k x_k y_k; value from q
    double part = qpart;
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
    unsigned long long key;
    double gk, gx;
    int par = 0;
    flip_and_select<WT, GT, CH, STG, BT>(c, -1, 0, red_key, red_x, par, &key, &gk, &gx);
    par ^= 1;
    for (int r = 0; r <= rounds; ++r) {
      // steepest ascent: flip the best node while its gain is positive
      for (int f = 0;; ++f) {
        if (key == 0ull || !(unord_f32((uint32_t)(key >> 32)) > 0.0f)) break;
        if (f >= flip_budget) {
          timeout = 1;
          break;
        }
        const int k = (int)(0x3FFFFFFFu - (((uint32_t)key) >> 1));
        const int xk = (int)(key & 1ull);
        const double gprev = gk;  // gain of k before the flip (exact for int / float64 fields)
        // float32 fields rank the candidates; the float64 gain of k, summed over
        // row k in the same pass, decides: not positive -> a second pass undoes
        // the flip and the ascent stops (one call site for both passes)
        bool undone = false;
#pragma unroll 1
        for (int pass = 0; pass < 2; ++pass) {
          flip_and_select<WT, GT, CH, STG, BT>(c, k, xk ^ pass, red_key, red_x, par, &key, &gk, &gx);
          par ^= 1;
          if (pass == 1 || !F32 || gx > 0.0) {
            undone = pass == 1;
            break;
          }
        }
        if (undone) break;
        val += scale * (F32 ? gx : gprev);
        ++nflips;
      }
      if (val > best) {
        best = val;
        for (int w = threadIdx.x; w < n32; w += blockDim.x) best_bits[w] = c.bits[w];
      }
      if (r == rounds) break;
      // kick: forced flips; every thread draws the same node, without
      // replacement within the round (a node drawn twice would undo its kick;
      // after 16 draws that all hit kicked nodes the last draw is taken)
      for (int w = threadIdx.x; w < n32; w += blockDim.x) kicked[w] = 0u;
      __syncthreads();
      for (int j = 0; j < kick; ++j) {
        int pick = 0;
        for (int attempt = 0; attempt < 16; ++attempt) {
          const double u =
              bunif(seed, (uint64_t)task * 1315423911ull + r, (uint64_t)j + ((uint64_t)attempt << 20));
          pick = draw_node(u, n, kick_cdf ? kick_cdf + cdf_offset[task_graph[task]] : nullptr);
          if (!((kicked[pick >> 5] >> (pick & 31)) & 1u)) break;
        }
        const int xp = (c.bits[pick >> 5] >> (pick & 31)) & 1;
        const double gp = xp ? (double)c.g[fpos<BT>(pick)] : -(double)c.g[fpos<BT>(pick)];
        __syncthreads();  // everyone has read bit, field and kicked set before they change
        if (threadIdx.x == 0) kicked[pick >> 5] |= 1u << (pick & 31);
        flip_and_select<WT, GT, CH, STG, BT>(c, pick, xp, red_key, red_x, par, &key, &gk, &gx);
        par ^= 1;
        val += scale * (F32 ? gx : gp);  // float64 gain of the kicked node
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
// Float64 local fields in tensor memory (float weights, 4096 < n <= 16384).
//
// The shared-memory form holds a task's float64 fields in shared memory:
// 64 KB at n = 8192, three tasks per SM, and each flip streams its 32 KB row in
// two register chunks. Here the fields live in the SM's tensor memory (TMEM,
// 128 lanes x 512 columns of 32 bits): a CTA of 128 threads allocates 8 J
// columns, thread t keeps its 4 J nodes' fields in its own lane (node
// v = 4 t + 512 j + i at columns 2 (4 j + i) and 2 (4 j + i) + 1), 512 / 8 J
// tasks per SM share the columns, and shared memory is left for the row:
// one bulk copy of the whole row per flip (mbarrier completion). A flip pass
// moves the fields through registers 32 columns (16 nodes) at a time with
// tcgen05.ld / tcgen05.st; the arithmetic, the selection (float gain, lowest
// node, the node's bit) and the float64 running value are those of the
// shared-memory form, so both return the same states, values and flip counts.
// Each CTA asks for enough shared memory that no further CTA can join an SM
// whose TMEM the resident CTAs hold.
// The shape per J (groups of four nodes per thread): J = 16 serves n <= 8192
// (128 columns, four CTAs per SM), J = 32 serves n <= 16384 (256 columns, two
// CTAs per SM, where the fields in shared memory leave one).
constexpr int TM_BT = 128;
template <int J>
struct TmShape {
  static constexpr int NMAX = 4 * TM_BT * J;      // nodes
  static constexpr int COLS = 2 * 4 * J;          // TMEM columns per CTA
  static constexpr int CTAS = 512 / COLS;         // CTAs sharing an SM's columns
  static constexpr int STAGE_BYTES = NMAX * 4;    // one float32 row
  // shared memory per CTA: the stage, bits and kicked set, and at least
  // enough that a further CTA cannot join an SM whose TMEM is taken
  static constexpr int SMEM = (228 * 1024) / (CTAS + 1) + 4096 > STAGE_BYTES + NMAX / 4
                                  ? (228 * 1024) / (CTAS + 1) + 4096
                                  : STAGE_BYTES + NMAX / 4;
};

__device__ __forceinline__ void tm_st32(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, "
      "%17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]),
      "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]),
      "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ double tm_ld_f64(uint32_t taddr) {
  uint32_t lo, hi;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(lo), "=r"(hi) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  return __hiloint2double((int)hi, (int)lo);
}

struct TmCtx {
  const float* W;
  int n, ld;
  uint32_t* bits;
  const float* stage;  // the flipped row (shared memory)
  uint32_t tbase;      // this warp's lanes, column 0 of the CTA's allocation
};

// One flip pass of the TMEM form: with k >= 0 the row k is in the stage,
// flip k (coefficient -2 x_k) in this thread's fields and bits, and return in
// *out_gk the exact gain of k before the flip (its field is unchanged by its
// own flip, W_kk = 0: the owner warp reads it back once instead of every
// thread keeping the field of its best node); then the CTA's best key.
template <bool UPD, int J>
__device__ __forceinline__ void tm_pass(const TmCtx& c, int k, int xk,
                                        unsigned long long (*red_key)[4], double* s_yk, int par,
                                        unsigned long long* out_key, double* out_gk) {
  const int t = threadIdx.x, n = c.n;
  const double coef = xk ? -2.0 : 2.0;
  float bv = -INFINITY;
  int bi = -1;
#pragma unroll 1
  for (int q = 0; q < J / 4; ++q) {
    if (2048 * q >= n) break;  // (uniform: no node of this chunk below n)
    uint32_t r[32];
    tc::tmem_load32(c.tbase + 32u * q, r);
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int v0 = 4 * t + 512 * (4 * q + jj);
      if (v0 >= n) continue;
      float w4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      if (UPD) {
        const float4 s4 = *reinterpret_cast<const float4*>(c.stage + v0);
        w4[0] = s4.x; w4[1] = s4.y; w4[2] = s4.z; w4[3] = s4.w;
        if ((unsigned)(k - v0) < 4u) c.bits[k >> 5] ^= 1u << (k & 31);
      }
      const uint32_t nib = c.bits[v0 >> 5] >> (v0 & 31);
      const bool full = v0 + 3 < n;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (full || v0 + i < n) {
          const int s = 8 * jj + 2 * i;
          double y = __hiloint2double((int)r[s + 1], (int)r[s]);
          if (UPD) {
            y += coef * (double)w4[i];
            r[s] = (uint32_t)__double2loint(y);
            r[s + 1] = (uint32_t)__double2hiint(y);
          }
          const float yf = (float)y;
          const float gv = ((nib >> i) & 1u) ? yf : -yf;
          if (gv > bv) {
            bv = gv;
            bi = v0 + i;
          }
        }
      }
    }
    if (UPD) tm_st32(c.tbase + 32u * q, r);
  }
  const int lane = t & 31, warp = t >> 5;
  if (UPD) {
    tm_wait_st();
    const int owner = (k >> 2) & (TM_BT - 1);
    if (warp == owner >> 5) {
      const double y = tm_ld_f64(c.tbase + 2u * (uint32_t)(4 * (k / 512) + (k & 3)));
      if (lane == (owner & 31)) s_yk[par] = y;
    }
  }
  const int bx = bi >= 0 ? (int)((c.bits[bi >> 5] >> (bi & 31)) & 1u) : 0;
  const unsigned long long key = bi >= 0 ? bkey(bv, bi, bx) : 0ull;
  const unsigned long long wk = bmax_key(key);
  const uint32_t src = __ballot_sync(0xFFFFFFFFu, key == wk && wk != 0ull);
  if (lane == (src ? __ffs(src) - 1 : 0)) red_key[par][warp] = wk;
  __syncthreads();
  const unsigned long long sk = lane < 4 ? red_key[par][lane] : 0ull;
  *out_key = bmax_key(sk);
  if (UPD) *out_gk = xk ? s_yk[par] : -s_yk[par];
}

template <int J>
__global__ void __launch_bounds__(TM_BT, TmShape<J>::CTAS) batch_search_tmem_kernel(
    const BatchGraph* __restrict__ graphs, const int* __restrict__ task_graph,
    const uint32_t* __restrict__ init_states, int words_pitch, int tasks, int spin, int rounds,
    int kick, int flip_budget, uint64_t seed, const double* __restrict__ kick_cdf,
    const long long* __restrict__ cdf_offset, uint32_t* __restrict__ best_states,
    double* __restrict__ best_values, unsigned long long* __restrict__ flips_total,
    int* __restrict__ status, const double* __restrict__ start_fields, int fields_pitch) {
  extern __shared__ __align__(16) unsigned char tm_smem[];
  __shared__ double red[4];
  __shared__ unsigned long long red_key[2][4];
  __shared__ double s_yk[2];
  __shared__ __align__(8) uint64_t row_bar;
  __shared__ uint32_t s_tmem;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  float* stage = reinterpret_cast<float*>(tm_smem);
  typedef TmShape<J> SH;
  uint32_t* bits = reinterpret_cast<uint32_t*>(tm_smem + SH::STAGE_BYTES);
  uint32_t* kicked = bits + SH::NMAX / 32;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&s_tmem)),
                 "r"(SH::COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) {
    tc::mbar_init(&row_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  uint32_t phase = 0;
  bool failed = false;
  for (int task = blockIdx.x; task < tasks && !failed; task += gridDim.x) {
    const BatchGraph G = graphs[task_graph[task]];
    const int n = G.n, n32 = (n + 31) >> 5;
    TmCtx c;
    c.W = static_cast<const float*>(G.W);
    c.n = n;
    c.ld = G.ld;
    c.bits = bits;
    c.stage = stage;
    c.tbase = s_tmem + ((uint32_t)(32 * warp) << 16);
    uint32_t* best_bits = best_states + (size_t)task * words_pitch;
    for (int w = t; w < n32; w += TM_BT) bits[w] = init_states[(size_t)task * words_pitch + w];
    __syncthreads();
    // 1. starting fields of this thread's own nodes (from the start pass, or
    // summed over the node's row list), stored to TMEM 16 nodes at a time;
    // x_v y_v into this thread's share of q = x^T W x
    double qpart = 0.0;
    const double* __restrict__ yrow =
        (start_fields && !G.adj_ptr) ? start_fields + (size_t)task * fields_pitch : nullptr;
#pragma unroll 1
    for (int q = 0; q < J / 4; ++q) {
      uint32_t r[32];
#pragma unroll
      for (int s = 0; s < 16; ++s) {
        const int v = 4 * t + 512 * (4 * q + (s >> 2)) + (s & 3);
        double y = 0.0;
        if (v < n) {
          if (yrow) {
            y = yrow[v];
          } else {
            const long long e1 = G.adj_ptr[v + 1];
            for (long long e = G.adj_ptr[v]; e < e1; ++e) {
              const int u = G.adj_col[e];
              if (u == v) continue;
              const double w = (double)G.adj_val[e];
              y += ((bits[u >> 5] >> (u & 31)) & 1) ? w : -w;
            }
          }
          qpart += ((bits[v >> 5] >> (v & 31)) & 1) ? y : -y;
        }
        r[2 * s] = (uint32_t)__double2loint(y);
        r[2 * s + 1] = (uint32_t)__double2hiint(y);
      }
      tm_st32(c.tbase + 32u * q, r);
    }
    tm_wait_st();
    for (int o = 16; o > 0; o >>= 1) qpart += __shfl_xor_sync(0xFFFFFFFFu, qpart, o);
    if (lane == 0) red[warp] = qpart;
    __syncthreads();
    const double qv = red[0] + red[1] + red[2] + red[3];
    const double scale = spin ? 2.0 : 1.0;
    double val = spin ? -qv / 2.0 : (2.0 * G.upper_sum - qv) / 4.0;
    double best = -INFINITY;
    unsigned long long nflips = 0;
    int timeout = 0;
    unsigned long long key;
    double gflip = 0.0;  // the gain of the node the last pass flipped, before the flip
    int par = 0;
    // the row of node k into the stage by one bulk copy (every thread has
    // finished reading the previous row: the pass before ended on a CTA
    // barrier)
    auto flip = [&](int k, int xk) -> bool {
      if (t == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint32_t bytes = (uint32_t)(((n + 3) & ~3) * 4);
        tc::mbar_expect_tx(&row_bar, bytes);
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                tc::smem_u32(stage)),
            "l"(c.W + (size_t)k * c.ld), "r"(bytes), "r"(tc::smem_u32(&row_bar))
            : "memory");
      }
      // (one lane per warp waits, bounded; the CTA then agrees, so a wait
      // that ran out anywhere stops the task everywhere)
      bool ok = true;
      if (lane == 0) ok = tc::mbar_wait_spin(&row_bar, phase);
      ok = __syncthreads_and(ok ? 1 : 0) != 0;
      phase ^= 1u;
      if (!ok) return false;
      tm_pass<true, J>(c, k, xk, red_key, s_yk, par, &key, &gflip);
      par ^= 1;
      return true;
    };
    tm_pass<false, J>(c, -1, 0, red_key, s_yk, par, &key, &gflip);
    par ^= 1;
    for (int r = 0; r <= rounds && !failed; ++r) {
      for (int f = 0;; ++f) {
        if (key == 0ull || !(unord_f32((uint32_t)(key >> 32)) > 0.0f)) break;
        if (f >= flip_budget) {
          timeout = 1;
          break;
        }
        const int k = (int)(0x3FFFFFFFu - (((uint32_t)key) >> 1));
        const int xk = (int)(key & 1ull);
        if (!flip(k, xk)) {
          failed = true;
          break;
        }
        val += scale * gflip;
        ++nflips;
      }
      if (failed) break;
      if (val > best) {
        best = val;
        for (int w = t; w < n32; w += TM_BT) best_bits[w] = bits[w];
      }
      if (r == rounds) break;
      for (int w = t; w < n32; w += TM_BT) kicked[w] = 0u;
      __syncthreads();
      for (int j = 0; j < kick; ++j) {
        int pick = 0;
        for (int attempt = 0; attempt < 16; ++attempt) {
          const double u =
              bunif(seed, (uint64_t)task * 1315423911ull + r, (uint64_t)j + ((uint64_t)attempt << 20));
          pick = draw_node(u, n, kick_cdf ? kick_cdf + cdf_offset[task_graph[task]] : nullptr);
          if (!((kicked[pick >> 5] >> (pick & 31)) & 1u)) break;
        }
        const int xp = (bits[pick >> 5] >> (pick & 31)) & 1;
        __syncthreads();  // everyone has read bit and kicked set before they change
        if (t == 0) kicked[pick >> 5] |= 1u << (pick & 31);
        if (!flip(pick, xp)) {
          failed = true;
          break;
        }
        val += scale * gflip;  // float64 gain of the kicked node
        ++nflips;
      }
    }
    if (t == 0) {
      best_values[task] = best;
      atomicAdd(flips_total, nflips);
      if (timeout) atomicExch(status, PQI_ETIMEOUT);
      if (failed) atomicExch(status, PQI_ETIMEOUT);
    }
    __syncthreads();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(SH::COLS)
                 : "memory");
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
      bs >= 0 ? bkey(bv, 128 * (bs >> 2) + 4 * lane + (bs & 3), bx) : 0ull;
  const unsigned long long wk = bmax_key(key);
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
      // kicks without replacement within the round (as the CTA form): the
      // kicked set lives in each lane's register, one bit per owned node
      uint32_t km = 0;
      for (int j = 0; j < kick; ++j) {
        int pick = 0;
        for (int attempt = 0; attempt < 16; ++attempt) {
          const double u =
              bunif(seed, (uint64_t)task * 1315423911ull + r, (uint64_t)j + ((uint64_t)attempt << 20));
          pick = draw_node(u, n, kick_cdf ? kick_cdf + cdf_offset[task_graph[task]] : nullptr);
          const int ow = (pick & 127) >> 2, sl = 4 * (pick >> 7) + (pick & 3);
          if (!((__shfl_sync(0xFFFFFFFFu, km, ow) >> sl) & 1u)) break;
        }
        // the owner reads the node's bit and exact gain, and marks it kicked
        const int owner = (pick & 127) >> 2, slot = 4 * (pick >> 7) + (pick & 3);
        double g = 0.0;
        int xv = 0;
#pragma unroll
        for (int e = 0; e < 4 * NG; ++e)
          if (e == slot) {
            xv = (xm >> e) & 1;
            g = xv ? (double)y[e] : -(double)y[e];
          }
        if (lane == owner) km |= 1u << slot;
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

// Starting fields of the dense-graph tasks into a stream-ordered buffer (below).
pqi_status start_fields(const void* graphs, const int* task_graph, const uint32_t* init_states,
                        int words_pitch, int tasks, int max_n, bool i8, cudaStream_t s,
                        double** out, int* pitch);

}  // namespace pqi

using namespace pqi;

extern "C" {

size_t pqi_batch_graph_desc_bytes(void) { return sizeof(BatchGraph); }

}  // extern "C"

static int g_batch_no_stage = 0;
static int g_batch_no_tmem = 0;
static int g_batch_no_start_pass = 0;

// Starting fields of the dense-graph tasks (start_fields_kernel) into a
// buffer from the stream-ordered pool, freed by the caller after its launch
// (cudaFreeAsync on the same stream). *out stays null (the search kernels
// then sum their own fields) below 64 nodes or when switched off.
pqi_status pqi::start_fields(const void* graphs, const int* task_graph,
                             const uint32_t* init_states, int words_pitch, int tasks, int max_n,
                             bool i8, cudaStream_t s, double** out, int* pitch) {
  const BatchGraph* gd = static_cast<const BatchGraph*>(graphs);
  *out = nullptr;
  *pitch = 0;
  if (max_n < 64 || g_batch_no_start_pass) return PQI_OK;
  static bool pool_kept = false;
  if (!pool_kept) {
    // keep freed pool memory for the next launch instead of returning it at
    // every synchronisation
    int dev = 0;
    cudaMemPool_t pool;
    PQI_TRY(cudaGetDevice(&dev));
    PQI_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t keep = UINT64_MAX;
    PQI_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pool_kept = true;
  }
  const int yp = (max_n + 3) & ~3;
  double* y = nullptr;
  PQI_TRY(cudaMallocAsync(reinterpret_cast<void**>(&y), (size_t)tasks * yp * sizeof(double), s));
  const dim3 grid((unsigned)((tasks + SF_T - 1) / SF_T), (unsigned)((max_n + SF_V - 1) / SF_V));
  if (i8) {
    start_fields_kernel<int8_t><<<grid, 256, 0, s>>>(gd, task_graph, init_states, words_pitch, tasks, y, yp);
  } else {
    start_fields_kernel<float><<<grid, 256, 0, s>>>(gd, task_graph, init_states, words_pitch, tasks, y, yp);
  }
  PQI_LAUNCHED("start_fields_kernel");
  *out = y;
  *pitch = yp;
  return PQI_OK;
}

static pqi_status batch_search_impl(const void* graphs, int num_graphs, const int* task_graph,
                                    const uint32_t* init_states, int words_pitch, int tasks,
                                    int max_n, int kind, int is_spin_glass, int rounds, int kick,
                                    int flip_budget, uint64_t seed, const double* kick_cdf,
                                    const long long* cdf_offset, uint32_t* best_states,
                                    double* best_values, unsigned long long* flips_total,
                                    int* status, void* stream, bool f32, int bt) {
  PQI_CHECK_ARG(bt == 256 || bt == 128 || bt == 64);
  PQI_CHECK_ARG(graphs && num_graphs > 0 && task_graph && init_states && tasks > 0 && max_n > 0);
  PQI_CHECK_ARG(best_states && best_values && flips_total && status && rounds >= 0 && kick >= 0);
  PQI_CHECK_ARG(words_pitch >= (max_n + 31) / 32 && flip_budget > 0);
  PQI_CHECK_ARG(!kick_cdf || cdf_offset);
  cudaStream_t s = as_stream(stream);
  const bool i8 = kind == PQI_W_I8;
  const size_t smem = (((size_t)((max_n + 31) >> 5) * 4 + 15) & ~size_t(15)) +
                      (size_t)((max_n + 4 * bt - 1) / (4 * bt) * (4 * bt)) *
                          (i8 ? sizeof(int) : (f32 ? sizeof(float) : sizeof(double))) +
                      (((size_t)((max_n + 31) >> 5) * 4 + 15) & ~size_t(15));  // kicked set of the round
  const int groups = (max_n + 4 * bt - 1) / (4 * bt);  // groups of four per thread
  // float32 fields beyond four groups: four more groups per pass staged in
  // shared memory (16 KB), all of SK n = 8192's row in flight per flip
  // (staging is skipped where its buffer would not fit: every row group in registers)
  const size_t stage_bytes = (size_t)kStageGroups * 256 * 4 * sizeof(float);
  const bool staged =
      bt == 256 && f32 && !i8 && groups > 4 && !g_batch_no_stage && smem + stage_bytes <= 200 * 1024;
  const size_t smem_all = smem + (staged ? stage_bytes : 0);
  PQI_CHECK_ARG(smem_all <= 200 * 1024);
  static int num_sms = 0;
  if (!num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  // persistent grid: exactly the CTAs that are resident at once
  int per_sm = 1;
  const BatchGraph* gd = static_cast<const BatchGraph*>(graphs);
  // the starting fields of dense-graph tasks as one pass over W per task tile
  double* sf = nullptr;
  int sf_pitch = 0;
  pqi_status sfst = start_fields(gd, task_graph, init_states, words_pitch, tasks, max_n, i8, s, &sf,
                                 &sf_pitch);
  if (sfst != PQI_OK) return sfst;
  // float weights with float64 fields and 4096 < n <= 16384: the fields in
  // tensor memory (four tasks per SM up to 8192 nodes, two up to 16384; each
  // flip's whole row in one bulk copy)
  if (!i8 && !f32 && bt == 256 && max_n > 4096 && max_n <= TmShape<32>::NMAX && sf &&
      !g_batch_no_tmem) {
    const bool small = max_n <= TmShape<16>::NMAX;
    const void* fn = small ? (const void*)batch_search_tmem_kernel<16> : (const void*)batch_search_tmem_kernel<32>;
    const int tsm = small ? TmShape<16>::SMEM : TmShape<32>::SMEM;
    PQI_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, tsm));
    PQI_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    // resident CTAs per SM: as many as the TMEM columns serve (shared memory
    // and registers allow them, and keep out one more; the occupancy query
    // reports one CTA per SM for a kernel that allocates tensor memory)
    int tper = 0;
    PQI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tper, fn, TM_BT, tsm));
    if (tper >= 1) {
      tper = small ? TmShape<16>::CTAS : TmShape<32>::CTAS;
      const int grid = std::max(1, std::min(tasks, num_sms * tper));
      if (small) {
        batch_search_tmem_kernel<16><<<grid, TM_BT, tsm, s>>>(
            gd, task_graph, init_states, words_pitch, tasks, is_spin_glass, rounds, kick, flip_budget,
            seed, kick_cdf, cdf_offset, best_states, best_values, flips_total, status, sf, sf_pitch);
      } else {
        batch_search_tmem_kernel<32><<<grid, TM_BT, tsm, s>>>(
            gd, task_graph, init_states, words_pitch, tasks, is_spin_glass, rounds, kick, flip_budget,
            seed, kick_cdf, cdf_offset, best_states, best_values, flips_total, status, sf, sf_pitch);
      }
      PQI_LAUNCHED("batch_search_tmem_kernel");
      PQI_TRY(cudaFreeAsync(sf, s));
      return PQI_OK;
    }
  }
  // row loads per thread: groups of four nodes, CH groups in flight per chunk
  // (the whole row for n <= 4 * 256 * CH). CH = 4 keeps three CTAs per SM
  // within the register file (8 groups spill at that occupancy and run slower
  // on SK n = 8192 than two chunks of 4).
#define PQI_BATCH_LAUNCH(WT_, CH_, F_, S_, BT_)                                                 \
  do {                                                                                         \
    PQI_TRY(cudaFuncSetAttribute(batch_search_kernel<WT_, CH_, F_, S_, BT_>,                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_all)); \
    PQI_TRY(cudaFuncSetAttribute(batch_search_kernel<WT_, CH_, F_, S_, BT_>,                   \
                                 cudaFuncAttributePreferredSharedMemoryCarveout, 100));        \
    PQI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(                                     \
        &per_sm, batch_search_kernel<WT_, CH_, F_, S_, BT_>, BT_, smem_all));                  \
    const int grid = std::max(1, std::min(tasks, num_sms * std::max(1, per_sm)));             \
    batch_search_kernel<WT_, CH_, F_, S_, BT_><<<grid, BT_, smem_all, s>>>(                    \
        gd, task_graph, init_states, words_pitch, tasks, is_spin_glass, rounds, kick,          \
        flip_budget, seed, kick_cdf, cdf_offset, best_states, best_values, flips_total,        \
        status, sf, sf_pitch);                                                                 \
  } while (0)
  if (bt == 64) {  // smallest graphs: four groups per thread cover n <= 1024
    if (i8) {
      if (groups <= 2) {
        PQI_BATCH_LAUNCH(int8_t, 2, false, false, 64);
      } else {
        PQI_BATCH_LAUNCH(int8_t, 4, false, false, 64);
      }
    } else if (f32) {
      if (groups <= 2) {
        PQI_BATCH_LAUNCH(float, 2, true, false, 64);
      } else {
        PQI_BATCH_LAUNCH(float, 4, true, false, 64);
      }
    } else {
      if (groups <= 2) {
        PQI_BATCH_LAUNCH(float, 2, false, false, 64);
      } else {
        PQI_BATCH_LAUNCH(float, 4, false, false, 64);
      }
    }
  } else if (bt == 128) {  // small graphs: two groups per thread cover n <= 1024
    if (i8) {
      if (groups <= 2) {
        PQI_BATCH_LAUNCH(int8_t, 2, false, false, 128);
      } else {
        PQI_BATCH_LAUNCH(int8_t, 4, false, false, 128);
      }
    } else if (f32) {
      if (groups <= 2) {
        PQI_BATCH_LAUNCH(float, 2, true, false, 128);
      } else {
        PQI_BATCH_LAUNCH(float, 4, true, false, 128);
      }
    } else {
      if (groups <= 2) {
        PQI_BATCH_LAUNCH(float, 2, false, false, 128);
      } else {
        PQI_BATCH_LAUNCH(float, 4, false, false, 128);
      }
    }
  } else if (i8) {
    if (groups <= 2) {
      PQI_BATCH_LAUNCH(int8_t, 2, false, false, 256);
    } else {
      PQI_BATCH_LAUNCH(int8_t, 4, false, false, 256);
    }
  } else if (f32) {
    if (groups <= 2) {
      PQI_BATCH_LAUNCH(float, 2, true, false, 256);
    } else if (staged) {
      PQI_BATCH_LAUNCH(float, 4, true, true, 256);
    } else {
      PQI_BATCH_LAUNCH(float, 4, true, false, 256);
    }
  } else {
    if (groups <= 2) {
      PQI_BATCH_LAUNCH(float, 2, false, false, 256);
    } else {
      PQI_BATCH_LAUNCH(float, 4, false, false, 256);
    }
  }
#undef PQI_BATCH_LAUNCH
  PQI_LAUNCHED("batch_search_kernel");
  if (sf) PQI_TRY(cudaFreeAsync(sf, s));
  return PQI_OK;
}

extern "C" {

pqi_status pqi_batch_set_start_pass(int on) {
  g_batch_no_start_pass = on ? 0 : 1;
  return PQI_OK;
}

pqi_status pqi_batch_set_staging(int on) {
  g_batch_no_stage = on ? 0 : 1;
  return PQI_OK;
}

pqi_status pqi_batch_set_tmem_fields(int on) {
  g_batch_no_tmem = on ? 0 : 1;
  return PQI_OK;
}

pqi_status pqi_batch_search(const void* graphs, int num_graphs, const int* task_graph,
                            const uint32_t* init_states, int words_pitch, int tasks, int max_n,
                            int kind, int is_spin_glass, int rounds, int kick, int flip_budget,
                            uint64_t seed, const double* kick_cdf, const long long* cdf_offset,
                            uint32_t* best_states, double* best_values,
                            unsigned long long* flips_total, int* status, void* stream) {
  return batch_search_impl(graphs, num_graphs, task_graph, init_states, words_pitch, tasks, max_n,
                           kind, is_spin_glass, rounds, kick, flip_budget, seed, kick_cdf,
                           cdf_offset, best_states, best_values, flips_total, status, stream,
                           false, 256);
}

pqi_status pqi_batch_search_f32(const void* graphs, int num_graphs, const int* task_graph,
                                const uint32_t* init_states, int words_pitch, int tasks,
                                int max_n, int kind, int is_spin_glass, int rounds, int kick,
                                int flip_budget, uint64_t seed, const double* kick_cdf,
                                const long long* cdf_offset, uint32_t* best_states,
                                double* best_values, unsigned long long* flips_total,
                                int* status, void* stream) {
  return batch_search_impl(graphs, num_graphs, task_graph, init_states, words_pitch, tasks, max_n,
                           kind, is_spin_glass, rounds, kick, flip_budget, seed, kick_cdf,
                           cdf_offset, best_states, best_values, flips_total, status, stream,
                           true, 256);
}

pqi_status pqi_batch_search_cta(const void* graphs, int num_graphs, const int* task_graph,
                                const uint32_t* init_states, int words_pitch, int tasks,
                                int max_n, int kind, int is_spin_glass, int rounds, int kick,
                                int flip_budget, uint64_t seed, const double* kick_cdf,
                                const long long* cdf_offset, uint32_t* best_states,
                                double* best_values, unsigned long long* flips_total,
                                int* status, int threads_per_task, int float32_fields,
                                void* stream) {
  return batch_search_impl(graphs, num_graphs, task_graph, init_states, words_pitch, tasks, max_n,
                           kind, is_spin_glass, rounds, kick, flip_budget, seed, kick_cdf,
                           cdf_offset, best_states, best_values, flips_total, status, stream,
                           float32_fields != 0, threads_per_task);
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
