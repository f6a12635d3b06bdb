// libpqi: the search path on a compressed-row (CSR) coupling matrix, for
// sparse graphs too large to hold as a dense n x n matrix. Replaces the
// reference's CSR kernels (pyqrackising/kernels.cl:233-414, 1072-1150) behind
// spin_glass_solver_sparse (pyqrackising/spin_glass_solver_sparse.py:517-864).
//
// Both triangles are stored (row r lists every neighbour once, columns
// ascending), so memory is O(n + nnz) and a flip touches only the flipped
// node's row: g_v -= 2 x_v x_k W_kv for each neighbour v, g_k = -g_k (8 bytes
// of the row per neighbour instead of n weights). Gains are float64 sums of
// the float32 weights (exact for integer weights).
//
// Semantics follow the dense entry points (pqi_core.cu, pqi_gray.cu): the same
// values, rounded to float32 where the reference compares in float32, and the
// same reference-order selection. The double-flip pass is exact over all
// n(n-1)/2 pairs with a 64-bit pair index, so it also covers n > 46341, where
// the reference's int32 pair count overflows (kernels.cl:197).
#include <algorithm>

#include "pqi_common.cuh"

namespace pqi {
namespace csr {

__device__ __forceinline__ int bit_at(const uint32_t* w, long long v) {
  return (int)((w[v >> 5] >> (v & 31)) & 1u);
}

// Gains of `count` states (grid.y): a warp per row, lanes over the row's
// entries; g_k = sum_v W_kv (s_k == s_v ? +1 : -1).
__global__ void gains_kernel(const long long* __restrict__ ptr, const int* __restrict__ col,
                             const float* __restrict__ val, int n,
                             const uint32_t* __restrict__ theta, int n32, float* __restrict__ g32,
                             double* __restrict__ g64) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const uint32_t* th = theta + (size_t)blockIdx.y * n32;
  for (int k = blockIdx.x * warps + (threadIdx.x >> 5); k < n; k += gridDim.x * warps) {
    const int xk = bit_at(th, k);
    double acc = 0.0;
    for (long long e = ptr[k] + lane; e < ptr[k + 1]; e += 32) {
      const double w = (double)__ldg(val + e);
      acc += (bit_at(th, __ldg(col + e)) == xk) ? w : -w;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) {
      if (g32) g32[(size_t)blockIdx.y * n + k] = (float)acc;
      if (g64) g64[(size_t)blockIdx.y * n + k] = acc;
    }
  }
}

// Flip node k of the block's state (all threads, same k): its neighbours'
// gains change, then g_k = -g_k and the bit toggles.
template <typename W>
__device__ __forceinline__ void block_flip(double* g, W* bits, const long long* __restrict__ ptr,
                                           const int* __restrict__ col,
                                           const float* __restrict__ val, int k) {
  constexpr int kShift = sizeof(W) == 8 ? 6 : 5;
  constexpr int kMask = sizeof(W) == 8 ? 63 : 31;
  const int xk = (int)((bits[k >> kShift] >> (k & kMask)) & 1);
  __syncthreads();
  for (long long e = ptr[k] + threadIdx.x; e < ptr[k + 1]; e += blockDim.x) {
    const int v = __ldg(col + e);
    const double w2 = 2.0 * (double)__ldg(val + e);
    const int xv = (int)((bits[v >> kShift] >> (v & kMask)) & 1);
    g[v] += (xv == xk) ? -w2 : w2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    g[k] = -g[k];
    bits[k >> kShift] ^= (W)1 << (k & kMask);
  }
  __syncthreads();
}

// Single CTA: repeat (best single flip under the reference geometry, flip it
// if its value is > 0) until none improves or max_flips is reached
// (spin_glass_solver_sparse.py:703-726, repeated).
//
// The nodes are cut into segments of `seg` nodes whose largest selection key
// stays in shared memory. A flip changes only the gains of the flipped node
// and its neighbours, so after it only their segments are rescanned (a warp
// per segment) and the next selection is a maximum over the segment keys:
// per flip O(degree * seg + n / seg) work instead of a pass over all n gains.
// The selected key is the same maximum over all nodes' keys.
__device__ __forceinline__ uint64_t segment_key(const double* __restrict__ g, int n, int seg, int q,
                                                int spin, const SelGeom& geo) {
  uint64_t best = 0;
  float bv = -INFINITY;
  const int k1 = min(n, (q + 1) * seg);
  for (int k = q * seg + (threadIdx.x & 31); k < k1; k += 32) {
    float v = (float)__ldcg(g + k);
    if (spin) v *= 2.0f;
    if (v >= bv) {  // a smaller value cannot give a larger key
      const uint64_t kk = sel_key(v, (uint64_t)k, geo);
      if (kk > best) {
        best = kk;
        bv = v;
      }
    }
  }
  return warp_max_u64(best);
}

__global__ void __launch_bounds__(1024) descent_kernel(
    const long long* __restrict__ ptr, const int* __restrict__ col, const float* __restrict__ val,
    int n, int seg, uint32_t* __restrict__ theta, double* __restrict__ g, int spin, SelGeom geo,
    int max_flips, double* __restrict__ energy_sum, int* __restrict__ flips,
    int* __restrict__ trace, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint64_t scratch[32];
  __shared__ int s_count;
  const int n32 = (n + 31) >> 5;
  const int nseg = (n + seg - 1) / seg;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint64_t* skey = reinterpret_cast<uint64_t*>(smem);
  int* list = reinterpret_cast<int*>(skey + nseg);
  uint8_t* dirty = reinterpret_cast<uint8_t*>(list + nseg);
  uint32_t* bits = reinterpret_cast<uint32_t*>(smem + (((size_t)nseg * 13 + 15) & ~size_t(15)));
  for (int q = threadIdx.x; q < n32; q += blockDim.x) bits[q] = theta[q];
  for (int q = threadIdx.x; q < nseg; q += blockDim.x) dirty[q] = 0;
  for (int q = warp; q < nseg; q += nwarps) {
    const uint64_t kq = segment_key(g, n, seg, q, spin, geo);
    if (lane == 0) skey[q] = kq;
  }
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  double esum = 0.0;
  int cnt = 0, st = PQI_OK;
  while (true) {
    uint64_t best = 0;
    for (int q = threadIdx.x; q < nseg; q += blockDim.x) best = skey[q] > best ? skey[q] : best;
    best = block_max_u64(best, scratch);
    float v;
    int64_t idx;
    sel_decode(best, geo, &v, &idx);
    if (!(v > 0.0f)) break;
    if (cnt >= max_flips) {
      st = PQI_ETIMEOUT;
      break;
    }
    esum += (double)v;
    if (threadIdx.x == 0 && trace) trace[cnt] = (int)idx;
    ++cnt;
    // the flip, marking the segments whose gains change
    const int k = (int)idx;
    const int xk = bit_at(bits, k);
    if (threadIdx.x == 0) dirty[k / seg] = 1;
    for (long long e = ptr[k] + threadIdx.x; e < ptr[k + 1]; e += blockDim.x) {
      const int u = __ldg(col + e);
      const double w2 = 2.0 * (double)__ldg(val + e);
      g[u] += (bit_at(bits, u) == xk) ? -w2 : w2;
      dirty[u / seg] = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // after the row's updates (as block_flip)
      g[k] = -g[k];
      bits[k >> 5] ^= 1u << (k & 31);
    }
    for (int q = threadIdx.x; q < nseg; q += blockDim.x) {
      if (dirty[q]) {
        dirty[q] = 0;
        list[atomicAdd(&s_count, 1)] = q;
      }
    }
    __syncthreads();
    const int nd = s_count;
    for (int i = warp; i < nd; i += nwarps) {
      const int q = list[i];
      const uint64_t kq = segment_key(g, n, seg, q, spin, geo);
      if (lane == 0) skey[q] = kq;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_count = 0;
  }
  for (int q = threadIdx.x; q < n32; q += blockDim.x) theta[q] = bits[q];
  if (threadIdx.x == 0) {
    *energy_sum = esum;
    *flips = cnt;
    *status = st;
  }
}

// Apply one or two flips to (theta, gains): one block.
__global__ void apply_flip_kernel(const long long* __restrict__ ptr, const int* __restrict__ col,
                                  const float* __restrict__ val, uint32_t* theta, double* g,
                                  int k, int l) {
  block_flip<uint32_t>(g, theta, ptr, col, val, k);
  if (l >= 0) block_flip<uint32_t>(g, theta, ptr, col, val, l);
}

// Gray search, one CTA per seed (grid-stride), the dense gray kernel's walk
// (kernels.cl:894-978 semantics; see pqi_gray.cu) with CSR flips. The 64-bit
// state words sit in shared memory, the seed's gains in g_all + block * n.
__global__ void __launch_bounds__(256) gray_kernel(
    const long long* __restrict__ ptr, const int* __restrict__ col, const float* __restrict__ val,
    int n, const uint64_t* __restrict__ theta64, const double* __restrict__ base_g, int spin,
    long long iters_bound, int S, uint64_t* __restrict__ theta_out,
    float* __restrict__ energy_out, double* __restrict__ g_all) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int blocks = (n + 63) >> 6;
  uint64_t* bits = reinterpret_cast<uint64_t*>(smem);
  double* g = g_all + (size_t)blockIdx.x * n;
  const int lane = threadIdx.x & 31;
  for (int s = blockIdx.x; s < S; s += gridDim.x) {
    for (int q = threadIdx.x; q < blocks; q += blockDim.x) bits[q] = theta64[q];
    for (int v = threadIdx.x; v < n; v += blockDim.x) g[v] = base_g[v];
    __syncthreads();
    // the seed mask of work-item s: 32-bit int shift, sign-extended at 31
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
    double E = 0.0;
    for (int q = 0; q < 2; ++q) {
      uint64_t mq = m[q];
      while (mq) {
        const int p = __ffsll((long long)mq) - 1;
        mq &= mq - 1;
        const int node = ((w0 + q) << 6) + p;
        if (node < n) {
          E += g[node];
          block_flip<uint64_t>(g, bits, ptr, col, val, node);
        } else if (node < (blocks << 6)) {
          __syncthreads();
          if (threadIdx.x == 0) bits[node >> 6] ^= 1ull << (node & 63);
          __syncthreads();
        }
      }
    }
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
        if (k < n) pos = g[k] > 0.0;
      }
      const unsigned bal = __ballot_sync(0xFFFFFFFFu, pos);
      if (!bal) {
        p0 += 32;
        continue;
      }
      const int f = __ffs(bal) - 1;
      const int kk = __shfl_sync(0xFFFFFFFFu, k, f);
      E += g[kk];
      block_flip<uint64_t>(g, bits, ptr, col, val, kk);
      p0 += f + 1;
    }
    for (int q = threadIdx.x; q < blocks; q += blockDim.x) theta_out[(size_t)s * blocks + q] = bits[q];
    if (threadIdx.x == 0) energy_out[s] = (float)(spin ? E : E / 2.0);
    __syncthreads();
  }
}

// float64 cut and energy of `rows` states: one block per state, each stored
// entry (both triangles) counted once, so every edge twice.
__global__ void rescore_kernel(const long long* __restrict__ ptr, const int* __restrict__ col,
                               const float* __restrict__ val, int n,
                               const uint32_t* __restrict__ words, int n32,
                               double* __restrict__ cut, double* __restrict__ energy) {
  __shared__ double sc[32], se[32];
  const uint32_t* th = words + (size_t)blockIdx.x * n32;
  double c = 0.0, e = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const int xr = bit_at(th, r);
    for (long long q = ptr[r]; q < ptr[r + 1]; ++q) {
      const double w = (double)__ldg(val + q);
      if (bit_at(th, __ldg(col + q)) != xr) {
        c += w;
        e += w;
      } else {
        e -= w;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sc[warp] = c;
    se[warp] = e;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tc = 0.0, te = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      tc += sc[i];
      te += se[i];
    }
    cut[blockIdx.x] = tc / 2.0;
    energy[blockIdx.x] = te / 2.0;
  }
}

// Candidate scoring (calculate_cut semantics, kernels.cl:44-94, on CSR): value
// = sum over edges u < v of W_uv where the edge is cut, and -W_uv where it is
// not (spin glass only); one block per candidate, float64 sum rounded to
// float32 (exact for integer weights).
__global__ void score_kernel(const long long* __restrict__ ptr, const int* __restrict__ col,
                             const float* __restrict__ val, int n,
                             const uint32_t* __restrict__ theta, int n32, int shots, int spin,
                             float* __restrict__ out) {
  __shared__ double part[32];
  for (int b = blockIdx.x; b < shots; b += gridDim.x) {
    const uint32_t* th = theta + (size_t)b * n32;
    double acc = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const int xr = bit_at(th, r);
      for (long long q = ptr[r]; q < ptr[r + 1]; ++q) {
        const int v = __ldg(col + q);
        if (v <= r) continue;  // each edge once: its upper-triangle entry
        const double w = (double)__ldg(val + q);
        if (bit_at(th, v) != xr) {
          acc += w;
        } else if (spin) {
          acc -= w;
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
      out[b] = (float)t;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Double flips over all pairs k < l: value(k, l) = float(g_k + g_l - 2 s W_kl)
// (s = +1 when the bits agree, else -1; x2 for a spin glass), selected as the
// maximum value, then the smallest tie priority of the reference geometry
// computed in 64 bits (pair index c = k(n-1) - k(k-1)/2 + (l-k-1)).
//
// Most pairs are not adjacent (W_kl = 0): the pair tiles stream only the gains
// (float32 copies, L2-resident) and take the exact value of a pair only when
// its fp32 estimate f_k + f_l could reach the running threshold (the bound of
// the dense pass, pqi_core.cu); adjacent pairs are all taken exactly by a
// separate pass over the stored entries. Phase 1 finds the maximum value,
// phase 2 the smallest priority among the pairs that reach it.

constexpr int DR = 8;
constexpr int DT = 256;
constexpr int VEC = 4;
constexpr int CW = VEC * DT;

struct PairGeom {
  uint32_t G, L;
  unsigned long long J;  // ceil(pairs / G)
  uint8_t rank[64];
};

// Tie priority of pair index c (smaller wins), or ~0 when the pair's work-item
// slot never reaches its group's slot 0 (never selected).
__device__ __forceinline__ unsigned long long pair_prio(unsigned long long c, const PairGeom& g) {
  const unsigned long long t = c % g.G, j = c / g.G;
  const uint32_t grp = (uint32_t)(t / g.L);
  const uint32_t r = g.rank[t - (unsigned long long)grp * g.L];
  if (r == 0xFFu) return ~0ull;
  return ((unsigned long long)grp * g.L + r) * g.J + j;
}

__device__ __forceinline__ long long pair_index(long long k, long long l, long long n) {
  return k * (n - 1) - (k * (k - 1)) / 2 + (l - k - 1);
}

// W_kl from row k (binary search), 0 when not adjacent.
__device__ __forceinline__ float weight_of(const long long* __restrict__ ptr,
                                           const int* __restrict__ col,
                                           const float* __restrict__ val, int k, int l) {
  long long lo = ptr[k], hi = ptr[k + 1];
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    const int c = __ldg(col + mid);
    if (c < l) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return (lo < ptr[k + 1] && __ldg(col + lo) == l) ? __ldg(val + lo) : 0.0f;
}

struct PairState {
  unsigned int* vmax;          // ordered float32 of the maximum (phase 1 result)
  unsigned long long* prio;    // smallest priority at the maximum (phase 2)
  unsigned int* thr;           // phase 1: shared threshold (ordered, unscaled value)
  unsigned int* bound;         // ordered: [0] max f_k, [1] max |f_k|, then the row
                               // groups' max f_k ([2, 2 + ng)), then the column
                               // chunks' max f_k ([2 + ng, 2 + ng + nc))
  int positive;                // only pairs of value > 0 are wanted
};

__device__ __forceinline__ float thr_of(uint32_t o) {
  return o < ord_f32(-INFINITY) ? -INFINITY : unord_f32(o);
}

// Exact value of pair (k, l), unscaled and as the reference's (scaled) float.
__device__ __forceinline__ void pair_value(double gk, double gl, float w, int xk, int xl, int spin,
                                           float* unscaled, float* scaled) {
  const double wd = (double)w;
  const double d = gk + gl - ((xk == xl) ? 2.0 * wd : -2.0 * wd);
  float v = (float)d;
  *unscaled = v;
  if (spin) v *= 2.0f;
  *scaled = v;
}

// Adjacent pairs: a warp per row k, lanes over entries with l > k.
template <int PHASE>
__global__ void pair_edges_kernel(const long long* __restrict__ ptr, const int* __restrict__ col,
                                  const float* __restrict__ val, int n,
                                  const uint32_t* __restrict__ theta,
                                  const double* __restrict__ g64, int spin, PairGeom geo,
                                  PairState ps) {
  const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  unsigned int best_o = 0;
  unsigned long long best_p = ~0ull;
  const unsigned int target = PHASE == 2 ? *ps.vmax : 0u;
  for (int k = blockIdx.x * warps + (threadIdx.x >> 5); k < n; k += gridDim.x * warps) {
    const int xk = bit_at(theta, k);
    const double gk = g64[k];
    for (long long e = ptr[k] + lane; e < ptr[k + 1]; e += 32) {
      const int l = __ldg(col + e);
      if (l <= k) continue;
      float vu, vs;
      pair_value(gk, __ldg(g64 + l), __ldg(val + e), xk, bit_at(theta, l), spin, &vu, &vs);
      const unsigned long long pr = pair_prio((unsigned long long)pair_index(k, l, n), geo);
      if (pr == ~0ull || vs != vs) continue;
      const unsigned int o = ord_f32(vs);
      if (PHASE == 1) {
        best_o = o > best_o ? o : best_o;
      } else if (o == target && pr < best_p) {
        best_p = pr;
      }
      (void)vu;
    }
  }
  if (PHASE == 1) {
    for (int o = 16; o > 0; o >>= 1) best_o = max(best_o, __shfl_xor_sync(0xFFFFFFFFu, best_o, o));
    if (lane == 0 && best_o) {
      atomicMax(ps.vmax, best_o);
      // seed the pair tiles' threshold with this (unscaled) value
      const float vs = unord_f32(best_o);
      atomicMax(ps.thr, ord_f32(spin ? vs * 0.5f : vs));
    }
  } else {
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xFFFFFFFFu, best_p, o);
      best_p = other < best_p ? other : best_p;
    }
    if (lane == 0 && best_p != ~0ull) atomicMin(ps.prio, best_p);
  }
}

// All pairs in tiles of DR rows x CW columns (the upper triangle), gains only.
// The float32 gains f_k are rounded up from the float64 gains (f_k >= g_k), so
// the fp32 estimate of a non-adjacent pair is > 0 whenever its value is, and
// the largest f_k of a row group plus that of a column chunk bounds every
// estimate of their tile: a row group or a tile whose bound is below the cut
// is passed over without loading its gains.
template <int PHASE>
__global__ void __launch_bounds__(DT) pair_tiles_kernel(
    const long long* __restrict__ ptr, const int* __restrict__ col, const float* __restrict__ val,
    int n, const uint32_t* __restrict__ theta, const double* __restrict__ g64,
    const float* __restrict__ g32, int spin, PairGeom geo, PairState ps) {
  __shared__ unsigned int s_thr;
  if (threadIdx.x == 0) s_thr = 0u;
  __syncthreads();
  const int ng = (n - 1 + DR - 1) / DR;
  const int nc = (n + CW - 1) / CW;
  unsigned int best_o = 0;
  unsigned long long best_p = ~0ull;
  // phase 2 looks for the pairs whose scaled value is vmax
  const unsigned int target = PHASE == 2 ? *ps.vmax : 0u;
  const float vt = PHASE == 2 ? thr_of(target) : 0.0f;
  if (PHASE == 2 && (target == 0u || (ps.positive && !(vt > 0.0f)))) return;
  // positive: an estimate must be > 0 (>= the smallest positive float)
  const float floor_cut = ps.positive ? __int_as_float(1) : -INFINITY;
  const float gmax = thr_of(ps.bound[0]);
  const float gabs = thr_of(ps.bound[1]);
  const unsigned int* rgmax = ps.bound + 2;
  const unsigned int* cmax = rgmax + ng;
  float thr = PHASE == 2 ? (spin ? vt * 0.5f : vt) : -INFINITY;
  for (int rg = blockIdx.x; rg < ng; rg += gridDim.x) {
    const int k0 = rg * DR;
    const float rmax = thr_of(__ldg(rgmax + rg));
    if (PHASE == 1) thr = fmaxf(thr, thr_of(max(*(volatile unsigned int*)&s_thr, __ldcg(ps.thr))));
    // (a cut at least as low as every tile's: its base bounds every base below)
    const float row_cut = fmaxf(thr - ldexpf(2.0f * gabs + fabsf(thr), -20), floor_cut);
    if (!(rmax + gmax >= row_cut)) continue;
    // the first column chunk with a column above the group's first row
    for (int c = (k0 + 1) / CW; c < nc; ++c) {
      if (PHASE == 1) thr = fmaxf(thr, thr_of(max(*(volatile unsigned int*)&s_thr, __ldcg(ps.thr))));
      const float tile_cut = fmaxf(thr - ldexpf(2.0f * gabs + fabsf(thr), -20), floor_cut);
      if (!(rmax + thr_of(__ldg(cmax + c)) >= tile_cut)) continue;
      const int l0 = c * CW + threadIdx.x * VEC;
      float fk[DR];
      float gt = 0.0f;
#pragma unroll
      for (int i = 0; i < DR; ++i) {
        fk[i] = __ldg(g32 + min(k0 + i, n - 1));
        gt = fmaxf(gt, fabsf(fk[i]));
      }
      float fl[VEC];
      float flmax = 0.0f;
#pragma unroll
      for (int e = 0; e < VEC; ++e) {
        fl[e] = (l0 + e < n) ? __ldg(g32 + l0 + e) : -INFINITY;
        if (l0 + e < n) flmax = fmaxf(flmax, fabsf(fl[e]));
      }
      const float base = gt + flmax;
      float cut = fmaxf(thr - ldexpf(base + fabsf(thr), -20), floor_cut);
#pragma unroll
      for (int i = 0; i < DR; ++i) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
          const float a = fk[i] + fl[e];
          if (a >= cut) {
            const int k = k0 + i, l = l0 + e;
            if (k < n - 1 && l > k && l < n) {
              float vu, vs;
              pair_value(__ldg(g64 + k), __ldg(g64 + l), weight_of(ptr, col, val, k, l),
                         bit_at(theta, k), bit_at(theta, l), spin, &vu, &vs);
              const unsigned long long pr =
                  pair_prio((unsigned long long)pair_index(k, l, n), geo);
              if (pr != ~0ull && vs == vs) {
                const unsigned int o = ord_f32(vs);
                if (PHASE == 1) {
                  best_o = o > best_o ? o : best_o;
                  if (vu > thr) {
                    thr = vu;
                    cut = fmaxf(thr - ldexpf(base + fabsf(thr), -20), floor_cut);
                  }
                } else if (o == target && pr < best_p) {
                  best_p = pr;
                }
              }
            }
          }
        }
      }
      if (PHASE == 1 && thr > -INFINITY) {
        const unsigned int o = ord_f32(thr);
        if (o > *(volatile unsigned int*)&s_thr) {
          atomicMax(&s_thr, o);
          if (o > __ldcg(ps.thr)) atomicMax(ps.thr, o);
        }
      }
    }
  }
  if (PHASE == 1) {
    for (int o = 16; o > 0; o >>= 1) best_o = max(best_o, __shfl_xor_sync(0xFFFFFFFFu, best_o, o));
    if ((threadIdx.x & 31) == 0 && best_o) atomicMax(ps.vmax, best_o);
  } else {
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xFFFFFFFFu, best_p, o);
      best_p = other < best_p ? other : best_p;
    }
    if ((threadIdx.x & 31) == 0 && best_p != ~0ull) atomicMin(ps.prio, best_p);
  }
}

__global__ void pair_finish_kernel(PairState ps, PairGeom geo, float* best_energy,
                                   long long* best_index) {
  const unsigned int o = *ps.vmax;
  const unsigned long long pr = *ps.prio;
  if (o == 0u || pr == ~0ull) {
    *best_energy = -INFINITY;
    *best_index = -1;
    return;
  }
  *best_energy = unord_f32(o);
  const unsigned long long j = pr % geo.J, gr = pr / geo.J;
  const unsigned long long grp = gr / geo.L, r = gr - grp * geo.L;
  unsigned long long slot = 0;
  for (uint32_t t = 0; t < geo.L; ++t)
    if (geo.rank[t] == r) slot = t;
  *best_index = (long long)(grp * geo.L + slot + j * geo.G);
}

// The sparse path's J_eff and degrees (maxcut_tfim_sparse.py:204-224) over the
// stored rows S (as the caller stores them, columns ascending): the dense
// rule of pqi_tfim_jz_f32 - every entry m of row r, stored or zero, counts
// when S_rm - gmin > eps, summed in float32 in column order, J = -(sum /
// degree) in float32 - with the zeros between stored entries added one by one
// (when gmin < 0 they count), so the float32 sums are the reference's.
// One thread per row.
__global__ void tfim_jz_kernel(const long long* __restrict__ ptr, const int* __restrict__ col,
                               const float* __restrict__ val, int n, float gmin,
                               double* __restrict__ J_eff, unsigned int* __restrict__ degrees) {
  const float zero_val = __fsub_rn(0.0f, gmin);
  const bool zero_counts = (double)zero_val > 1.1920928955078125e-07;  // eps = 2^-23
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    unsigned int deg = 0;
    float J = 0.0f;
    long long e = ptr[r];
    const long long e1 = ptr[r + 1];
    int m = 0;
    while (m < n) {
      const int next = e < e1 ? __ldg(col + e) : n;
      if (zero_counts) {
        for (; m < next; ++m) {  // zeros before the next stored entry
          ++deg;
          J = __fadd_rn(J, zero_val);
        }
      }
      m = next;
      if (m >= n) break;
      const float v = __fsub_rn(__ldg(val + e), gmin);
      if ((double)v > 1.1920928955078125e-07) {
        ++deg;
        J = __fadd_rn(J, v);
      }
      ++e;
      ++m;
    }
    J_eff[r] = deg > 0 ? (double)(-__fdiv_rn(J, (float)deg)) : 0.0;
    degrees[r] = deg;
  }
}

// f_k = g_k rounded up to float32, and the bounds the pair tiles skip by: the
// largest f_k and |f_k| overall, per row group of DR and per column chunk of
// CW (ordered float32, the bound array zeroed beforehand). Whole warps walk
// 32 consecutive gains (DR and CW divide by the warp's 32).
__global__ void gains_f32_bounds_kernel(const double* __restrict__ a, float* __restrict__ b, int n,
                                        unsigned int* __restrict__ bound) {
  const int lane = threadIdx.x & 31;
  const int ng = (n - 1 + DR - 1) / DR;
  for (long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) & ~31ll; w0 < n;
       w0 += (long long)gridDim.x * blockDim.x) {
    const long long i = w0 + lane;
    float f = -INFINITY;
    if (i < n) {
      f = __double2float_ru(a[i]);
      b[i] = f;
    }
    float r = f, m = i < n ? fabsf(f) : 0.0f;
    for (int o = 1; o < DR; o <<= 1) r = fmaxf(r, __shfl_xor_sync(0xFFFFFFFFu, r, o));
    if ((lane & (DR - 1)) == 0 && i / DR < ng) bound[2 + i / DR] = ord_f32(r);
    float c = r;
    for (int o = DR; o < 32; o <<= 1) c = fmaxf(c, __shfl_xor_sync(0xFFFFFFFFu, c, o));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if (lane == 0) {
      const unsigned int oc = ord_f32(c);
      atomicMax(bound + 2 + ng + w0 / CW, oc);
      atomicMax(bound, oc);
      atomicMax(bound + 1, ord_f32(m));
    }
  }
}

static int grid_of(long long work, int per_block, int cap) {
  return (int)std::max<long long>(1, std::min<long long>((work + per_block - 1) / per_block, cap));
}

static bool check_graph(const pqi_csr* g) {
  return g && g->ptr && g->n > 0 && g->nnz >= 0 && (g->nnz == 0 || (g->col && g->val));
}

}  // namespace csr
}  // namespace pqi

using namespace pqi;
using namespace pqi::csr;

extern "C" {

pqi_status pqi_csr_gains(const pqi_csr* g, const uint32_t* theta, int count, float* g32,
                         double* g64, void* stream) {
  PQI_CHECK_ARG(check_graph(g) && theta && count > 0 && (g32 || g64));
  const int n = g->n;
  dim3 grid((unsigned)grid_of(n, 8, 148 * 8), (unsigned)count);
  gains_kernel<<<grid, 256, 0, as_stream(stream)>>>(g->ptr, g->col, g->val, n, theta, (n + 31) >> 5,
                                                    g32, g64);
  PQI_LAUNCHED("csr gains_kernel");
  return PQI_OK;
}

pqi_status pqi_csr_single_bit_flips(const pqi_csr* g, const uint32_t* theta, int is_spin_glass,
                                    int global_size, int local_size, float* best_energy,
                                    int* best_index, void* workspace, size_t workspace_bytes,
                                    void* stream) {
  PQI_CHECK_ARG(check_graph(g) && theta);
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(g->n, global_size, local_size, &geo));
  Workspace ws(workspace, workspace_bytes);
  unsigned long long* key = ws.take<unsigned long long>(1);
  float* g32 = ws.take<float>(g->n);
  PQI_CHECK_ARG(key && g32);
  pqi_status rc = pqi_csr_gains(g, theta, 1, g32, nullptr, stream);
  if (rc) return rc;
  return launch_select(g32, g->n, is_spin_glass ? 2.0f : 1.0f, geo, key, best_energy, best_index,
                       as_stream(stream));
}

pqi_status pqi_csr_apply_flip(const pqi_csr* g, uint32_t* theta, double* gains64, int k, int l,
                              void* stream) {
  PQI_CHECK_ARG(check_graph(g) && theta && gains64 && k >= 0 && k < g->n && l < g->n && l != k);
  apply_flip_kernel<<<1, 256, 0, as_stream(stream)>>>(g->ptr, g->col, g->val, theta, gains64, k, l);
  PQI_LAUNCHED("csr apply_flip_kernel");
  return PQI_OK;
}

pqi_status pqi_csr_single_descent(const pqi_csr* g, uint32_t* theta, double* gains64,
                                  int is_spin_glass, int global_size, int local_size,
                                  int max_flips, double* energy_sum, int* flips, int* trace,
                                  void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(check_graph(g) && theta && gains64 && energy_sum && flips && max_flips >= 0);
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(g->n, global_size, local_size, &geo));
  Workspace ws(workspace, workspace_bytes);
  int* status = ws.take<int>(1);
  PQI_CHECK_ARG(status);
  // segments of 256 nodes, wider when the segment keys, the rescan list and
  // the dirty flags (13 bytes per segment) and the state bits (n / 8 bytes)
  // would not fit in shared memory
  const size_t bits_bytes = (((size_t)((g->n + 31) >> 5) * 4 + 15) & ~size_t(15));
  int seg = 256;
  auto smem_of = [&](int sg) {
    const size_t nseg = ((size_t)g->n + sg - 1) / sg;
    return ((nseg * 13 + 15) & ~size_t(15)) + bits_bytes;
  };
  while (smem_of(seg) > 200 * 1024 && seg < (1 << 20)) seg *= 2;
  const size_t smem = smem_of(seg);
  PQI_CHECK_ARG(smem <= 200 * 1024);
  cudaStream_t s = as_stream(stream);
  PQI_TRY(cudaFuncSetAttribute(descent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  descent_kernel<<<1, 1024, smem, s>>>(g->ptr, g->col, g->val, g->n, seg, theta, gains64,
                                       is_spin_glass, geo, max_flips, energy_sum, flips, trace,
                                       status);
  PQI_LAUNCHED("csr descent_kernel");
  int hst = 0;
  PQI_TRY(cudaMemcpyAsync(&hst, status, sizeof(int), cudaMemcpyDeviceToHost, s));
  PQI_TRY(cudaStreamSynchronize(s));
  return (pqi_status)hst;
}

static pqi_status csr_double(const pqi_csr* g, const uint32_t* theta, const double* gains64,
                             int is_spin_glass, int global_size, int local_size, int positive,
                             float* best_energy, long long* best_index, void* workspace,
                             size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(check_graph(g) && theta && best_energy && best_index && g->n >= 2);
  const int n = g->n;
  SelGeom sg;
  PQI_CHECK_ARG(make_sel_geom(1, global_size, local_size, &sg));  // (the slot ranks only)
  PairGeom geo;
  geo.G = (uint32_t)global_size;
  geo.L = (uint32_t)local_size;
  const unsigned long long pairs = (unsigned long long)n * (unsigned long long)(n - 1) / 2ull;
  geo.J = std::max<unsigned long long>(1ull, (pairs + geo.G - 1) / geo.G);
  memcpy(geo.rank, sg.rank, sizeof(geo.rank));
  const int ng = (n - 1 + DR - 1) / DR, nc = (n + CW - 1) / CW;
  const size_t nbound = 2 + (size_t)ng + nc;
  Workspace ws(workspace, workspace_bytes);
  unsigned long long* ctl = ws.take<unsigned long long>(2);  // prio, then vmax | thr
  unsigned int* bound = ws.take<unsigned int>(nbound);
  float* g32 = ws.take<float>(n);
  double* gown = gains64 ? nullptr : ws.take<double>(n);
  PQI_CHECK_ARG(ctl && bound && g32 && (gains64 || gown));
  cudaStream_t s = as_stream(stream);
  if (!gains64) {
    pqi_status rc = pqi_csr_gains(g, theta, 1, nullptr, gown, stream);
    if (rc) return rc;
    gains64 = gown;
  }
  PairState ps;
  ps.prio = ctl;
  ps.vmax = reinterpret_cast<unsigned int*>(ctl + 1);
  ps.thr = ps.vmax + 1;
  ps.bound = bound;
  ps.positive = positive;
  PQI_TRY(cudaMemsetAsync(ctl, 0xFF, 8, s));      // prio = ~0
  PQI_TRY(cudaMemsetAsync(ctl + 1, 0, 8, s));     // vmax = thr = 0 (nothing yet)
  PQI_TRY(cudaMemsetAsync(bound, 0, nbound * sizeof(unsigned int), s));
  gains_f32_bounds_kernel<<<grid_of(n, 256, 148 * 4), 256, 0, s>>>(gains64, g32, n, bound);
  PQI_LAUNCHED("csr gains_f32_bounds_kernel");
  const int eg = grid_of(n, 8, 148 * 8);
  static int resident = 0;
  if (!resident) {
    int dev = 0, sms = 0, per = 0;
    PQI_TRY(cudaGetDevice(&dev));
    PQI_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PQI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pair_tiles_kernel<1>, DT, 0));
    resident = std::max(1, sms * std::max(1, per));
  }
  pair_edges_kernel<1><<<eg, 256, 0, s>>>(g->ptr, g->col, g->val, n, theta, gains64, is_spin_glass, geo, ps);
  PQI_LAUNCHED("csr pair_edges_kernel");
  pair_tiles_kernel<1><<<resident, DT, 0, s>>>(g->ptr, g->col, g->val, n, theta, gains64, g32,
                                                is_spin_glass, geo, ps);
  PQI_LAUNCHED("csr pair_tiles_kernel");
  pair_edges_kernel<2><<<eg, 256, 0, s>>>(g->ptr, g->col, g->val, n, theta, gains64, is_spin_glass, geo, ps);
  PQI_LAUNCHED("csr pair_edges_kernel");
  pair_tiles_kernel<2><<<resident, DT, 0, s>>>(g->ptr, g->col, g->val, n, theta, gains64, g32,
                                                is_spin_glass, geo, ps);
  PQI_LAUNCHED("csr pair_tiles_kernel");
  pair_finish_kernel<<<1, 1, 0, s>>>(ps, geo, best_energy, best_index);
  PQI_LAUNCHED("csr pair_finish_kernel");
  return PQI_OK;
}

pqi_status pqi_csr_double_bit_flips(const pqi_csr* g, const uint32_t* theta, const double* gains64,
                                    int is_spin_glass, int global_size, int local_size,
                                    float* best_energy, long long* best_index, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  return csr_double(g, theta, gains64, is_spin_glass, global_size, local_size, 0, best_energy,
                    best_index, workspace, workspace_bytes, stream);
}

pqi_status pqi_csr_improving_double_flip(const pqi_csr* g, const uint32_t* theta,
                                         const double* gains64, int is_spin_glass,
                                         int global_size, int local_size, float* best_energy,
                                         long long* best_index, void* workspace,
                                         size_t workspace_bytes, void* stream) {
  return csr_double(g, theta, gains64, is_spin_glass, global_size, local_size, 1, best_energy,
                    best_index, workspace, workspace_bytes, stream);
}

pqi_status pqi_csr_gray(const pqi_csr* g, const uint64_t* theta64, const double* gains64,
                        int is_spin_glass, long long iters_bound, int seeds, uint64_t* theta_out,
                        float* energy_out, void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(check_graph(g) && theta64 && gains64 && theta_out && energy_out && seeds > 0 &&
                iters_bound >= 0);
  const int n = g->n;
  const size_t smem = (size_t)((n + 63) >> 6) * 8;
  PQI_CHECK_ARG(smem <= 200 * 1024);
  Workspace ws(workspace, workspace_bytes);
  const size_t avail = (ws.size > ws.used + 256) ? (ws.size - ws.used - 256) : 0;
  const long long ctas = (long long)(avail / ((size_t)n * sizeof(double)));
  PQI_CHECK_ARG(ctas >= 1);
  const int grid = (int)std::min<long long>(std::min<long long>(ctas, seeds), 148 * 4);
  double* gall = ws.take<double>((size_t)grid * n);
  PQI_CHECK_ARG(gall);
  cudaStream_t s = as_stream(stream);
  PQI_TRY(cudaFuncSetAttribute(gray_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  gray_kernel<<<grid, 256, smem, s>>>(g->ptr, g->col, g->val, n, theta64, gains64, is_spin_glass,
                                      iters_bound, seeds, theta_out, energy_out, gall);
  PQI_LAUNCHED("csr gray_kernel");
  return PQI_OK;
}

pqi_status pqi_csr_rescore_fp64(const pqi_csr* g, const uint32_t* words, int rows, double* cut,
                                double* energy, void* stream) {
  PQI_CHECK_ARG(check_graph(g) && words && rows > 0 && cut && energy);
  rescore_kernel<<<rows, 256, 0, as_stream(stream)>>>(g->ptr, g->col, g->val, g->n, words,
                                                      (g->n + 31) >> 5, cut, energy);
  PQI_LAUNCHED("csr rescore_kernel");
  return PQI_OK;
}

pqi_status pqi_csr_tfim_jz(const long long* ptr, const int* col, const float* val, int n, float gmin,
                          double* J_eff, unsigned int* degrees, void* stream) {
  PQI_CHECK_ARG(ptr && n > 0 && J_eff && degrees);
  tfim_jz_kernel<<<grid_of(n, 128, 148 * 16), 128, 0, as_stream(stream)>>>(ptr, col, val, n, gmin,
                                                                           J_eff, degrees);
  PQI_LAUNCHED("csr tfim_jz_kernel");
  return PQI_OK;
}

pqi_status pqi_csr_calculate_cut(const pqi_csr* g, const uint32_t* theta, int shots,
                                 int is_spin_glass, int global_size, int local_size,
                                 float* energies, float* best_energy, int* best_index,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  PQI_CHECK_ARG(check_graph(g) && theta && shots > 0);
  SelGeom geo;
  PQI_CHECK_ARG(make_sel_geom(shots, global_size, local_size, &geo));
  Workspace ws(workspace, workspace_bytes);
  unsigned long long* key = ws.take<unsigned long long>(1);
  float* vals = energies ? energies : ws.take<float>(shots);
  PQI_CHECK_ARG(key && vals);
  cudaStream_t s = as_stream(stream);
  score_kernel<<<grid_of(shots, 1, 148 * 8), 256, 0, s>>>(g->ptr, g->col, g->val, g->n, theta,
                                                          (g->n + 31) >> 5, shots, is_spin_glass,
                                                          vals);
  PQI_LAUNCHED("csr score_kernel");
  return launch_select(vals, shots, 1.0f, geo, key, best_energy, best_index, s);
}

}  // extern "C"
